/*
 * CPU oracle for the sparse solver path of nickreserved/CompressionTests.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py (its
 * cpu_baseline leg and --impl reference) may load it.  The product library
 * (compressiontests_b200/libduvigpu.so) never links, loads or calls it.
 *
 * It is a faithful, single-threaded restatement of the reference's CPU
 * algorithms (C#, not buildable here: no dotnet/mono), compiled with
 * -ffp-contract=off so that every multiply and add rounds separately, as the
 * .NET JIT does.  Each function cites the reference file:line it follows.
 * Parity against the reference itself is pinned by the reference's own
 * known-answer tests (tests/test_oracle_golden.py):
 *   - DuVi 2x1024 KAT          CompressedSparseMatrixTests.cs:15-39
 *   - diagonal CSR KAT         GMCantileverOpenCLTests.cs:16-52
 *   - manufactured solution    FemCantileverBase.cs:53-62 (b = Kff*u_EB, so a
 *                              converged solve must return u_EB)
 * Numbering conventions of the external MSolve mesh (x-fastest nodes and
 * elements, VTK hexa/quad corner order) are fixed here and checked by the
 * rigid-body null space of the element stiffness.
 */
#ifndef DUVI_ORACLE_H
#define DUVI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- containers ---------------------------------------------------------- */
typedef struct or_csr or_csr;         /* sorted CSR, int32 indices, double values */
typedef struct or_model or_model;     /* FemCantilever{2D,3D} restatement        */
typedef struct or_duvi or_duvi;       /* GPU DuVi SoA (OpenCLDuViGeometricMultigridSolver.cs:16-31) */
typedef struct or_units or_units;     /* CPU DuVi Unit stream (DuViCompressedSparseMatrix.cs:11-152) */
typedef struct or_gmg or_gmg;         /* GeometricMultigridSolver restatement   */

or_csr *or_csr_create(int32_t n_rows, int32_t n_cols, const int32_t *rowptr,
                      const int32_t *col, const double *val);
void or_csr_free(or_csr *a);
void or_csr_info(const or_csr *a, int32_t *n_rows, int32_t *n_cols, int64_t *nnz);
void or_csr_copy(const or_csr *a, int32_t *rowptr, int32_t *col, double *val);
/* y = A x, entries summed from 0.0 in stored (column) order. */
void or_csr_spmv(const or_csr *a, const double *x, double *y);
/* One forward Gauss-Seidel sweep in row order (x updated in place). */
void or_csr_gs_forward(const or_csr *a, const double *b, double *x);

/* ---- model (FemCantileverBase.cs / FemCantilever3D.cs / FemCantilever2D.cs) */
/* dim = 2 or 3; ne = elements per axis; len = length per axis (3 entries
 * always, as in the reference constructors); densities may be NULL (all 1). */
or_model *or_model_create(int dim, const int32_t *ne, const double *len,
                          double E, double nu, double q, const double *densities);
void or_model_free(or_model *m);
int32_t or_model_num_free(const or_model *m);
int32_t or_model_num_all(const or_model *m);
const or_csr *or_model_kff(const or_model *m);              /* borrowed */
void or_model_rhs(const or_model *m, double *b);            /* manufactured b = Kff u_EB */
void or_model_uf(const or_model *m, double *uf);            /* u_EB on free dofs */
void or_model_free_dofs(const or_model *m, int32_t *free_dofs);
void or_model_element_stiffness(int dim, double E, double nu, double *ke);
/* Row-ratio spectral bound max_i sum|a_ij| / max|a_ij| (GeometricMultigridSolver.cs:144-151),
 * summed in DOK insertion order. */
double or_model_row_ratio_bound(const or_model *m);
/* Consistent nodal loads of a uniform traction t on the face x = max. */
void or_traction_rhs(int dim, const int32_t *ne, const double *len, const double *t, double *b);

/* Restriction / interpolation (IGeometricMultigridModel.cs:76-194), free-dof
 * submatrices, sorted CSR. */
void or_transfer_create(int dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                        or_csr **restriction, or_csr **interpolation);

/* ---- GPU DuVi SoA (OpenCLDuViGeometricMultigridSolver.cs:753-851) --------- */
/* force_bits: 0 = auto (8 if <=256 distinct, else 16 if <=65536, else 32). */
or_duvi *or_duvi_encode(const or_csr *a, double tol, int force_bits);
void or_duvi_free(or_duvi *d);
/* sizes: [n_rows, nblocks, nnz, nuniq, vi_bits] */
void or_duvi_info(const or_duvi *d, int64_t *sizes);
void or_duvi_copy(const or_duvi *d, uint32_t *row_to_col, uint32_t *row_to_dist,
                  uint32_t *col_idx, uint8_t *dist, uint32_t *vidx, double *values);
/* y = A x (clear = 1) or y += A x (clear = 0), DuViGeometricMultigrid.cl:57-99 order. */
void or_duvi_spmv(const or_duvi *d, const double *x, double *y, int clear);
/* Decode back to dense row-major (DuVi2Mat, OpenCLDuViGeometricMultigridSolver.cs:394-415). */
void or_duvi_to_dense(const or_duvi *d, int32_t n_cols, double *dense);

/* ---- CPU DuVi Unit stream (DuViCompressedSparseMatrix.cs) ----------------- */
or_units *or_units_from_csr(const or_csr *a, double tol);
or_units *or_units_from_dense(int32_t h, int32_t w, const double *values, double tol);
void or_units_free(or_units *u);
/* sizes: [n_units, n_bytes, n_vidx, nuniq] */
void or_units_info(const or_units *u, int64_t *sizes);
void or_units_copy(const or_units *u, uint8_t *bytes, int64_t *unit_offsets,
                   int32_t *vidx, double *values);
void or_units_multiply(const or_units *u, const double *x, double *y);
double or_units_get(const or_units *u, int32_t row, int32_t col);
void or_units_gs(const or_units *u, const double *b, double *x);

/* ---- solver pieces --------------------------------------------------------- */
/* Power-method bound (GeometricMultigridSolver.cs:80-103). */
double or_power_bound(const or_csr *a, const double *inv_diag);
/* Dense LDL^T, no pivoting (restated; SkylineMatrix.FactorLdl is external).
 * Returns 0 or -1 on a pivot below tol.  a is overwritten by the factor. */
int or_ldl_factor(int32_t n, double *a, double tol);
void or_ldl_solve(int32_t n, const double *f, const double *b, double *x);
/* MakePath (GeometricMultigridSolver.cs:178-201).  level_down in/out with
 * capacity cap; returns the new length; writes total_levels, first_level. */
int32_t or_make_path(uint8_t *level_down, int32_t n, int32_t cap,
                     int32_t *total_levels, int32_t *first_level);

/* GeometricMultigridSolver (CPU) over the cantilever model hierarchy.
 * Mirrors Initialize (:216-261) and Solve (:297-418). */
or_gmg *or_gmg_create(int dim, const int32_t *ne, const double *len, double E, double nu,
                      int gauss_seidel, int duvi, int32_t max_cycles, int coarse_relaxation,
                      double tol, const uint8_t *level_down, int32_t n_steps,
                      const int32_t *level_iterations, int32_t n_level_iterations);
void or_gmg_free(or_gmg *g);
/* stats: [cycles, converged, failed]; res: [max|r|, ||r||_2] at exit. */
void or_gmg_solve(or_gmg *g, const double *x0, double *x, int32_t *stats, double *res);
int32_t or_gmg_num_levels(const or_gmg *g);
double or_gmg_omega_scale(const or_gmg *g, int32_t level);

/* Jacobi PCG as written in GMCantileverTests.cs:400-433 (absolute max-norm stop).
 * Returns the iteration index at convergence, or -1. */
int32_t or_pcg_jacobi(const or_csr *a, const double *b, double *x, int32_t max_iter, double tol);
/* The same with the stop test ||r||_2 <= tol ||b||_2 (build-defined option). */
int32_t or_pcg_jacobi_rel(const or_csr *a, const double *b, double *x, int32_t max_iter, double tol);

/* ---- build-defined extensions (no reference counterpart; FP64 checkers) --- */
/* Structured hex assembly at element size h: K = h * sum_e E_e Ke (3-D). */
or_csr *or_hex_stiffness(const int32_t *ne, const double *elem_E, double scale, double E, double nu);
/* Trilinear prolongation between factor-2 structured hex grids, free dofs. */
or_csr *or_hex_trilinear(const int32_t *ne_fine);
/* Galerkin product P^T A P (sorted CSR). */
or_csr *or_galerkin(const or_csr *a, const or_csr *p);
/* Flexible PCG (FCG(1)) with a V(nu,nu) weighted-Jacobi multigrid preconditioner,
 * FP64, relative 2-norm stop.  levels: A[0..L-1], P[0..L-2] (fine from coarse);
 * restriction is P^T.  omega_eff multiplies D^-1.  Coarse solve by LDL^T.
 * Returns iterations (or -1); relres gets the true ||b-Ax||/||b||. */
int32_t or_mg_fcg(int32_t n_levels, or_csr *const *A, or_csr *const *P, double omega_eff,
                  int32_t nu, const double *b, double *x, int32_t max_iter, double tol,
                  double *relres);
/* Wall time of the iteration phase (after the coarse factorisation) of the last or_mg_fcg. */
double or_last_solve_seconds(void);
/* Adjoint gradient dJ/drho_e = -3 rho_e^2 lambda_e^T Ke u_e over free dofs
 * (E_e = rho_e^3), given u and lambda on free dofs. */
void or_adjoint_element_gradient(const int32_t *ne, double E, double nu, const double *rho,
                                 const double *u, const double *lambda, double *grad);
/* Objective helpers for finite differences: element moduli E_e = rho_e^3. */
void or_rho_to_modulus(int64_t n, const double *rho, double *E);

/* ---- parallel baseline (restatement, parallelised with OpenMP) ----------- */
/* Threads for the row loops (SpMV, structured assembly, element-wise vector
 * updates); default 1.  Row sums keep their order, so results do not change. */
void or_set_threads(int n);
void or_csr_spmv_omp(const or_csr *a, const double *x, double *y);
int or_omp_threads(void);

#ifdef __cplusplus
}
#endif
#endif
