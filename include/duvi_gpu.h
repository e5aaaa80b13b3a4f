/*
 * duvi_gpu.h -- C ABI of the B200 sparse solver path (libduvigpu.so).
 *
 * Drop-in replacement for the OpenCL layer of nickreserved/CompressionTests
 * (the OpenCL kernels in src/MGroup.OCL and the three solver classes that drive them), callable
 * from C# through [DllImport] or from any C FFI.  Plain pointers and sizes
 * only.  One CUDA device per context, one stream per context; every call that
 * takes host arrays copies them and returns after the device work finished
 * (like the reference's blocking WriteBuffer/ReadBuffer).  Calls on one
 * handle are not thread-safe.  There is no CPU fallback: without a usable
 * GPU every compute call fails with DV_ERR_NO_DEVICE.
 *
 * Reference interfaces replaced (file:line inside the reference project):
 *   OpenCLCsrGeometricMultigridSolver  src/MGroup.Solvers/Multigrid/OpenCLCsrGeometricMultigridSolver.cs:55-83,145-285,334-536
 *   OpenCLDuViGeometricMultigridSolver src/MGroup.Solvers/Multigrid/OpenCLDuViGeometricMultigridSolver.cs:77-104,172-391,455-751
 *   OpenCLCsrPcgSolver                 src/MGroup.Solvers/Multigrid/OpenCLCsrPcgSolver.cs:40-45,84-218,250-331
 *   IGeometricMultigridSolver.Solve    src/MGroup.Solvers/Multigrid/IGeometricMultigridSolver.cs:8
 *   IOpenCLGeometricMultigridSolver.ReleaseOpenCLResources  IOpenCLGeometricMultigridSolver.cs:5
 *   DuViCompressedSparseMatrix.Multiply src/MGroup.LinearAlgebra/Matrices/DuViCompressedSparseMatrix.cs:419-441
 *   OpenCL kernels                     src/MGroup.OCL/CsrCG.cl, CsrGeometricMultigrid.cl, DuViGeometricMultigrid.cl
 */
#ifndef DUVI_GPU_H
#define DUVI_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define DV_API __attribute__((visibility("default")))
#else
#define DV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------------
 * Mirrors the exceptions of the reference: DV_ERR_NOT_INITIALIZED for
 * InvalidOperationException("You must call Initialize(model) first")
 * (OpenCLCsrGeometricMultigridSolver.cs:336), DV_ERR_UNSUPPORTED for
 * NotImplementedException (firstLevel != 0, :345), DV_ERR_CUDA for
 * OpenCLException (OpenCLDuViGeometricMultigridSolver.cs:859). */
enum {
    DV_OK = 0,
    DV_ERR_ARG = -1,
    DV_ERR_CUDA = -2,
    DV_ERR_NOT_INITIALIZED = -3,
    DV_ERR_UNSUPPORTED = -4,
    DV_ERR_NOMEM = -5,
    DV_ERR_FORMAT = -6,
    DV_ERR_NO_DEVICE = -7,
    DV_ERR_SINGULAR = -8
};

/* DV_FORMAT_HEX: matrix-free hexahedral operator (dv_matrix_create_hex); DV_FORMAT_TRILINEAR:
 * matrix-free trilinear transfer of a structured grid (dv_matrix_create_trilinear). */
enum { DV_FORMAT_CSR = 0, DV_FORMAT_DUVI = 1, DV_FORMAT_HEX = 2, DV_FORMAT_TRILINEAR = 3 };
enum { DV_F64 = 0, DV_F32 = 1, DV_MIXED = 2 };
enum { DV_SMOOTHER_JACOBI = 0, DV_SMOOTHER_GS_LEX = 1, DV_SMOOTHER_GS_COLOR = 2 };
enum { DV_TOL_ABS_MAX = 0, DV_TOL_REL_L2 = 1 };
enum { DV_OMEGA_ABSOLUTE = 0, DV_OMEGA_SPECTRAL = 1 };

typedef struct dv_context dv_context;
typedef struct dv_matrix dv_matrix;
typedef struct dv_gmg dv_gmg;
typedef struct dv_pcg dv_pcg;
typedef struct dv_mgpcg dv_mgpcg;
typedef struct dv_batch dv_batch;
typedef struct dv_adjoint dv_adjoint;

/* Host CSR view (int32 indices, float64 values; columns sorted per row). */
typedef struct {
    int32_t n_rows, n_cols;
    const int32_t *rowptr;
    const int32_t *col;
    const double *val;
} dv_csr_host;

/* Solve statistics.  Every solver fills iterations, converged, failed,
 * relative_residual (||b - A x||_2 / ||b||_2 of the returned x, recomputed in FP64
 * at exit; for dv_mgpcg_solve_multi and dv_batch_solve the worst load case or mesh)
 * and solve_ms (device time of the solve, CUDA events).  residual_norm2 is the
 * 2-norm of the last residual the stop test checked (the worst one for several
 * load cases or meshes).  residual_max, its max-norm, is filled by the solvers
 * whose stop test can use it (dv_gmg_solve, dv_pcg_solve, dv_pcg_solve_noalloc);
 * the flexible-CG solvers (dv_mgpcg_*, dv_batch_*, dv_adjoint_*) stop on the
 * 2-norm and leave it NaN. */
typedef struct {
    int32_t iterations;        /* NumIterationsRequired (cycles or PCG iterations) */
    int32_t converged;         /* HasConverged: flag bit 1 of the reference kernels */
    int32_t failed;            /* NaN or |r_i| > 1e50: flag bit 2 (CsrCG.cl:274-276) */
    int32_t reserved;          /* always 0 */
    double residual_max;       /* max_i |r_i| of the last checked residual */
    double residual_norm2;     /* ||r||_2 of the last checked residual */
    double relative_residual;  /* ||b - A x||_2 / ||b||_2, recomputed in FP64 at exit */
    double solve_ms;           /* device time of the solve (CUDA events) */
} dv_stats;

DV_API const char *dv_status_string(int status);
/* Message of the last failing call on this thread. */
DV_API const char *dv_last_error(void);
DV_API int dv_version(void);

/* ---- context (replaces Platform/Device/Program/command queue,
 *      src/MGroup.OCL/Platform.cs:26-46, Device.cs:32-57) ---------------- */
DV_API int dv_context_create(int device_ordinal, dv_context **out);
DV_API int dv_context_destroy(dv_context *ctx);
DV_API int dv_context_synchronize(dv_context *ctx);
/* The context's cudaStream_t, for callers that launch their own work. */
DV_API void *dv_context_stream(dv_context *ctx);
/* Number of device kernel launches issued by this context so far. */
DV_API int64_t dv_context_launch_count(const dv_context *ctx);

/* ---- matrices (buffers of OpenCL*Solver.Initialize) ----------------------- */
typedef struct {
    int32_t n_rows, n_cols;
    int64_t nnz;
    int64_t nblocks;           /* DuVi blocks (0 for CSR) */
    int64_t nuniq;             /* DuVi distinct values (0 for CSR) */
    int32_t format;            /* DV_FORMAT_* */
    int32_t precision;         /* DV_F64 / DV_F32 value storage */
    int32_t value_index_bits;  /* 8, 16, 32 (DuVi) */
    int32_t kernel_variant;    /* autotuned launch shape */
    int64_t device_bytes;      /* bytes one product reads from the matrix arrays */
    int32_t row_group;         /* 3 (or 2) when consecutive rows share one column list (node dofs), else 1 */
    int32_t reserved;
} dv_matrix_info;

/* CSR upload (uint row offsets / column indices / double values of
 * OpenCLCsrPcgSolver.cs:125-130).  precision selects FP64 or FP32 storage. */
DV_API int dv_matrix_create_csr(dv_context *ctx, const dv_csr_host *a, int32_t precision, dv_matrix **out);
/* DuVi encode on the host (FromDokRowMajor, OpenCLDuViGeometricMultigridSolver.cs:753-851)
 * and upload.  value_index_bits: 0 = auto (8 up to 256 distinct values, 16 up
 * to 65536, else 32); dedup_tol: ToleranceComparer tolerance (1e-10 in the
 * reference; 0 = exact equality).  Up to 256 distinct values the arrays equal
 * the reference encoder's bit for bit. */
DV_API int dv_matrix_create_duvi(dv_context *ctx, const dv_csr_host *a, int32_t precision,
                                 int32_t value_index_bits, double dedup_tol, dv_matrix **out);
/* The same DuVi encode on the host only, no device needed: the SoA arrays that
 * dv_matrix_create_duvi uploads, for storage or interchange.  Call once with
 * row_to_col == NULL for the sizes (*nblocks, *nuniq, *bits), then with arrays of
 * n_rows+1, n_rows+1, nblocks, nnz, nnz and nuniq elements (value indices
 * widened to uint32). */
DV_API int dv_duvi_encode(const dv_csr_host *a, int32_t value_index_bits, double dedup_tol, int64_t *nblocks,
                          int64_t *nuniq, int32_t *bits, uint32_t *row_to_col, uint32_t *row_to_dist,
                          uint32_t *col_idx, uint8_t *dist, uint32_t *value_indices, double *values);
/* The CPU DuVi Unit stream (DuViCompressedSparseMatrix, DuViCompressedSparseMatrix.cs:11-152 and
 * its CSR constructor :285-400) as one flat byte stream, for storage and interchange; host only.
 * Each row is one or more units (header byte: new-row bit | step width class << 1; step count
 * byte; column gap as a 1-4 byte big-endian prefix code; little-endian column steps of 1, 2
 * or 4 bytes); an empty row is one unit of gap 0 whose value is 0.0.  value_indices (int32,
 * one per entry and per empty row) number the values in entry order with the reference's
 * Dictionary semantics (dedup_tol as in dv_matrix_create_duvi).  Call with bytes == NULL for
 * the sizes, then with bytes[n_bytes], unit_offsets[n_units + 1], value_indices[n_indices]
 * and values[nuniq].  Rows that would need a unit of more than 255 steps (the reference
 * wraps its one-byte count) or a gap of 2^29 + 2,113,664 or more: DV_ERR_FORMAT. */
DV_API int dv_units_encode(const dv_csr_host *a, double dedup_tol, int64_t *n_units, int64_t *n_bytes,
                           int64_t *n_indices, int64_t *nuniq, uint8_t *bytes, int64_t *unit_offsets,
                           int32_t *value_indices, double *values);
/* Unit stream back to CSR, walking the units as DuViCompressedSparseMatrix.Multiply does
 * (:419-441): *nnz with rowptr == NULL, then rowptr[n_rows + 1], col[nnz], val[nnz].  An
 * empty row comes back as one entry (column 0, value of its index: 0.0).  Malformed streams
 * (truncated units, columns past n_cols or not increasing within a row, index or row counts
 * that do not match): DV_ERR_FORMAT. */
DV_API int dv_units_decode(int32_t n_rows, int32_t n_cols, const uint8_t *bytes, int64_t n_bytes,
                           const int32_t *value_indices, int64_t n_indices, const double *values, int64_t nuniq,
                           int64_t *nnz, int32_t *rowptr, int32_t *col, double *val);
/* The same DuVi encode of a CSR matrix that is already in device memory, run on the device:
 * d_rowptr (n_rows + 1), d_col and d_val (nnz < 2^31) are device arrays (context stream).
 * The arrays equal dv_matrix_create_duvi's bit for bit; the distinct values pass through the
 * dedup_tol dictionary on the host (all values do when the tolerance makes a lookup depend on
 * insertion time).  The node-pattern and grid-stencil layouts are derived on the device too; the
 * lane layout is not built (matrices without node patterns run the staged kernel).  Pairs with
 * dv_hex_assemble_device for an operator that never passes through host memory. */
DV_API int dv_matrix_create_duvi_device(dv_context *ctx, int32_t n_rows, int32_t n_cols, const int32_t *d_rowptr,
                                        const int32_t *d_col, const double *d_val, int32_t precision,
                                        int32_t value_index_bits, double dedup_tol, dv_matrix **out);
/* Upload an already encoded DuVi SoA (DuViMat8/16, :16-31). value_indices has
 * value_index_bits per entry. */
DV_API int dv_matrix_create_duvi_soa(dv_context *ctx, int32_t n_rows, int32_t n_cols,
                                     const uint32_t *row_to_col, const uint32_t *row_to_dist,
                                     const uint32_t *col_idx, int64_t nblocks, const uint8_t *dist,
                                     int64_t nnz, const void *value_indices, int32_t value_index_bits,
                                     const double *values, int64_t nuniq, int32_t precision,
                                     dv_matrix **out);
/* Matrix-free operator of the structured hexahedral stiffness (format DV_FORMAT_HEX): the
 * same operator as dv_hex_assemble(ne, elem_E, scale, E, nu), applied element by element
 * from one factor scale * E_e per element (elem_E NULL: uniform) and the 24 x 24 element
 * stiffness, without storing the matrix.  A product reads the factors, x and y only.
 * Usable wherever an operator is applied (dv_spmv, dv_spmv_device, dv_residual_device, the
 * diagonal for Jacobi weights); not for dv_spmm_device or DuVi export (DV_ERR_UNSUPPORTED).
 * FP64 products equal the assembled matrix's to rounding (another summation order), not bit
 * for bit.  The reference assembles the matrix (FemCantileverBase.cs:87-104); it has no
 * matrix-free counterpart. */
DV_API int dv_matrix_create_hex(dv_context *ctx, const int32_t *ne, const double *elem_E, double scale, double E,
                                double nu, int32_t precision, dv_matrix **out);
/* The trilinear prolongation of dv_hex_trilinear (restrict = 0; fine free x coarse free) or its
 * transpose, the restriction (restrict = 1), for an even grid of ne_fine elements, applied without
 * storing the matrix; products equal the assembled matrix's bit for bit (same column order and
 * rounding).  Replaces the transfer matrices of IGeometricMultigridModel.cs:76-194 on structured
 * grids.  Odd element counts: DV_ERR_UNSUPPORTED. */
DV_API int dv_matrix_create_trilinear(dv_context *ctx, const int32_t *ne_fine, int32_t restrict_, int32_t precision,
                                      dv_matrix **out);
DV_API int dv_matrix_get_info(const dv_matrix *m, dv_matrix_info *info);
/* Copy the DuVi arrays back (value indices widened to uint32). */
DV_API int dv_matrix_export_duvi(const dv_matrix *m, uint32_t *row_to_col, uint32_t *row_to_dist,
                                 uint32_t *col_idx, uint8_t *dist, uint32_t *value_indices,
                                 double *values);
DV_API int dv_matrix_destroy(dv_matrix *m);

/* y = A x (clear != 0) or y += A x (matrix_vector_product, CsrGeometricMultigrid.cl:49-62,
 * DuViGeometricMultigrid.cl:122-159).  Host vectors, FP64. */
DV_API int dv_spmv(dv_matrix *m, const double *x, double *y, int32_t clear);
/* Same on device pointers (vec_precision DV_F64 or DV_F32), asynchronous on
 * the context stream. */
DV_API int dv_spmv_device(dv_matrix *m, const void *x, void *y, int32_t vec_precision, int32_t clear);
/* r = b - A x (residual, CsrGeometricMultigrid.cl:96-110), device pointers. */
DV_API int dv_residual_device(dv_matrix *m, const void *b, const void *x, void *r, int32_t vec_precision);
/* k right-hand sides at once: X and Y are n x k row-interleaved (X[i*k + j]);
 * the matrix is read once per call.  Device pointers. */
DV_API int dv_spmm_device(dv_matrix *m, int32_t k, const void *X, void *Y, int32_t vec_precision,
                          int32_t clear);

/* ---- geometric multigrid (stationary V-cycle, reference semantics) --------
 * OpenCL{Csr,DuVi}GeometricMultigridSolver.CreateDeepV/CreateSimpleV + Solve.
 * A has n_levels operators (level 0 finest, the last one is factorised and
 * solved directly), R and P have n_levels - 1. */
typedef struct {
    int32_t smoother;               /* DV_SMOOTHER_* (GaussSeidel flag of the reference) */
    int32_t format;                 /* DV_FORMAT_CSR / DV_FORMAT_DUVI */
    int32_t max_cycles;             /* maxCircleIterations */
    int32_t coarse_relaxation;      /* 1: w = 2/l, l = row-ratio bound of the coarsest A;
                                       0: w = 2/(1.2 l), l from the power method per level */
    double tol;                     /* convergenceTolerance, absolute max-norm */
    int32_t n_steps;                /* length of level_down; 0 = deep V of depth n_levels-1 */
    const uint8_t *level_down;      /* LevelDown path (true = go coarser) */
    int32_t n_level_iterations;
    const int32_t *level_iterations;/* levelIterations (last value repeats) */
    int32_t cycles_per_sync;        /* cycles run per host convergence read (0 = 16) */
} dv_gmg_config;

DV_API int dv_gmg_create(dv_context *ctx, int32_t n_levels, const dv_csr_host *A,
                         const dv_csr_host *R, const dv_csr_host *P, const dv_gmg_config *cfg,
                         dv_gmg **out);
/* b: level-0 right-hand side; x0 may be NULL (zero initial guess). */
DV_API int dv_gmg_solve(dv_gmg *g, const double *b, const double *x0, double *x, dv_stats *stats);
/* Relaxation factor w applied to D^-1 on level l (for parity checks). */
DV_API int dv_gmg_omega(const dv_gmg *g, int32_t level, double *omega);
DV_API int dv_gmg_destroy(dv_gmg *g);

/* ---- Jacobi PCG (OpenCLCsrPcgSolver, FP64, absolute max-norm stop) ------- */
DV_API int dv_pcg_create(dv_context *ctx, const dv_csr_host *A, int32_t format, int32_t max_iterations,
                         double tol, dv_pcg **out);
/* Stop test of later solves: DV_TOL_ABS_MAX (default) stops when every |r_i| <= tol,
 * the reference's test (CsrCG.cl:257-277, GMCantileverTests.cs:420-424); DV_TOL_REL_L2
 * stops when ||r||_2 <= tol ||b||_2 (r the recurrence residual, checked at the same
 * place of the iteration). */
DV_API int dv_pcg_set_tolerance_kind(dv_pcg *p, int32_t tol_kind);
DV_API int dv_pcg_solve(dv_pcg *p, const double *b, const double *x0, double *x, dv_stats *stats);
DV_API int dv_pcg_destroy(dv_pcg *p);

/* Jacobi PCG that allocates nothing.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory when they solve -- hosts that
 * reserve all device memory up front and forbid later allocations, and
 * time-critical loops that cannot afford cudaFree's device-wide
 * synchronisation.  Same algorithm and stop test as dv_pcg_solve; the
 * work vectors live in one fixed device array of this library (4,325,632 bytes
 * per device, held until the process exits), which limits A to 131,072 rows
 * (larger: DV_ERR_ARG).  A must be an FP64 square matrix created beforehand;
 * d_b and d_x are device pointers (x: initial guess if use_x0, else zeroed; the
 * solution on return), read and written on A's context stream
 * (dv_context_stream): work the caller queued on another stream to fill d_b or
 * d_x must be ordered before the call (an event wait or a synchronize).  The
 * call returns after the solve finished.  All calls on a device share the
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on a device looks up the array's device address;
 * make it before any stream capture.  The array and the kernels' code are
 * device memory that CUDA allocates when it loads them; with CUDA's default
 * lazy module loading that is at the first call on a device (a kernel's code at
 * its first launch), so a caller that reserves all free device memory makes
 * one call with each matrix format it will use before reserving, or runs with
 * CUDA_MODULE_LOADING=EAGER.  stats->relative_residual is recomputed in FP64 at
 * exit, inside the same array. */
DV_API int dv_pcg_solve_noalloc(dv_matrix *A, const double *d_b, double *d_x, int32_t use_x0,
                                int32_t max_iterations, double tol, dv_stats *stats);

/* ---- multigrid-preconditioned flexible PCG (FP64 or mixed precision) ------
 * Build-defined extension of the reference pieces: an FP64 flexible CG
 * (FCG(1)) outer loop with true-residual refinement restarts, preconditioned
 * by one V(nu,nu) cycle of weighted Jacobi.  DV_MIXED runs the V-cycle on
 * FP32 values and vectors with FP32 accumulation; the outer residual, the
 * alpha/beta dot products and the solution update stay FP64.  Restriction is
 * P^T.  The coarsest level is solved with a dense inverse computed from an
 * LDL^T factorisation. */
typedef struct {
    int32_t precision;          /* DV_F64 or DV_MIXED */
    int32_t format;             /* V-cycle operators: DV_FORMAT_CSR / DV_FORMAT_DUVI */
    int32_t outer_format;       /* FP64 operator of the outer loop */
    int32_t nu;                 /* pre- and post-smoothing sweeps */
    double omega;               /* Jacobi weight */
    int32_t omega_mode;         /* DV_OMEGA_ABSOLUTE: x += omega D^-1 r;
                                   DV_OMEGA_SPECTRAL: x += omega (2/l) D^-1 r, l = spectral
                                   radius estimate of D^-1 A per level */
    int32_t max_iterations;
    double tol;                 /* relative 2-norm */
    int32_t iterations_per_sync;/* most outer iterations per host convergence read (0 = 4); the single
                                  right-hand-side solve shortens a chunk when the convergence rate so
                                  far predicts the tolerance within it */
    int32_t use_graphs;         /* capture the iteration sequence in a CUDA graph */
    int32_t smoother;           /* DV_SMOOTHER_JACOBI (default, 0): weighted Jacobi as above;
                                   DV_SMOOTHER_GS_LEX: nu forward Gauss-Seidel sweeps before and after
                                   the coarse correction, rows in the reference's order
                                   (GaussSeidelIterationCsrDuVi.cs:22-50; dependency levels on the GPU);
                                   DV_SMOOTHER_GS_COLOR: the same with multicolor node blocks.
                                   Gauss-Seidel is unweighted (omega unused); dv_batch_* accept Jacobi only. */
} dv_mgpcg_config;

DV_API int dv_mgpcg_create(dv_context *ctx, int32_t n_levels, const dv_csr_host *A,
                           const dv_csr_host *P, const dv_mgpcg_config *cfg, dv_mgpcg **out);
/* The same solver for the uniform hexahedral cantilever (ne elements, modulus E, Poisson
 * ratio nu, x = 0 face clamped), its hierarchy built on the device: the factor-2
 * re-discretised levels K_l = 2^l sum_e E Ke down to coarse_ne elements along the shortest
 * axis (or an odd count) are assembled by dv_hex_assemble_device and DuVi-encoded on the
 * device; only the trilinear prolongations and the coarsest level are built on the host.
 * The operators equal those of dv_mgpcg_create on the host-built hierarchy bit for bit, so
 * solves match it exactly.  cfg: DuVi V-cycle and outer operators, Jacobi smoother
 * (otherwise DV_ERR_UNSUPPORTED). */
DV_API int dv_mgpcg_create_hex(dv_context *ctx, const int32_t *ne, double E, double nu, int32_t coarse_ne,
                               const dv_mgpcg_config *cfg, dv_mgpcg **out);
DV_API int dv_mgpcg_solve(dv_mgpcg *s, const double *b, double *x, dv_stats *stats);
/* Device-resident right-hand side and solution (FP64), context stream. */
DV_API int dv_mgpcg_solve_device(dv_mgpcg *s, const double *d_b, double *d_x, dv_stats *stats);
/* Effective Jacobi weight omega_eff applied to D^-1 on V-cycle level l. */
DV_API int dv_mgpcg_omega(const dv_mgpcg *s, int32_t level, double *omega_eff);
/* k load cases (1 <= k <= 128) in one solve on the same hierarchy.  B and X are
 * n x k row-interleaved (B[i*k + j] = load case j at dof i).  Every operator
 * application reads the matrix once for all k vectors; each load case has its
 * own FCG scalars and stops at ||r_j|| <= tol ||b_j|| (FP64-verified).
 * converged_per_rhs (optional, k entries) receives 1 per converged load case;
 * stats->relative_residual is the worst case.  Replaces calling
 * PcgSolver2.InverseSystemMatrixTimesOtherMatrix (PcgSolver2.cs:92-136), which
 * solves the columns one after another. */
DV_API int dv_mgpcg_solve_multi(dv_mgpcg *s, int32_t k, const double *B, double *X, int32_t *converged_per_rhs,
                                dv_stats *stats);
/* Same with device-resident B and X (FP64, n x k), context stream. */
DV_API int dv_mgpcg_solve_multi_device(dv_mgpcg *s, int32_t k, const double *d_B, double *d_X,
                                       int32_t *converged_per_rhs, dv_stats *stats);
DV_API int dv_mgpcg_destroy(dv_mgpcg *s);

/* ---- batched MG-PCG over many independent meshes ------------------------
 * n_meshes systems, mesh m with n_levels[m] levels: A[m][0..n_levels[m]-1]
 * (square, finest first) and P[m][0..n_levels[m]-2] (prolongation from level
 * l+1 to l; restriction is its transpose).  Every mesh's coarsest level is
 * solved with a dense inverse (at most 16384 dofs).  Per level the operators
 * of all meshes are concatenated block-diagonally, so each smoothing sweep,
 * transfer and outer product is one launch for all meshes, and the iteration
 * sequence is captured in one CUDA graph.  cfg as for dv_mgpcg (mixed: FP32
 * V-cycles inside the FP64 flexible CG).  Each mesh stops at its own
 * ||r_m|| <= tol ||b_m|| (FP64-verified).  The reference builds one solver per
 * model (GeometricMultigridSolver.Initialize, GeometricMultigridSolver.cs:57-77). */
DV_API int dv_batch_create(dv_context *ctx, int32_t n_meshes, const int32_t *n_levels, const dv_csr_host *const *A,
                           const dv_csr_host *const *P, const dv_mgpcg_config *cfg, dv_batch **out);
/* The same batch for n_meshes uniform hexahedral cantilevers (ne: 3 element counts per mesh,
 * modulus E, Poisson ratio nu, x = 0 faces clamped): each mesh's Galerkin hierarchy (vertex
 * factor-2 coarsening, trilinear P) down to at most max_coarse_dofs dofs is built here, and the
 * finest operators of all meshes are applied matrix-free in one launch (the element operator of
 * dv_matrix_create_hex over a table of meshes); DV_MATRIX_FREE=0 keeps them assembled. */
DV_API int dv_batch_create_hex(dv_context *ctx, int32_t n_meshes, const int32_t *ne, double E, double nu,
                               int32_t max_coarse_dofs, const dv_mgpcg_config *cfg, dv_batch **out);
/* Total fine rows, levels of the deepest mesh, kernel launches per captured chunk (0 before the first solve). */
DV_API int dv_batch_info(const dv_batch *b, int32_t *n_rows, int32_t *n_levels_max, int32_t *n_launches_per_chunk);
/* Effective Jacobi weight of batch level l (one weight for all meshes smoothing on that level). */
DV_API int dv_batch_omega(const dv_batch *b, int32_t level, double *omega_eff);
/* rhs and x: the meshes' fine-level vectors concatenated in mesh order (host
 * arrays, FP64).  converged_per_mesh / iterations_per_mesh: optional, n_meshes entries. */
DV_API int dv_batch_solve(dv_batch *b, const double *rhs, double *x, int32_t *converged_per_mesh,
                          int32_t *iterations_per_mesh, dv_stats *stats);
/* Same with device-resident rhs and x, context stream. */
DV_API int dv_batch_solve_device(dv_batch *b, const double *d_rhs, double *d_x, int32_t *converged_per_mesh,
                                 int32_t *iterations_per_mesh, dv_stats *stats);
DV_API int dv_batch_destroy(dv_batch *b);

/* ---- adjoint sensitivities of a density-parametrised cantilever -----------
 * Unit-cube hexahedra on an ne[0] x ne[1] x ne[2] grid (x = 0 face clamped),
 * element moduli E_e = E0 rho_e^penal.  Forward/Backward pair in the shape of
 * an autograd function: forward u = K(rho)^-1 f; backward takes dJ/du, solves
 * K lambda = dJ/du with the forward's solver (K is symmetric; no state of the
 * forward iterations is kept) and returns dJ/drho_e = -lambda_e^T (dK_e/drho_e) u_e
 * from an element kernel over the connectivity.  The reference has no adjoint
 * path; the elements, dof numbering and load follow FemCantilever3D
 * (FemCantileverBase.cs:87-158).  create builds K(rho) and a Galerkin
 * hierarchy (vertex factor-2 coarsening, trilinear P) down to at most
 * max_coarse_dofs dofs, then the MG-PCG solver of cfg.  With the Jacobi smoother
 * the finest K(rho) is applied matrix-free (as dv_matrix_create_hex) in the outer
 * loop and the finest V-cycle level; the environment variable DV_MATRIX_FREE=0
 * keeps the assembled operator there. */
DV_API int dv_adjoint_create(dv_context *ctx, const int32_t *ne, const double *rho, double penal, double E0, double nu,
                             int32_t max_coarse_dofs, const dv_mgpcg_config *cfg, dv_adjoint **out);
DV_API int dv_adjoint_info(const dv_adjoint *a, int32_t *n_dofs, int64_t *n_elements);
/* u = K(rho)^-1 f (host arrays, free dofs); keeps u on the device for backward. */
DV_API int dv_adjoint_forward(dv_adjoint *a, const double *f, double *u, dv_stats *stats);
/* dJdrho (n_elements) from dJdu (free dofs); lambda optional (free dofs).
 * DV_ERR_NOT_INITIALIZED before the first forward. */
DV_API int dv_adjoint_backward(dv_adjoint *a, const double *dJdu, double *dJdrho, double *lambda, dv_stats *stats);
DV_API int dv_adjoint_destroy(dv_adjoint *a);
/* The element kernel alone (device pointers, context stream, synchronous):
 * grad_e = -penal rho_e^(penal-1) lambda_e^T Ke(E0, nu) u_e. */
DV_API int dv_hex_element_gradient(dv_context *ctx, const int32_t *ne, const double *d_rho, double penal, double E0,
                                   double nu, const double *d_u, const double *d_lambda, double *d_grad);

/* ---- structured hex workload generator (FemCantilever3D on unit cubes) ----
 * Free dofs: all nodes with x index > 0 (FemCantileverBase.cs:137-158), node
 * ids x-fastest, VTK hexa corner order.  Entry (i,j) = sum over elements in
 * increasing id of (scale * E_e) * Ke_ij, the summation order of the DOK
 * assembly (FemCantileverBase.cs:87-104, DokRowMajor.cs:182-207). */
DV_API int dv_hex_csr_size(const int32_t *ne, int32_t *n_rows, int64_t *nnz);
DV_API int dv_hex_assemble(const int32_t *ne, const double *elem_E, double scale, double E, double nu,
                           int32_t *rowptr, int32_t *col, double *val);
/* The same assembly on the device, bit for bit (one thread per node writes its three
 * rows in the summation order above): d_rowptr, d_col, d_val are device arrays of
 * n_rows + 1, nnz and nnz elements (sizes from dv_hex_csr_size, nnz < 2^31); d_elem_E
 * is a device array of ne[0] ne[1] ne[2] moduli, or NULL for a uniform modulus.
 * Replaces the element loop of FemCantileverBase.AssembleGlobalMatrix
 * (FemCantileverBase.cs:87-104) into DokRowMajor (DokRowMajor.cs:182-207, 286-324).
 * Context stream; returns when the arrays are written. */
DV_API int dv_hex_assemble_device(dv_context *ctx, const int32_t *ne, const double *d_elem_E, double scale, double E,
                                  double nu, int32_t *d_rowptr, int32_t *d_col, double *d_val);
/* Trilinear prolongation of the factor-2 vertex coarsening (fine free x coarse
 * free).  Per axis with n elements the coarse nodes are the even fine nodes
 * and the last one, so odd n coarsens to (n+1)/2 elements (the last of length
 * 1); for even n this is the standard trilinear interpolation. */
DV_API int dv_hex_trilinear_size(const int32_t *ne_fine, int32_t *n_rows, int32_t *n_cols, int64_t *nnz);
DV_API int dv_hex_trilinear(const int32_t *ne_fine, int32_t *rowptr, int32_t *col, double *val);
/* Galerkin coarse operator P^T A P (square A, P with as many rows as A),
 * sorted rows; row I sums over the entries (r, I) of P, then (r, j) of A,
 * then (j, J) of P in storage order.  Size query, then fill. */
DV_API int dv_galerkin_size(const dv_csr_host *A, const dv_csr_host *P, int32_t *n, int64_t *nnz);
DV_API int dv_galerkin(const dv_csr_host *A, const dv_csr_host *P, int32_t *rowptr, int32_t *col, double *val);

/* Restriction and interpolation between two structured Cartesian meshes
 * (IGeometricMultigridModel.CreateRestrictionAndInterpolationMatrix,
 * src/MGroup.Solvers/Multigrid/IGeometricMultigridModel.cs:76-194): radial
 * weights 1 - |(w - c) / h| over the fine nodes in a window around each coarse
 * node, rows normalised to sum 1 before the fixed dofs are removed, then the
 * free-dof submatrices (rows/columns in the order of the free-dof lists).
 * Node ids are x-fastest; dof = dofs_per_node * node + component.  Outputs are
 * sorted CSR: R is n_coarse_free x n_fine_free, P is n_fine_free x n_coarse_free. */
DV_API int dv_cartesian_transfer_size(int32_t dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                                      int32_t dofs_per_node, int32_t n_fine_free, const int32_t *fine_free,
                                      int32_t n_coarse_free, const int32_t *coarse_free, int64_t *nnz_r,
                                      int64_t *nnz_p);
DV_API int dv_cartesian_transfer(int32_t dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                                 int32_t dofs_per_node, int32_t n_fine_free, const int32_t *fine_free,
                                 int32_t n_coarse_free, const int32_t *coarse_free, int32_t *r_rowptr,
                                 int32_t *r_col, double *r_val, int32_t *p_rowptr, int32_t *p_col,
                                 double *p_val);

#ifdef __cplusplus
}
#endif
#endif /* DUVI_GPU_H */
