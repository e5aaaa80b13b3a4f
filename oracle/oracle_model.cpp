// CPU oracle: CSR, DOK builder semantics, cantilever model and transfer operators.
// Test infrastructure only (see oracle.h).
#include "oracle_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>

// ---------------------------------------------------------------------------
// CSR
// ---------------------------------------------------------------------------
extern "C" or_csr *or_csr_create(int32_t n_rows, int32_t n_cols, const int32_t *rowptr,
                                 const int32_t *col, const double *val) {
    or_csr *a = new or_csr;
    a->n_rows = n_rows;
    a->n_cols = n_cols;
    a->rowptr.assign(rowptr, rowptr + n_rows + 1);
    int64_t nnz = rowptr[n_rows];
    a->col.assign(col, col + nnz);
    a->val.assign(val, val + nnz);
    return a;
}
extern "C" void or_csr_free(or_csr *a) { delete a; }
extern "C" void or_csr_info(const or_csr *a, int32_t *r, int32_t *c, int64_t *nnz) {
    *r = a->n_rows; *c = a->n_cols; *nnz = (int64_t)a->col.size();
}
extern "C" void or_csr_copy(const or_csr *a, int32_t *rowptr, int32_t *col, double *val) {
    if (rowptr) std::memcpy(rowptr, a->rowptr.data(), sizeof(int32_t) * a->rowptr.size());
    if (col) std::memcpy(col, a->col.data(), sizeof(int32_t) * a->col.size());
    if (val) std::memcpy(val, a->val.data(), sizeof(double) * a->val.size());
}
// Threads used by the row loops of the oracle (1 = the faithful single-threaded
// reference; more threads only split the row range, each row still sums in order).
int g_or_threads = 1;
extern "C" void or_set_threads(int n) { g_or_threads = n < 1 ? 1 : n; }

// CsrMatrix.Multiply (external MSolve; managed provider, GeometricMultigridSolver.cs:355,367):
// each row summed from 0.0 in stored order.
extern "C" void or_csr_spmv(const or_csr *a, const double *x, double *y) {
#pragma omp parallel for schedule(static) num_threads(g_or_threads) if (g_or_threads > 1)
    for (int32_t i = 0; i < a->n_rows; ++i) {
        double s = 0.0;
        for (int32_t k = a->rowptr[i]; k < a->rowptr[i + 1]; ++k) s += a->val[k] * x[a->col[k]];
        y[i] = s;
    }
}
// Forward Gauss-Seidel in row order.  The CSR variant used by the reference is
// MSolve's GaussSeidelIterationCsr (GeometricMultigridSolver.cs:305, external);
// it is restated as the same sweep as GaussSeidelIterationCsrDuVi.cs:22-50:
// x_i = (b_i - sum_{j != i} a_ij x_j) / a_ii, accumulated in column order.
extern "C" void or_csr_gs_forward(const or_csr *a, const double *b, double *x) {
    for (int32_t i = 0; i < a->n_rows; ++i) {
        double s = b[i], d = 0.0;
        for (int32_t k = a->rowptr[i]; k < a->rowptr[i + 1]; ++k) {
            int32_t c = a->col[k];
            if (c != i) s -= a->val[k] * x[c];
            else d = a->val[k];
        }
        x[i] = s / d;
    }
}

// ---------------------------------------------------------------------------
// DOK builder semantics
// ---------------------------------------------------------------------------
Dok Dok::submatrix(const std::vector<int32_t> &keep_rows, const std::vector<int32_t> &keep_cols) const {
    std::vector<int32_t> old_to_new(n_cols, -1);
    for (size_t j = 0; j < keep_cols.size(); ++j) old_to_new[keep_cols[j]] = (int32_t)j;
    Dok r((int32_t)keep_rows.size(), (int32_t)keep_cols.size());
    for (size_t i = 0; i < keep_rows.size(); ++i) {
        for (auto &cv : rows[keep_rows[i]].entries) {
            int32_t j = old_to_new[cv.first];
            if (j >= 0) r.rows[i].set(j, cv.second);
        }
    }
    return r;
}

or_csr *Dok::to_csr(bool sorted) const {
    or_csr *a = new or_csr;
    a->n_rows = n_rows;
    a->n_cols = n_cols;
    a->rowptr.resize(n_rows + 1);
    int64_t nnz = 0;
    for (int32_t i = 0; i < n_rows; ++i) { a->rowptr[i] = (int32_t)nnz; nnz += (int64_t)rows[i].entries.size(); }
    a->rowptr[n_rows] = (int32_t)nnz;
    a->col.resize(nnz);
    a->val.resize(nnz);
    int64_t k = 0;
    for (int32_t i = 0; i < n_rows; ++i) {
        auto e = rows[i].entries;
        if (sorted) std::stable_sort(e.begin(), e.end(), [](auto &p, auto &q) { return p.first < q.first; });
        for (auto &cv : e) { a->col[k] = cv.first; a->val[k] = cv.second; ++k; }
    }
    return a;
}

// ---------------------------------------------------------------------------
// Element stiffness
// ---------------------------------------------------------------------------
std::vector<double> element_stiffness(int dim, double E, double v) {
    if (dim == 2) {
        // FemCantilever2D.cs:29-49 (top88 quad, 2 dofs/node).
        double k[8] = {0.5 - v / 6.0, 0.125 + v / 8.0, -0.25 - v / 12.0, -0.125 + 3 * v / 8.0,
                       -0.25 + v / 12.0, -0.125 - v / 8.0, v / 6.0, 0.125 - 3 * v / 8.0};
        static const int idx[8][8] = {{0, 1, 2, 3, 4, 5, 6, 7}, {1, 0, 7, 6, 5, 4, 3, 2},
                                      {2, 7, 0, 5, 6, 3, 4, 1}, {3, 6, 5, 0, 7, 2, 1, 4},
                                      {4, 5, 6, 7, 0, 1, 2, 3}, {5, 4, 3, 2, 1, 0, 7, 6},
                                      {6, 3, 4, 1, 2, 7, 0, 5}, {7, 2, 1, 4, 3, 6, 5, 0}};
        double f = E / (1 - v * v);
        std::vector<double> ke(64);
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) ke[i * 8 + j] = k[idx[i][j]] * f;
        return ke;
    }
    // FemCantilever3D.cs:225-313 (top3d hexa, 3 dofs/node).
    static const double A[2][14] = {{32, 6, -8, 6, -6, 4, 3, -6, -10, 3, -3, -3, -4, -8},
                                    {-48, 0, 0, -24, 24, 0, 0, 0, 12, -12, 0, 12, 12, 12}};
    double k[15];
    k[0] = 0;
    for (int i = 0; i < 14; ++i) {
        double t = 0.0;           // A^T * [1, v]: managed dot product from 0
        t += A[0][i] * 1.0;
        t += A[1][i] * v;
        k[i + 1] = t * (1.0 / 72.0);   // ScaleIntoThis(1.0 / 72.0)
    }
    static const int K1[6][6] = {{1, 2, 2, 3, 5, 5}, {2, 1, 2, 4, 6, 7}, {2, 2, 1, 4, 7, 6},
                                 {3, 4, 4, 1, 8, 8}, {5, 6, 7, 8, 1, 2}, {5, 7, 6, 8, 2, 1}};
    static const int K2[6][6] = {{9, 8, 12, 6, 4, 7}, {8, 9, 12, 5, 3, 5}, {10, 10, 13, 7, 4, 6},
                                 {6, 5, 11, 9, 2, 10}, {4, 3, 5, 2, 9, 12}, {11, 4, 6, 12, 10, 13}};
    static const int K3[6][6] = {{6, 7, 4, 9, 12, 8}, {7, 6, 4, 10, 13, 10}, {5, 5, 3, 8, 12, 9},
                                 {9, 10, 2, 6, 11, 5}, {12, 13, 10, 11, 6, 4}, {2, 12, 9, 4, 5, 3}};
    static const int K4[6][6] = {{14, 11, 11, 13, 10, 10}, {11, 14, 11, 12, 9, 8}, {11, 11, 14, 12, 8, 9},
                                 {13, 12, 12, 14, 7, 7}, {10, 9, 8, 7, 14, 11}, {10, 8, 9, 7, 11, 14}};
    static const int K5[6][6] = {{1, 2, 8, 3, 5, 4}, {2, 1, 8, 4, 6, 11}, {8, 8, 1, 5, 11, 6},
                                 {3, 4, 5, 1, 8, 2}, {5, 6, 11, 8, 1, 8}, {4, 11, 6, 2, 8, 1}};
    static const int K6[6][6] = {{14, 11, 7, 13, 10, 12}, {11, 14, 7, 12, 9, 2}, {7, 7, 14, 10, 2, 9},
                                 {13, 12, 10, 14, 7, 11}, {10, 9, 2, 7, 14, 7}, {12, 2, 9, 11, 7, 14}};
    // Block layout {K1,K2,K3,K4; K2',K5,K6,K3'; K3',K6,K5',K2'; K4,K3,K2,K1'}.
    const int (*blk[4][4])[6] = {{K1, K2, K3, K4}, {K2, K5, K6, K3}, {K3, K6, K5, K2}, {K4, K3, K2, K1}};
    const bool tr[4][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {1, 0, 1, 1}, {0, 0, 0, 1}};
    double f = E / ((v + 1) * (1 - 2 * v));
    std::vector<double> ke(576);
    for (int bi = 0; bi < 4; ++bi)
        for (int bj = 0; bj < 4; ++bj)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    int m = tr[bi][bj] ? blk[bi][bj][j][i] : blk[bi][bj][i][j];
                    ke[(bi * 6 + i) * 24 + bj * 6 + j] = k[m] * f;
                }
    return ke;
}

extern "C" void or_model_element_stiffness(int dim, double E, double nu, double *ke) {
    auto k = element_stiffness(dim, E, nu);
    std::memcpy(ke, k.data(), sizeof(double) * k.size());
}

void Mesh::element_nodes(int32_t e, int32_t *out) const {
    int32_t a = e % ne[0];
    int32_t b = (e / ne[0]) % ne[1];
    int32_t c = e / (ne[0] * ne[1]);
    if (dim == 2) {
        out[0] = node_id(a, b, 0); out[1] = node_id(a + 1, b, 0);
        out[2] = node_id(a + 1, b + 1, 0); out[3] = node_id(a, b + 1, 0);
        return;
    }
    out[0] = node_id(a, b, c);         out[1] = node_id(a + 1, b, c);
    out[2] = node_id(a + 1, b + 1, c); out[3] = node_id(a, b + 1, c);
    out[4] = node_id(a, b, c + 1);     out[5] = node_id(a + 1, b, c + 1);
    out[6] = node_id(a + 1, b + 1, c + 1); out[7] = node_id(a, b + 1, c + 1);
}

// ---------------------------------------------------------------------------
// Cantilever model (FemCantileverBase.cs, FemCantilever3D.cs, FemCantilever2D.cs)
// ---------------------------------------------------------------------------
struct or_model {
    Mesh mesh;
    double E = 1, nu = 0.3, q = 1, I = 0;
    int dofs_per_node = 3;
    std::vector<int32_t> free_dofs;
    Dok *kff_dok = nullptr;
    or_csr *kff = nullptr;
    std::vector<double> uf, b;
    ~or_model() { delete kff_dok; delete kff; }
};

static Mesh make_mesh(int dim, const int32_t *ne, const double *len) {
    Mesh m;
    m.dim = dim;
    for (int a = 0; a < 3; ++a) { m.ne[a] = 1; m.nn[a] = 1; m.len[a] = len[a]; }
    for (int a = 0; a < dim; ++a) { m.ne[a] = ne[a]; m.nn[a] = ne[a] + 1; }
    return m;
}

// FindFreeDofs (FemCantileverBase.cs:137-158): all dofs of nodes with x index > 0.
static std::vector<int32_t> find_free_dofs(const Mesh &m, int dpn) {
    std::vector<int32_t> f;
    for (int32_t n = 0; n < m.nodes_total(); ++n) {
        if (n % m.nn[0] == 0) continue;
        for (int d = 0; d < dpn; ++d) f.push_back(dpn * n + d);
    }
    return f;
}

extern "C" or_model *or_model_create(int dim, const int32_t *ne, const double *len, double E,
                                     double nu, double q, const double *densities) {
    or_model *m = new or_model;
    m->mesh = make_mesh(dim, ne, len);
    m->E = E; m->nu = nu; m->q = q;
    m->dofs_per_node = dim;
    // Moment of inertia passed by the constructors (FemCantilever3D.cs:220-222, FemCantilever2D.cs:22-24).
    if (dim == 3) m->I = len[1] * len[2] / 12 * len[2] * len[2];
    else m->I = len[1] * len[2] / 12 * len[1] * len[1];
    const Mesh &M = m->mesh;
    int dpn = dim, npe = M.nodes_per_element(), ned = npe * dpn;
    int32_t n_all = dpn * M.nodes_total();
    // AssembleGlobalMatrix (FemCantileverBase.cs:87-104).
    std::vector<double> ke = element_stiffness(dim, E, nu);
    Dok K(n_all, n_all);
    std::vector<double> sub(ned * ned);
    int32_t nodes[8], g[24];
    for (int32_t e = 0; e < M.elements_total(); ++e) {
        M.element_nodes(e, nodes);
        for (int a = 0; a < npe; ++a)
            for (int d = 0; d < dpn; ++d) g[a * dpn + d] = dpn * nodes[a] + d;
        double dens = densities ? densities[e] : 1.0;
        for (int i = 0; i < ned * ned; ++i) sub[i] = dens * ke[i];   // density * Ke
        for (int i = 0; i < ned; ++i)
            for (int j = 0; j < ned; ++j) K.rows[g[i]].add(g[j], sub[i * ned + j]);
    }
    m->free_dofs = find_free_dofs(M, dpn);
    m->kff_dok = new Dok(K.submatrix(m->free_dofs, m->free_dofs));
    m->kff = m->kff_dok->to_csr(true);
    // CalcFreeDisplacements (FemCantileverBase.cs:160-182) with the Euler-Bernoulli
    // field (FemCantileverBase.cs:70-82) and CalcKnownDisplacementsForNode.
    double L = len[0];
    double dx[3];
    for (int a = 0; a < 3; ++a) dx[a] = a < dim ? len[a] / ne[a] : 0.0;
    for (int32_t n = 0; n < M.nodes_total(); ++n) {
        int32_t i = n % M.nn[0], j = (n / M.nn[0]) % M.nn[1], k = n / (M.nn[0] * M.nn[1]);
        if (i == 0) continue;
        double c[3] = {i * dx[0], j * dx[1], k * dx[2]};
        double x = c[0];
        double z = dim == 3 ? c[2] - (len[2] - 0.0) / 2 : c[1] - (len[1] - 0.0) / 2;
        double w = -q / (24 * E * m->I) * (std::pow(x, 4) - 4 * L * std::pow(x, 3) + 6 * L * L * x * x);
        double rot = -q / (6 * E * m->I) * (std::pow(x, 3) - 3 * L * x * x + 3 * L * L * x);
        double u = -rot * z;
        if (dim == 3) { m->uf.push_back(u); m->uf.push_back(0.0); m->uf.push_back(w); }
        else { m->uf.push_back(u); m->uf.push_back(w); }
    }
    // Ff = Kff.MultiplyRight(Uf): unsorted CSR (insertion order), managed multiply.
    int32_t nf = (int32_t)m->free_dofs.size();
    m->b.assign(nf, 0.0);
    for (int32_t r = 0; r < nf; ++r) {
        double s = 0.0;
        for (auto &cv : m->kff_dok->rows[r].entries) s += cv.second * m->uf[cv.first];
        m->b[r] = s;
    }
    return m;
}
extern "C" void or_model_free(or_model *m) { delete m; }
extern "C" int32_t or_model_num_free(const or_model *m) { return (int32_t)m->free_dofs.size(); }
extern "C" int32_t or_model_num_all(const or_model *m) { return m->dofs_per_node * m->mesh.nodes_total(); }
extern "C" const or_csr *or_model_kff(const or_model *m) { return m->kff; }
extern "C" void or_model_rhs(const or_model *m, double *b) { std::memcpy(b, m->b.data(), sizeof(double) * m->b.size()); }
extern "C" void or_model_uf(const or_model *m, double *u) { std::memcpy(u, m->uf.data(), sizeof(double) * m->uf.size()); }
extern "C" void or_model_free_dofs(const or_model *m, int32_t *f) {
    std::memcpy(f, m->free_dofs.data(), sizeof(int32_t) * m->free_dofs.size());
}
// EigenValueUpperBound(DokRowMajor) (GeometricMultigridSolver.cs:144-151), row values
// enumerated in Dictionary insertion order.
extern "C" double or_model_row_ratio_bound(const or_model *m) {
    double l = 0;
    for (auto &row : m->kff_dok->rows) {
        double s = 0.0, mx = -INFINITY;
        for (auto &cv : row.entries) { double a = std::fabs(cv.second); s += a; if (a > mx) mx = a; }
        double r = s / mx;
        l = std::max(l, r);
    }
    return l;
}

// Consistent nodal forces of a uniform traction t on the face x = len[0]
// (build-defined load of the benchmark configurations; the reference uses the
// manufactured right-hand side instead).  Face elements are bilinear, so each
// face cell of area A adds A/4 * t to its 4 corner nodes (2-D: segment length/2).
extern "C" void or_traction_rhs(int dim, const int32_t *ne, const double *len, const double *t, double *b) {
    Mesh M = make_mesh(dim, ne, len);
    int dpn = dim;
    std::vector<int32_t> fd = find_free_dofs(M, dpn);
    std::vector<double> ball(dpn * M.nodes_total(), 0.0);
    int32_t i = M.ne[0];
    if (dim == 3) {
        double hy = len[1] / ne[1], hz = len[2] / ne[2], a4 = hy * hz / 4;
        for (int32_t c = 0; c < M.ne[2]; ++c)
            for (int32_t bb = 0; bb < M.ne[1]; ++bb) {
                int32_t nd[4] = {M.node_id(i, bb, c), M.node_id(i, bb + 1, c), M.node_id(i, bb, c + 1),
                                 M.node_id(i, bb + 1, c + 1)};
                for (int q = 0; q < 4; ++q)
                    for (int d = 0; d < 3; ++d) ball[3 * nd[q] + d] += a4 * t[d];
            }
    } else {
        double hy = len[1] / ne[1], a2 = hy / 2;
        for (int32_t bb = 0; bb < M.ne[1]; ++bb) {
            int32_t nd[2] = {M.node_id(i, bb, 0), M.node_id(i, bb + 1, 0)};
            for (int q = 0; q < 2; ++q)
                for (int d = 0; d < 2; ++d) ball[2 * nd[q] + d] += a2 * t[d];
        }
    }
    for (size_t r = 0; r < fd.size(); ++r) b[r] = ball[fd[r]];
}

// ---------------------------------------------------------------------------
// Restriction / interpolation (IGeometricMultigridModel.cs:76-194)
// ---------------------------------------------------------------------------
extern "C" void or_transfer_create(int dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                                   or_csr **restriction, or_csr **interpolation) {
    double unit_len[3] = {1, 1, 1};
    Mesh F = make_mesh(dim, ne_fine, unit_len), C = make_mesh(dim, ne_coarse, unit_len);
    int dpn = dim;
    int nfn[3] = {1, 1, 1}, ncn[3] = {1, 1, 1};
    double dist[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i) {
        dist[i] = (double)ne_fine[i] / ne_coarse[i];
        nfn[i] = ne_fine[i] + 1;
        ncn[i] = ne_coarse[i] + 1;
    }
    int32_t nf_all = dpn * F.nodes_total(), nc_all = dpn * C.nodes_total();
    Dok R(nc_all, nf_all), P(nf_all, nc_all);
    int a[3] = {0, 0, 0}, start[3] = {0, 0, 0}, end[3] = {0, 0, 0}, w[3] = {0, 0, 0};
    double cursor[3] = {0, 0, 0};
    std::vector<double> sum_interp(F.nodes_total(), 0.0);
    if (dim < 3) end[2] = 1;
    for (a[0] = 0; a[0] < ncn[0]; ++a[0])
        for (a[2] = 0; a[2] < ncn[2]; ++a[2])
            for (a[1] = 0; a[1] < ncn[1]; ++a[1]) {
                for (int i = 0; i < dim; ++i) {
                    cursor[i] = a[i] * dist[i];
                    start[i] = (int)std::ceil(std::nextafter(cursor[i] - dist[i], INFINITY));
                    if (start[i] < 0) start[i] = 0;
                    end[i] = (int)std::floor(std::nextafter(cursor[i] + dist[i], -INFINITY)) + 1;
                    if (end[i] > nfn[i]) end[i] = nfn[i];
                }
                int32_t cnode = C.node_id(a[0], a[1], dim == 3 ? a[2] : 0);
                int32_t cbase = cnode * dpn;
                double sum_r = 0;
                for (w[0] = start[0]; w[0] < end[0]; ++w[0])
                    for (w[2] = start[2]; w[2] < end[2]; ++w[2])
                        for (w[1] = start[1]; w[1] < end[1]; ++w[1]) {
                            int32_t fnode = F.node_id(w[0], w[1], dim == 3 ? w[2] : 0);
                            int32_t fbase = fnode * dpn;
                            double infl = 0;
                            for (int i = 0; i < dim; ++i) {
                                double d0 = (w[i] - cursor[i]) / dist[i];
                                infl += d0 * d0;
                            }
                            infl = 1 - std::sqrt(infl);
                            sum_r += infl;
                            sum_interp[fnode] += infl;
                            R.rows[cbase].set(fbase, infl);
                            P.rows[fbase].set(cbase, infl);
                        }
                DokRow &rr = R.rows[cbase];
                std::vector<int32_t> keys;
                for (auto &cv : rr.entries) keys.push_back(cv.first);
                for (int32_t key : keys) {
                    double v0 = 0.0;
                    rr.get(key, v0);
                    double value = v0 / sum_r;
                    rr.set(key, value);
                    for (int i = 1; i < dpn; ++i) R.rows[cbase + i].set(key + i, value);
                }
            }
    for (int32_t fnode = 0; fnode < F.nodes_total(); ++fnode) {
        int32_t fbase = fnode * dpn;
        DokRow &pr = P.rows[fbase];
        std::vector<int32_t> keys;
        for (auto &cv : pr.entries) keys.push_back(cv.first);
        for (int32_t key : keys) {
            double v0 = 0.0;
            pr.get(key, v0);
            double value = v0 / sum_interp[fnode];
            pr.set(key, value);
            for (int i = 1; i < dpn; ++i) P.rows[fbase + i].set(key + i, value);
        }
    }
    std::vector<int32_t> ff = find_free_dofs(F, dpn), cf = find_free_dofs(C, dpn);
    *restriction = R.submatrix(cf, ff).to_csr(true);
    *interpolation = P.submatrix(ff, cf).to_csr(true);
}

// ---------------------------------------------------------------------------
// Build-defined structured pieces (benchmark hierarchy), 3-D only.
// ---------------------------------------------------------------------------
// Row-wise assembly of K = sum_e (scale*E_e) Ke over free dofs, each entry
// summed in increasing element id, exactly as the DOK assembly orders its adds.
extern "C" or_csr *or_hex_stiffness(const int32_t *ne, const double *elem_E, double scale, double E, double nu) {
    double len[3] = {(double)ne[0], (double)ne[1], (double)ne[2]};
    Mesh M = make_mesh(3, ne, len);
    std::vector<double> ke = element_stiffness(3, E, nu);
    int32_t nx = M.nn[0], ny = M.nn[1], nz = M.nn[2];
    int32_t nf = 3 * (nx - 1) * ny * nz;
    or_csr *A = new or_csr;
    A->n_rows = A->n_cols = nf;
    A->rowptr.assign(nf + 1, 0);
    auto free_index = [&](int32_t i, int32_t j, int32_t k) -> int32_t {   // node -> first free dof
        return 3 * ((i - 1) + (nx - 1) * (j + ny * k));
    };
    // Row lengths.
    for (int32_t k = 0; k < nz; ++k)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t i = 1; i < nx; ++i) {
                int cnt = 0;
                for (int dk = -1; dk <= 1; ++dk)
                    for (int dj = -1; dj <= 1; ++dj)
                        for (int di = -1; di <= 1; ++di) {
                            int32_t ii = i + di, jj = j + dj, kk = k + dk;
                            if (ii < 1 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
                            ++cnt;
                        }
                int32_t r = free_index(i, j, k);
                for (int d = 0; d < 3; ++d) A->rowptr[r + d + 1] = 3 * cnt;
            }
    for (int32_t r = 0; r < nf; ++r) A->rowptr[r + 1] += A->rowptr[r];
    A->col.resize(A->rowptr[nf]);
    A->val.resize(A->rowptr[nf]);
#pragma omp parallel for collapse(2) schedule(static) num_threads(g_or_threads) if (g_or_threads > 1)
    for (int32_t k = 0; k < nz; ++k)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t i = 1; i < nx; ++i) {
                int32_t r0 = free_index(i, j, k);
                for (int d = 0; d < 3; ++d) {
                    int32_t p = A->rowptr[r0 + d];
                    for (int dk = -1; dk <= 1; ++dk)
                        for (int dj = -1; dj <= 1; ++dj)
                            for (int di = -1; di <= 1; ++di) {
                                int32_t ii = i + di, jj = j + dj, kk = k + dk;
                                if (ii < 1 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
                                for (int d2 = 0; d2 < 3; ++d2) {
                                    double s = 0.0;
                                    bool first = true;
                                    // elements containing both nodes, increasing id: (c, b, a) lexicographic
                                    for (int32_t c = std::max(std::max(k, kk) - 1, 0); c <= std::min(std::min(k, kk), ne[2] - 1); ++c)
                                        for (int32_t b = std::max(std::max(j, jj) - 1, 0); b <= std::min(std::min(j, jj), ne[1] - 1); ++b)
                                            for (int32_t a = std::max(std::max(i, ii) - 1, 0); a <= std::min(std::min(i, ii), ne[0] - 1); ++a) {
                                                int32_t e = a + ne[0] * (b + ne[1] * c);
                                                int la = (i - a) + 2 * (j - b) + 4 * (k - c);
                                                int lb = (ii - a) + 2 * (jj - b) + 4 * (kk - c);
                                                static const int vtk[8] = {0, 1, 3, 2, 4, 5, 7, 6};
                                                la = vtk[la]; lb = vtk[lb];
                                                double ce = elem_E ? scale * elem_E[e] : scale;
                                                double t = ce * ke[(3 * la + d) * 24 + 3 * lb + d2];
                                                if (first) { s = t + 0.0; first = false; }
                                                else s = t + s;
                                            }
                                    A->col[p] = free_index(ii, jj, kk) + d2;
                                    A->val[p] = s;
                                    ++p;
                                }
                            }
                }
            }
    return A;
}

// Trilinear interpolation (fine free dofs x coarse free dofs) for factor-2 grids.
// Trilinear prolongation of a factor-2 vertex coarsening (free dofs of the
// clamped cantilever, x-fastest nodes, 3 dofs per node).  Per axis with n
// elements the coarse nodes are the even fine nodes plus the last fine node;
// an odd fine node between two coarse nodes takes 1/2 of each, every other
// fine node coincides with one coarse node.  Even n: the standard trilinear P.
static int or_coarse_axis(int32_t i, int32_t n, int32_t c[2], double w[2]) {
    if ((i % 2 == 1) && i != n) {
        c[0] = (i - 1) / 2;
        c[1] = (i + 1) / 2;
        w[0] = 0.5;
        w[1] = 0.5;
        return 2;
    }
    c[0] = (i == n) ? (n + 1) / 2 : i / 2;
    w[0] = 1.0;
    return 1;
}

extern "C" or_csr *or_hex_trilinear(const int32_t *nef) {
    int32_t nx = nef[0] + 1, ny = nef[1] + 1, nz = nef[2] + 1;
    int32_t cx = (nef[0] + 1) / 2 + 1, cy = (nef[1] + 1) / 2 + 1, cz = (nef[2] + 1) / 2 + 1;
    int32_t nf = 3 * (nx - 1) * ny * nz, nc = 3 * (cx - 1) * cy * cz;
    or_csr *P = new or_csr;
    P->n_rows = nf; P->n_cols = nc;
    P->rowptr.push_back(0);
    for (int32_t k = 0; k < nz; ++k)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t i = 1; i < nx; ++i)
                for (int d = 0; d < 3; ++d) {
                    int32_t ci[2], cj[2], ck[2];
                    double wi[2], wj[2], wk[2];
                    int ni = or_coarse_axis(i, nef[0], ci, wi);
                    int nj = or_coarse_axis(j, nef[1], cj, wj);
                    int nk = or_coarse_axis(k, nef[2], ck, wk);
                    // columns sorted: k outer, j, i inner
                    for (int c = 0; c < nk; ++c)
                        for (int b = 0; b < nj; ++b)
                            for (int a = 0; a < ni; ++a) {
                                if (ci[a] == 0) continue;   // clamped coarse node
                                P->col.push_back(3 * ((ci[a] - 1) + (cx - 1) * (cj[b] + cy * ck[c])) + d);
                                P->val.push_back(wi[a] * wj[b] * wk[c]);
                            }
                    P->rowptr.push_back((int32_t)P->col.size());
                }
    return P;
}

// Galerkin P^T A P with sorted rows (sparse accumulator, sums in k-order).
extern "C" or_csr *or_galerkin(const or_csr *A, const or_csr *P) {
    int32_t nc = P->n_cols, nf = P->n_rows;
    // transpose P
    std::vector<int32_t> tp(nc + 1, 0), tc(P->col.size());
    std::vector<double> tv(P->col.size());
    for (int32_t c : P->col) tp[c + 1]++;
    for (int32_t i = 0; i < nc; ++i) tp[i + 1] += tp[i];
    std::vector<int32_t> fill(tp.begin(), tp.end() - 1);
    for (int32_t r = 0; r < nf; ++r)
        for (int32_t k = P->rowptr[r]; k < P->rowptr[r + 1]; ++k) {
            int32_t c = P->col[k];
            tc[fill[c]] = r; tv[fill[c]] = P->val[k]; fill[c]++;
        }
    or_csr *G = new or_csr;
    G->n_rows = G->n_cols = nc;
    G->rowptr.push_back(0);
    std::vector<double> acc(nc, 0.0);
    std::vector<char> mark(nc, 0);
    std::vector<int32_t> cols;
    for (int32_t I = 0; I < nc; ++I) {
        cols.clear();
        for (int32_t k = tp[I]; k < tp[I + 1]; ++k) {
            int32_t r = tc[k];
            double pr = tv[k];
            for (int32_t q = A->rowptr[r]; q < A->rowptr[r + 1]; ++q) {
                int32_t j = A->col[q];
                double ar = pr * A->val[q];
                for (int32_t s = P->rowptr[j]; s < P->rowptr[j + 1]; ++s) {
                    int32_t J = P->col[s];
                    if (!mark[J]) { mark[J] = 1; acc[J] = 0.0; cols.push_back(J); }
                    acc[J] += ar * P->val[s];
                }
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int32_t J : cols) { G->col.push_back(J); G->val.push_back(acc[J]); mark[J] = 0; }
        G->rowptr.push_back((int32_t)G->col.size());
    }
    return G;
}
