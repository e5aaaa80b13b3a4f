// On-device assembly of the structured hexahedral stiffness (free dofs, sorted CSR).
//
// The reference assembles element by element into a dictionary-of-keys builder
// (FemCantileverBase.AssembleGlobalMatrix, FemCantileverBase.cs:87-104, through
// DokRowMajor.AddSubmatrix, DokRowMajor.cs:182-207) and converts it to CSR
// (DokRowMajor.BuildCsrArrays, :286-324).  Every stored entry (i, j) is therefore
// the sum, in increasing element id, of (scale * E_e) * Ke(a_i, a_j) over the
// elements that contain both dofs, the first term added to +0.0; rows are sorted
// by column and structural zeros are kept.  Here one thread owns one free node
// (its three rows) and writes its entries straight into the CSR arrays, with
// separately rounded products and sums in exactly that order, so the arrays equal
// the host assembler's (dv_hex_assemble) bit for bit.  Row offsets are closed-form:
// the number of stored columns of a node is a product of per-axis neighbour
// counts, so the entries before a node are sums of per-axis prefix counts.
//
// dv_matrix_create_hex builds the matrix-free form of the same operator (the element
// kernel k_hex_elem): the per-element factors on the device, the value classes of Ke,
// and the diagonal for Jacobi weights (summed on the host in the assembly's order, so it
// equals the assembled matrix's diagonal bit for bit).
#include "dv_kernels.cuh"

#include <algorithm>
#include <vector>

using namespace dvk;

namespace {

struct HexAxes {
    int32_t nx, ny, nz;            // node counts per axis (x: node 0 is clamped)
    int32_t ne0, ne1, ne2;         // element counts per axis
    int64_t sx, sy;                // sums of the x (free nodes) and y neighbour counts
};

// neighbours of a node along one axis (itself included); x counts free nodes 1..nx-1 only
__device__ __forceinline__ int nbr_x(int32_t i, int32_t nx) { return (i > 1 ? 1 : 0) + 1 + (i + 1 < nx ? 1 : 0); }
__device__ __forceinline__ int nbr_yz(int32_t j, int32_t n) { return (j > 0 ? 1 : 0) + 1 + (j + 1 < n ? 1 : 0); }
// sums of those counts over the nodes before i: free x nodes 1..i-1 (3 each, minus node 1's
// missing -x neighbour); y or z nodes 0..j-1 (3 each, minus node 0's missing -y neighbour)
__device__ __forceinline__ int64_t pre_x(int32_t i) { return i <= 1 ? 0 : 3 * (int64_t)(i - 1) - 1; }
__device__ __forceinline__ int64_t pre_yz(int32_t j) { return j <= 0 ? 0 : 3 * (int64_t)j - 1; }

__global__ void k_hex_assemble(HexAxes H, const double *__restrict__ ke_g, const double *__restrict__ elem_E,
                               double scale, int32_t *__restrict__ rowptr, int32_t *__restrict__ col,
                               double *__restrict__ val) {
    __shared__ double ke[576];
    __shared__ int vtk[8];
    for (int t = threadIdx.x; t < 576; t += blockDim.x) ke[t] = ke_g[t];
    if (threadIdx.x < 8) {
        const int v[8] = {0, 1, 3, 2, 4, 5, 7, 6};   // lexicographic corner (dx + 2 dy + 4 dz) -> VTK hexa order
        vtk[threadIdx.x] = v[threadIdx.x];
    }
    __syncthreads();
    const int32_t fx = H.nx - 1;   // free nodes per x line
    const int64_t nodes = (int64_t)fx * H.ny * H.nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nodes; q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = (int32_t)(q % fx) + 1, j = (int32_t)((q / fx) % H.ny), k = (int32_t)(q / ((int64_t)fx * H.ny));
        const int cx = nbr_x(i, H.nx), cy = nbr_yz(j, H.ny), cz = nbr_yz(k, H.nz);
        // stored entries before this node: 9 per pair of neighbouring nodes (3 rows x 3 columns)
        const int64_t before = 9 * (pre_yz(k) * H.sy * H.sx + (int64_t)cz * pre_yz(j) * H.sx + (int64_t)cz * cy * pre_x(i));
        const int32_t per_row = 3 * cx * cy * cz;
        const int32_t r0 = (int32_t)(3 * q);
        for (int d = 0; d < 3; ++d) {
            int64_t p = before + (int64_t)d * per_row;
            rowptr[r0 + d] = (int32_t)p;
            if (q == nodes - 1 && d == 2) rowptr[r0 + 3] = (int32_t)(p + per_row);
            for (int dk = -1; dk <= 1; ++dk)
                for (int dj = -1; dj <= 1; ++dj)
                    for (int di = -1; di <= 1; ++di) {
                        const int32_t ii = i + di, jj = j + dj, kk = k + dk;
                        if (ii < 1 || ii >= H.nx || jj < 0 || jj >= H.ny || kk < 0 || kk >= H.nz) continue;
                        const int32_t c0 = max(max(k, kk) - 1, 0), c1 = min(min(k, kk), H.ne2 - 1);
                        const int32_t b0 = max(max(j, jj) - 1, 0), b1 = min(min(j, jj), H.ne1 - 1);
                        const int32_t a0 = max(max(i, ii) - 1, 0), a1 = min(min(i, ii), H.ne0 - 1);
                        const int32_t cbase = 3 * ((ii - 1) + fx * (jj + H.ny * kk));
                        for (int d2 = 0; d2 < 3; ++d2) {
                            double s = 0.0;
                            bool first = true;
                            for (int32_t c = c0; c <= c1; ++c)
                                for (int32_t b = b0; b <= b1; ++b)
                                    for (int32_t a = a0; a <= a1; ++a) {
                                        const int64_t e = a + (int64_t)H.ne0 * (b + (int64_t)H.ne1 * c);
                                        const int la = vtk[(i - a) + 2 * (j - b) + 4 * (k - c)];
                                        const int lb = vtk[(ii - a) + 2 * (jj - b) + 4 * (kk - c)];
                                        const double ce = elem_E ? __dmul_rn(scale, __ldg(elem_E + e)) : scale;
                                        const double t = __dmul_rn(ce, ke[(3 * la + d) * 24 + 3 * lb + d2]);
                                        s = first ? __dadd_rn(t, 0.0) : __dadd_rn(t, s);
                                        first = false;
                                    }
                            col[p] = cbase + d2;
                            val[p] = s;
                            ++p;
                        }
                    }
        }
    }
}

}  // namespace

extern "C" DV_API int dv_hex_assemble_device(dv_context *ctx, const int32_t *ne, const double *d_elem_E, double scale,
                                             double E, double nu, int32_t *d_rowptr, int32_t *d_col, double *d_val) {
    return dv_guard([&] {
        dv_ctx_check(ctx);
        int32_t nrows;
        int64_t nnz;
        const int st = dv_hex_csr_size(ne, &nrows, &nnz);
        DV_REQUIRE(st == DV_OK, st, "bad mesh");
        DV_REQUIRE(d_rowptr && d_col && d_val, DV_ERR_ARG, "null output array");
        DV_REQUIRE(nnz < INT32_MAX, DV_ERR_ARG, "more stored entries than int32 row offsets hold");
        std::vector<double> ke(576);
        dv_hex_ke(E, nu, ke.data());
        cudaStream_t s = ctx->stream;
        DevMem dke(sizeof(double) * 576);
        DV_CUDA(cudaMemcpyAsync(dke.p, ke.data(), sizeof(double) * 576, cudaMemcpyHostToDevice, s));
        HexAxes H;
        H.nx = ne[0] + 1;
        H.ny = ne[1] + 1;
        H.nz = ne[2] + 1;
        H.ne0 = ne[0];
        H.ne1 = ne[1];
        H.ne2 = ne[2];
        auto total = [](int32_t n, bool clamp) {   // sum of the neighbour counts along one axis
            int64_t t = 0;
            for (int32_t i = clamp ? 1 : 0; i < n; ++i) t += (clamp ? (i > 1) : (i > 0)) + 1 + (i + 1 < n);
            return t;
        };
        H.sx = total(H.nx, true);
        H.sy = total(H.ny, false);
        const int64_t nodes = (int64_t)nrows / 3;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nodes + 127) / 128, (int64_t)ctx->num_sms * 16));
        k_hex_assemble<<<blocks, 128, 0, s>>>(H, dke.as<double>(), d_elem_E, scale, d_rowptr, d_col, d_val);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        DV_CUDA(cudaStreamSynchronize(s));   // dke is released on return
    });
}

// Matrix-free operator of several meshes (block-diagonal, meshes in the given order); ne holds
// 3 element counts per mesh, elem_E (or NULL) the moduli of all meshes' elements in order.
dv_matrix *dv_hex_operator_build(dv_context *ctx, int32_t nmesh, const int32_t *ne, const double *elem_E, double scale,
                                 double E, double nu, int32_t precision) {
    DV_REQUIRE(ne && nmesh >= 1, DV_ERR_ARG, "null argument");
    DV_REQUIRE(precision == DV_F64 || precision == DV_F32, DV_ERR_ARG, "precision must be DV_F64 or DV_F32");
    dv_ctx_check(ctx);
    std::vector<double> ke(576);
    dv_hex_ke(E, nu, ke.data());
    auto m = std::make_unique<dv_matrix>();
    bool seen[kKeClasses] = {};
    for (int i = 0; i < 576; ++i) {
        const int c = ke_class(i);
        if (!seen[c]) {
            seen[c] = true;
            m->hex_cls[c] = ke[i];
        } else {
            DV_REQUIRE(ke[i] == m->hex_cls[c], DV_ERR_UNSUPPORTED, "element stiffness without the hexahedron's symmetries");
        }
    }
    // mesh table: tiles of 32 x 8 nodes over runs of z planes
    std::vector<HexMesh> meshes(nmesh);
    int64_t rows = 0, nnz = 0, nel = 0, tiles = 0;
    int64_t plane_tiles_all = 0;
    for (int32_t k = 0; k < nmesh; ++k) {
        const int32_t *n = ne + 3 * k;
        int32_t r;
        int64_t z;
        const int st = dv_hex_csr_size(n, &r, &z);
        DV_REQUIRE(st == DV_OK, st, "bad mesh");
        HexMesh &h = meshes[k];
        h.ne0 = n[0];
        h.ne1 = n[1];
        h.ne2 = n[2];
        h.ntx = (n[0] + kGridTX - 1) / kGridTX;
        h.nty = (n[1] + 1 + kGridTY - 1) / kGridTY;
        h.row0 = rows;
        h.fac0 = nel;
        h.pad = 0;
        rows += r;
        nnz += z;
        nel += (int64_t)n[0] * n[1] * n[2];
        plane_tiles_all += (int64_t)h.ntx * h.nty;
    }
    DV_REQUIRE(rows < INT32_MAX, DV_ERR_ARG, "operator exceeds int32 rows");
    // run length: one mesh from the waves x steps model; several meshes share a run of 8 planes
    const int64_t conc = (int64_t)ctx->num_sms * (precision == DV_F64 ? 1 : 3);
    for (auto &h : meshes) {
        h.zc = nmesh == 1 ? stream_run_length((int64_t)h.ntx * h.nty, h.ne2 + 1, conc) : 8;
        h.tile0 = (int32_t)tiles;
        tiles += (int64_t)h.ntx * h.nty * ((h.ne2 + 1 + h.zc - 1) / h.zc);
    }
    DV_REQUIRE(tiles < INT32_MAX, DV_ERR_ARG, "too many tiles");
    std::vector<double> f(nel);
    for (int64_t e = 0; e < nel; ++e) f[e] = elem_E ? scale * elem_E[e] : scale;
    m->ctx = ctx;
    m->n_rows = m->n_cols = (int32_t)rows;
    m->nnz = nnz;
    m->format = DV_FORMAT_HEX;
    m->precision = precision;
    for (int d = 0; d < 3; ++d) m->hex_ne[d] = ne[d];
    m->hex_nmesh = nmesh;
    m->hex_ntile = (int32_t)tiles;
    cudaStream_t s = ctx->stream;
    m->hex_meshes.alloc(sizeof(HexMesh) * meshes.size());
    DV_CUDA(cudaMemcpyAsync(m->hex_meshes.p, meshes.data(), sizeof(HexMesh) * meshes.size(), cudaMemcpyHostToDevice, s));
    if (precision == DV_F64) {
        m->hex_factor.alloc(8 * (size_t)nel);
        DV_CUDA(cudaMemcpyAsync(m->hex_factor.p, f.data(), 8 * (size_t)nel, cudaMemcpyHostToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<float> f32(f.begin(), f.end());
        m->hex_factor.alloc(4 * (size_t)nel);
        DV_CUDA(cudaMemcpyAsync(m->hex_factor.p, f32.data(), 4 * (size_t)nel, cudaMemcpyHostToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
    }
    // diagonal: sum over the node's elements in increasing id of (scale E_e) Ke(a, a), as assembled
    static const int vtk[8] = {0, 1, 3, 2, 4, 5, 7, 6};
    m->host_diag.assign(rows, 0.0);
    for (int32_t q = 0; q < nmesh; ++q) {
        const int32_t *n = ne + 3 * q;
        const int32_t nx = n[0] + 1, ny = n[1] + 1, nz = n[2] + 1;
        const double *fq = f.data() + meshes[q].fac0;
        double *dq = m->host_diag.data() + meshes[q].row0;
#pragma omp parallel for collapse(2) schedule(static)
        for (int32_t k = 0; k < nz; ++k)
            for (int32_t j = 0; j < ny; ++j)
                for (int32_t i = 1; i < nx; ++i) {
                    const int32_t r0 = 3 * ((i - 1) + (nx - 1) * (j + ny * k));
                    for (int d = 0; d < 3; ++d) {
                        double s2 = 0.0;
                        bool first = true;
                        for (int32_t c = std::max(k - 1, 0); c <= std::min(k, n[2] - 1); ++c)
                            for (int32_t b = std::max(j - 1, 0); b <= std::min(j, n[1] - 1); ++b)
                                for (int32_t a = std::max(i - 1, 0); a <= std::min(i, n[0] - 1); ++a) {
                                    const int64_t e = a + (int64_t)n[0] * (b + (int64_t)n[1] * c);
                                    const int la = vtk[(i - a) + 2 * (j - b) + 4 * (k - c)];
                                    const double t = fq[e] * ke[(3 * la + d) * 24 + 3 * la + d];
                                    s2 = first ? t + 0.0 : t + s2;
                                    first = false;
                                }
                        dq[r0 + d] = s2;
                    }
                }
    }
    m->zero_diag = std::any_of(m->host_diag.begin(), m->host_diag.end(), [](double d) { return d == 0.0; });
    m->diag.alloc(8 * (size_t)rows);
    DV_CUDA(cudaMemcpyAsync(m->diag.p, m->host_diag.data(), 8 * (size_t)rows, cudaMemcpyHostToDevice, s));
    DV_CUDA(cudaStreamSynchronize(s));
    m->device_bytes = (int64_t)(precision == DV_F64 ? 8 : 4) * nel;
    return m.release();
}

extern "C" DV_API int dv_matrix_create_hex(dv_context *ctx, const int32_t *ne, const double *elem_E, double scale,
                                           double E, double nu, int32_t precision, dv_matrix **out) {
    return dv_guard([&] {
        DV_REQUIRE(ne && out, DV_ERR_ARG, "null argument");
        *out = dv_hex_operator_build(ctx, 1, ne, elem_E, scale, E, nu, precision);
    });
}

dv_matrix *dv_trilinear_build(dv_context *ctx, const int32_t *nef, int restrict_, int32_t precision) {
    DV_REQUIRE(nef && nef[0] >= 2 && nef[1] >= 2 && nef[2] >= 2, DV_ERR_ARG, "element counts must be >= 2");
    DV_REQUIRE(!(nef[0] & 1) && !(nef[1] & 1) && !(nef[2] & 1), DV_ERR_UNSUPPORTED,
               "matrix-free transfers need even element counts");
    DV_REQUIRE(precision == DV_F64 || precision == DV_F32, DV_ERR_ARG, "precision must be DV_F64 or DV_F32");
    dv_ctx_check(ctx);
    int32_t nr, nc;
    int64_t nnz;
    const int st = dv_hex_trilinear_size(nef, &nr, &nc, &nnz);
    DV_REQUIRE(st == DV_OK, st, "bad mesh");
    auto m = std::make_unique<dv_matrix>();
    m->ctx = ctx;
    m->n_rows = restrict_ ? nc : nr;
    m->n_cols = restrict_ ? nr : nc;
    m->nnz = nnz;
    m->format = DV_FORMAT_TRILINEAR;
    m->precision = precision;
    for (int d = 0; d < 3; ++d) m->tri_ne[d] = nef[d];
    m->tri_restrict = restrict_ ? 1 : 0;
    m->device_bytes = 0;
    return m.release();
}

extern "C" DV_API int dv_matrix_create_trilinear(dv_context *ctx, const int32_t *ne_fine, int32_t restrict_,
                                                 int32_t precision, dv_matrix **out) {
    return dv_guard([&] {
        DV_REQUIRE(out, DV_ERR_ARG, "null argument");
        *out = dv_trilinear_build(ctx, ne_fine, restrict_, precision);
    });
}
