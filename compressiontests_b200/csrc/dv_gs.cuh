// Gauss-Seidel row updates shared by the stationary multigrid (dv_gmg.cu) and
// the V-cycle of the multigrid-preconditioned CG (dv_mgpcg.cuh).
//
// Row update x_i = (b_i - sum_{j != i} a_ij x_j) / a_ii in column order, each
// product and difference rounded separately (GaussSeidelIterationCsrDuVi.cs:22-50).
// A launch updates the rows of one independent group: one dependency level of
// the forward sweep (the reference's own order) or the node blocks of one color.
#pragma once

#include "dv_kernels.cuh"

namespace dvk {

template <class T> __device__ __forceinline__ T rn_mul(T a, T b);
template <> __device__ __forceinline__ double rn_mul<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float rn_mul<float>(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ __forceinline__ T rn_sub(T a, T b);
template <> __device__ __forceinline__ double rn_sub<double>(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float rn_sub<float>(float a, float b) { return __fsub_rn(a, b); }
template <class T> __device__ __forceinline__ T rn_div(T a, T b);
template <> __device__ __forceinline__ double rn_div<double>(double a, double b) { return __ddiv_rn(a, b); }
template <> __device__ __forceinline__ float rn_div<float>(float a, float b) { return __fdiv_rn(a, b); }

template <class T>
__device__ __forceinline__ void gs_row_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                           const T *__restrict__ va, const T *__restrict__ b, T *x, int32_t i) {
    T s = b[i], d = T(0);
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
        const int32_t c = ci[k];
        const T a = va[k];
        if (c != i) s = rn_sub<T>(s, rn_mul<T>(a, ((volatile T *)x)[c]));
        else d = a;
    }
    x[i] = rn_div<T>(s, d);
}

template <class VI, class T>
__device__ __forceinline__ void gs_row_duvi(const DuviArgs &A, const T *__restrict__ b, T *x, int32_t i) {
    const T *tab = static_cast<const T *>(A.values);
    const VI *vi = static_cast<const VI *>(A.vidx);
    T s = b[i], d = T(0);
    uint32_t di = A.row_to_dist[i];
    for (uint32_t bl = A.row_to_col[i]; bl < A.row_to_col[i + 1]; ++bl) {
        uint32_t c = A.col_idx[bl];
        const int cnt = A.dist[di];
        for (int k = 0;; ++k) {
            const T a = tab[vi[di]];
            if ((int32_t)c != i) s = rn_sub<T>(s, rn_mul<T>(a, ((volatile T *)x)[c]));
            else d = a;
            ++di;
            if (k == cnt) break;
            c += A.dist[di] + 1u;
        }
    }
    x[i] = rn_div<T>(s, d);
}

// rows[0..count): first rows of the group's blocks of bs consecutive rows
template <class T>
__global__ void k_gs_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci, const T *__restrict__ va,
                         const T *__restrict__ b, T *x, const int32_t *__restrict__ rows, int32_t count, int bs,
                         const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int32_t r0 = rows[t];
        for (int q = 0; q < bs; ++q) gs_row_csr<T>(rp, ci, va, b, x, r0 + q);
    }
}
template <class VI, class T>
__global__ void k_gs_duvi(DuviArgs A, const T *__restrict__ b, T *x, const int32_t *__restrict__ rows, int32_t count,
                          int bs, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int32_t r0 = rows[t];
        for (int q = 0; q < bs; ++q) gs_row_duvi<VI, T>(A, b, x, r0 + q);
    }
}

// Multicolor node-block update on the node-pattern layout: one thread per node of the color,
// its pattern's records from shared memory.  One pass over the records gathers every column
// of another node once and subtracts it from all three rows (fused multiply-adds); the node's
// own 3 x 3 block is then solved row by row in order, each row using the rows of the node
// already updated in this sweep and the old values of the later ones (the block Gauss-Seidel
// step of the raw kernels above, with the neighbour sum taken first).
template <class T>
__global__ void __launch_bounds__(256) k_gs_pattern(const uint16_t *__restrict__ pid, const uint32_t *__restrict__ pstart,
                                                    const PatRec<T> *__restrict__ grec, int32_t npat, int32_t nrec,
                                                    const T *__restrict__ b, T *x, const int32_t *__restrict__ rows,
                                                    int32_t count, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 gs_smem[];
    const PatRec<T> *rec = reinterpret_cast<const PatRec<T> *>(gs_smem);
    const uint32_t *st = reinterpret_cast<const uint32_t *>(rec + nrec);
    stage_patterns<T>(gs_smem, grec, pstart, npat, nrec);
    __syncthreads();
    for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int32_t r0 = rows[t];
        const uint32_t p = __ldg(pid + r0 / 3);
        const uint32_t kb = st[p], ke = st[p + 1];
        T s0 = b[r0], s1 = b[r0 + 1], s2 = b[r0 + 2];
        T a[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
#pragma unroll 4
        for (uint32_t k = kb; k < ke; ++k) {
            const PatRec<T> q = rec[k];
            if (q.off >= 0 && q.off < 3) {   // the node's own block, column q.off
                if (q.off == 0) { a[0][0] = q.v[0]; a[1][0] = q.v[1]; a[2][0] = q.v[2]; }
                else if (q.off == 1) { a[0][1] = q.v[0]; a[1][1] = q.v[1]; a[2][1] = q.v[2]; }
                else { a[0][2] = q.v[0]; a[1][2] = q.v[1]; a[2][2] = q.v[2]; }
                continue;
            }
            const T xv = __ldg(x + (r0 + q.off));
            s0 = fma(-q.v[0], xv, s0);
            s1 = fma(-q.v[1], xv, s1);
            s2 = fma(-q.v[2], xv, s2);
        }
        const T x1o = x[r0 + 1], x2o = x[r0 + 2];
        const T x0 = (s0 - a[0][1] * x1o - a[0][2] * x2o) / a[0][0];
        const T x1 = (s1 - a[1][0] * x0 - a[1][2] * x2o) / a[1][1];
        const T x2 = (s2 - a[2][0] * x0 - a[2][1] * x1) / a[2][2];
        x[r0] = x0;
        x[r0 + 1] = x1;
        x[r0 + 2] = x2;
    }
}

inline DuviArgs gs_duvi_args(const dv_matrix *m) {
    DuviArgs a;
    a.row_to_col = m->row_to_col.as<uint32_t>();
    a.row_to_dist = m->row_to_dist.as<uint32_t>();
    a.col_idx = m->col_idx.as<uint32_t>();
    a.dist = m->dist.as<uint8_t>();
    a.vidx = m->vidx.p;
    a.values = m->values.p;
    a.bundles = m->bundles.as<int32_t>();
    a.nbundles = m->nbundles;
    a.nuniq = (int32_t)m->nuniq;
    return a;
}

// Row groups of one Gauss-Seidel ordering (device rows + host group offsets).
struct GsOrder {
    DevMem rows;
    std::vector<int32_t> off;
    int bs = 1;
};

// Builds the ordering: lex = dependency levels of the forward sweep (rows);
// otherwise a greedy coloring of node blocks (3 or 2 consecutive rows when the size allows).
inline void gs_build_order(const dv_csr_host &a, bool lex, cudaStream_t s, GsOrder &o) {
    std::vector<int32_t> rows;
    if (lex) {
        dv_gs_level_sets(a, rows, o.off);
        o.bs = 1;
    } else {
        o.bs = (a.n_rows % 3 == 0) ? 3 : (a.n_rows % 2 == 0 ? 2 : 1);
        std::vector<int32_t> color;
        const int nc = dv_block_coloring(a, o.bs, color);
        o.off.assign(nc + 1, 0);
        rows.resize(color.size());
        for (int32_t c : color) o.off[c + 1]++;
        for (int c = 0; c < nc; ++c) o.off[c + 1] += o.off[c];
        std::vector<int32_t> fill(o.off.begin(), o.off.end() - 1);
        for (size_t b = 0; b < color.size(); ++b) rows[fill[color[b]]++] = (int32_t)b * o.bs;
    }
    o.rows.alloc(4 * rows.size());
    DV_CUDA(cudaMemcpyAsync(o.rows.p, rows.data(), 4 * rows.size(), cudaMemcpyHostToDevice, s));
    DV_CUDA(cudaStreamSynchronize(s));
}

// One forward sweep over all groups of the ordering (x updated in place).
template <class T>
void gs_sweep(const LaunchEnv &e, const dv_matrix *A, const GsOrder &o, const T *b, T *x) {
    dv_context *ctx = e.ctx;
    const int32_t ngroups = (int32_t)o.off.size() - 1;
    for (int32_t q = 0; q < ngroups; ++q) {
        const int32_t cnt = o.off[q + 1] - o.off[q];
        const int32_t *rows = o.rows.as<int32_t>() + o.off[q];
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cnt + kThreads - 1) / kThreads, ctx->num_sms * 8));
        if (o.bs == 3 && A->format == DV_FORMAT_DUVI && A->pat_ok && A->lanes_group == 3 && !A->pat_based &&
            sizeof(T) == (A->precision == DV_F64 ? 8 : 4)) {
            // node blocks of one color on the pattern layout
            const size_t smem = sizeof(PatRec<T>) * (size_t)A->pat_entries + 4 * ((size_t)A->pat_count + 1);
            static SmemLimit limit;   // per instantiation and device
            limit.raise(k_gs_pattern<T>, smem, ctx->device);
            k_gs_pattern<T><<<grid, kThreads, smem, e.stream>>>(A->pat_id.as<uint16_t>(), A->pat_start.as<uint32_t>(),
                                                               static_cast<const PatRec<T> *>(A->pat_rec.p),
                                                               A->pat_count, A->pat_entries, b, x, rows, cnt, e.done);
        } else if (A->format == DV_FORMAT_CSR) {
            k_gs_csr<T><<<grid, kThreads, 0, e.stream>>>(A->rowptr.as<int32_t>(), A->col.as<int32_t>(),
                                                         static_cast<const T *>(A->val.p), b, x, rows, cnt, o.bs, e.done);
        } else if (A->vi_bits == 8) {
            k_gs_duvi<uint8_t, T><<<grid, kThreads, 0, e.stream>>>(gs_duvi_args(A), b, x, rows, cnt, o.bs, e.done);
        } else if (A->vi_bits == 16) {
            k_gs_duvi<uint16_t, T><<<grid, kThreads, 0, e.stream>>>(gs_duvi_args(A), b, x, rows, cnt, o.bs, e.done);
        } else {
            k_gs_duvi<uint32_t, T><<<grid, kThreads, 0, e.stream>>>(gs_duvi_args(A), b, x, rows, cnt, o.bs, e.done);
        }
        DV_CUDA(cudaGetLastError());
        ctx->count();
    }
}

}  // namespace dvk
