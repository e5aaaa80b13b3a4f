// Block (multi-right-hand-side) products Y = A X with fused epilogues.
//
// X and Y are row-interleaved n x ld blocks: the ld values of a row are
// contiguous, so the k values one matrix entry multiplies are one coalesced
// read.  One warp per row group: the group's G rows (the dofs of one node,
// which share one column list) are walked once with warp-uniform loads and the
// lanes own right-hand-side columns j = lane + 32 u (u < U), so each gathered
// X(c, j) serves G rows and the matrix is decoded once per k vectors.  Every
// row sums its entries in storage order with the same multiply-add as the
// single-vector kernels, so an FP64 block product equals k single products
// (and the oracle's sequential walk) bit for bit.
//
// Epilogues that reduce per column (dot products of the flexible CG) keep
// per-lane partial sums and finish with a deterministic per-column grid
// reduction: per-block partials, then the last block sums them in block order.
#pragma once

#include "dv_kernels.cuh"

dvk::LaunchEnv dv_default_env(dv_context *ctx);

namespace dvb {

using dvk::LaunchEnv;
using dvk::madd;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCols = 128;   // columns of one launch (lanes x U)

// ---------------------------------------------------------------------------
// per-column deterministic grid reduction
// ---------------------------------------------------------------------------
// acc[u][c]: this lane's sums for column j = lane + 32 u.  Partials hold
// gridDim.x * kc * NC doubles.  The last block calls fin(j, totals) for each column.
template <int NC, int U, class Fin>
__device__ void col_reduce(double (&acc)[U][NC], int kc, double *partials, unsigned *ticket, Fin fin) {
    __shared__ double sh[kWarps][32 * U * NC];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) sh[warp][(lane + 32 * u) * NC + c] = acc[u][c];
    __syncthreads();
    const int nq = kc * NC;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kWarps; ++w) t += sh[w][q];
        partials[(size_t)blockIdx.x * nq + q] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // warp w sums quantities q = w, w + 8, ...: lanes stride over blocks, then a fixed butterfly
    for (int q = warp; q < nq; q += kWarps) {
        double t = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) t += __ldcg(partials + (size_t)b * nq + q);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) sh[0][q] = t;   // sh[0] is free: every warp finished reading it above
    }
    __syncthreads();
    for (int j = threadIdx.x; j < kc; j += blockDim.x) fin(j, &sh[0][j * NC]);
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0;
}

// ---------------------------------------------------------------------------
// gathers: X(c, j) of the product
// ---------------------------------------------------------------------------
template <class XT, class AT>
struct BGatherVec {
    const XT *__restrict__ x;
    int ld;
    __device__ __forceinline__ AT operator()(uint32_t c, int j) const { return (AT)__ldg(x + (size_t)c * ld + j); }
};
// w(c) B(c, j): the first Jacobi sweep from zero fused into the second
template <class T>
struct BGatherWB {
    const T *__restrict__ w;
    const T *__restrict__ b;
    int ld;
    __device__ __forceinline__ T operator()(uint32_t c, int j) const { return __ldg(w + c) * __ldg(b + (size_t)c * ld + j); }
};

// ---------------------------------------------------------------------------
// epilogues: apply(row, column, row sum, this lane's reduction slots)
// ---------------------------------------------------------------------------
struct NoFin {
    __device__ void operator()(int, const double *) const {}
};
template <class T>
struct BEpiSpmm {   // Y = A X, or Y += A X
    static constexpr int NC = 0;
    T *y;
    int ld, clear;
    NoFin fin;
    __device__ __forceinline__ void apply(int32_t i, int j, T s, double *) const {
        T *p = y + (size_t)i * ld + j;
        *p = clear ? s : *p + s;
    }
};
template <class T>
struct BEpiResid {   // R = B - A X
    static constexpr int NC = 0;
    const T *b;
    T *r;
    int ld;
    NoFin fin;
    __device__ __forceinline__ void apply(int32_t i, int j, T s, double *) const {
        const size_t q = (size_t)i * ld + j;
        r[q] = b[q] - s;
    }
};
template <class T>
struct BEpiJacobi {   // Y = X + w (B - A X)
    static constexpr int NC = 0;
    const T *x, *w, *b;
    T *y;
    int ld;
    NoFin fin;
    __device__ __forceinline__ void apply(int32_t i, int j, T s, double *) const {
        const size_t q = (size_t)i * ld + j;
        y[q] = x[q] + w[i] * (b[q] - s);
    }
};
template <class T>
struct BEpiJacobiFromZero {   // two sweeps from zero: Y = wB + w (B - A (wB))
    static constexpr int NC = 0;
    const T *w, *b;
    T *y;
    int ld;
    NoFin fin;
    __device__ __forceinline__ void apply(int32_t i, int j, T s, double *) const {
        const size_t q = (size_t)i * ld + j;
        const T wi = w[i], bi = b[q];
        y[q] = wi * bi + wi * (bi - s);
    }
};

// ---------------------------------------------------------------------------
// block product kernels
// ---------------------------------------------------------------------------
template <class AT, int G, int U, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                                        const AT *__restrict__ va, int32_t ngroups, int kc, Gather g,
                                                        Epi ep, const int *__restrict__ done, double *partials,
                                                        unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    constexpr int NC = Epi::NC > 0 ? Epi::NC : 1;
    double red[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[u][c] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; grp < ngroups; grp += nw) {
        const int32_t r0 = grp * G;
        int32_t s[G];
#pragma unroll
        for (int t = 0; t < G; ++t) s[t] = __ldg(rp + r0 + t);
        const int32_t len = __ldg(rp + r0 + 1) - s[0];
        AT acc[G][U];
#pragma unroll
        for (int t = 0; t < G; ++t)
#pragma unroll
            for (int u = 0; u < U; ++u) acc[t][u] = AT(0);
#pragma unroll 2
        for (int32_t e = 0; e < len; ++e) {
            const uint32_t c = (uint32_t)__ldg(ci + s[0] + e);
            AT a[G];
#pragma unroll
            for (int t = 0; t < G; ++t) a[t] = __ldg(va + s[t] + e);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = lane + 32 * u;
                if (j < kc) {
                    const AT x = g(c, j);
#pragma unroll
                    for (int t = 0; t < G; ++t) acc[t][u] = madd<AT>(acc[t][u], a[t], x);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < kc)
#pragma unroll
                for (int t = 0; t < G; ++t) ep.apply(r0 + t, j, acc[t][u], red[u]);
        }
    }
    if constexpr (Epi::NC > 0) col_reduce<Epi::NC, U>(red, kc, partials, ticket, ep.fin);
}

struct BDuviArgs {
    const uint32_t *__restrict__ row_to_col;
    const uint32_t *__restrict__ row_to_dist;
    const uint32_t *__restrict__ col_idx;
    const uint8_t *__restrict__ dist;
    const void *__restrict__ vidx;
    const void *__restrict__ values;
    int vi_bits;
};

__device__ __forceinline__ uint32_t load_vi(const void *v, int bits, uint32_t i) {
    if (bits == 8) return __ldg(static_cast<const uint8_t *>(v) + i);
    if (bits == 16) return __ldg(static_cast<const uint16_t *>(v) + i);
    return __ldg(static_cast<const uint32_t *>(v) + i);
}

// Walks the leader row's blocks (count byte at a block start, gap bytes
// inside: DuViGeometricMultigrid.cl:84-98); the G rows of a group have equal
// block structure, so their value indices sit at the same offsets of their
// own entry ranges.
template <class AT, int G, int U, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_duvi(BDuviArgs A, int32_t ngroups, int kc, Gather g, Epi ep,
                                                         const int *__restrict__ done, double *partials,
                                                         unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    constexpr int NC = Epi::NC > 0 ? Epi::NC : 1;
    double red[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[u][c] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    const AT *tab = static_cast<const AT *>(A.values);
    for (int32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; grp < ngroups; grp += nw) {
        const int32_t r0 = grp * G;
        const uint32_t b0 = __ldg(A.row_to_col + r0), b1 = __ldg(A.row_to_col + r0 + 1);
        uint32_t d[G];
#pragma unroll
        for (int t = 0; t < G; ++t) d[t] = __ldg(A.row_to_dist + r0 + t);
        AT acc[G][U];
#pragma unroll
        for (int t = 0; t < G; ++t)
#pragma unroll
            for (int u = 0; u < U; ++u) acc[t][u] = AT(0);
        uint32_t off = 0;   // entry offset inside the rows
        for (uint32_t bl = b0; bl < b1; ++bl) {
            uint32_t c = __ldg(A.col_idx + bl);
            const uint32_t cnt = __ldg(A.dist + d[0] + off);
            for (uint32_t q = 0;; ++q) {
                AT a[G];
#pragma unroll
                for (int t = 0; t < G; ++t) a[t] = __ldg(tab + load_vi(A.vidx, A.vi_bits, d[t] + off));
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = lane + 32 * u;
                    if (j < kc) {
                        const AT x = g(c, j);
#pragma unroll
                        for (int t = 0; t < G; ++t) acc[t][u] = madd<AT>(acc[t][u], a[t], x);
                    }
                }
                ++off;
                if (q == cnt) break;
                c += __ldg(A.dist + d[0] + off) + 1u;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < kc)
#pragma unroll
                for (int t = 0; t < G; ++t) ep.apply(r0 + t, j, acc[t][u], red[u]);
        }
    }
    if constexpr (Epi::NC > 0) col_reduce<Epi::NC, U>(red, kc, partials, ticket, ep.fin);
}

// Grid of a block product: one warp per group, at most max_blocks blocks
// (products that reduce use fewer blocks so the last block's sum stays short).
inline int bprod_blocks(const LaunchEnv &e, int64_t ngroups, bool reduces) {
    const int64_t want = (ngroups * 32 + kThreads - 1) / kThreads;
    const int64_t cap = reduces ? (int64_t)e.ctx->num_sms * 4 : (int64_t)e.max_blocks;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

template <class AT, int G, int U, class Gather, class Epi>
void launch_bprod_gu(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    const int32_t ngroups = m->n_rows / G;
    const int blocks = bprod_blocks(e, ngroups, Epi::NC > 0);
    if (m->format == DV_FORMAT_CSR) {
        k_bprod_csr<AT, G, U, Gather, Epi><<<blocks, kThreads, 0, e.stream>>>(
            m->rowptr.as<int32_t>(), m->col.as<int32_t>(), static_cast<const AT *>(m->val.p), ngroups, kc, g, ep,
            e.done, e.partials, e.ticket);
    } else {
        BDuviArgs a{m->row_to_col.as<uint32_t>(), m->row_to_dist.as<uint32_t>(), m->col_idx.as<uint32_t>(),
                    m->dist.as<uint8_t>(), m->vidx.p, m->values.p, m->vi_bits};
        k_bprod_duvi<AT, G, U, Gather, Epi><<<blocks, kThreads, 0, e.stream>>>(a, ngroups, kc, g, ep, e.done,
                                                                               e.partials, e.ticket);
    }
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

// Y-epilogue product over kc <= kMaxCols columns; the matrix's values have type AT.
template <class AT, class Gather, class Epi>
void launch_bprod(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    DV_REQUIRE(kc >= 1 && kc <= kMaxCols, DV_ERR_ARG, "block product of more than 128 columns");
    const bool g3 = m->row_group == 3;
    if (kc <= 32) {
        if (g3) launch_bprod_gu<AT, 3, 1>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 1>(e, m, kc, g, ep);
    } else if (kc <= 64) {
        if (g3) launch_bprod_gu<AT, 3, 2>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 2>(e, m, kc, g, ep);
    } else {
        if (g3) launch_bprod_gu<AT, 3, 4>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 4>(e, m, kc, g, ep);
    }
}

}  // namespace dvb
