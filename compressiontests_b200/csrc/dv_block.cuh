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
constexpr int kReduceBlocksPerSm = 8;   // grid cap of products and vector kernels that reduce per column

// ---------------------------------------------------------------------------
// per-column deterministic grid reduction
// ---------------------------------------------------------------------------
// acc[u][c]: this lane's sums for column j = lane + 32 u.  Partials hold
// gridDim.x * kc * NC doubles.  The last block calls fin(j, totals) for each column.
template <int NC, int U, class Fin>
__device__ __forceinline__ void col_reduce(double (&acc)[U][NC], int kc, double *partials, unsigned *ticket, Fin fin) {
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
//
// A warp walks its group's entries in chunks of 32: the lanes decode one
// entry each (coalesced loads of columns, gaps and value indices; for DuVi a
// segmented warp scan turns block starts and gaps into columns) into a
// shared-memory record {column, G values}, then every lane runs over the
// chunk's records (one broadcast shared load per entry) and gathers its
// columns of X.  Per entry the warp issues one shared load and U gathers.
// ---------------------------------------------------------------------------
template <class AT, int G>
struct alignas(16) Rec {
    uint32_t c;
    AT a[G];
};

// EXACT: product rounded, then added (the oracle's order, bit-exact for FP64);
// otherwise one fused multiply-add per term.
template <class AT, int G, int U, bool EXACT, class Gather>
__device__ __forceinline__ void chunk_fma(const Rec<AT, G> *rec, int n, int kc, int lane, const Gather &g,
                                          AT (&acc)[G][U]) {
#pragma unroll 4
    for (int e = 0; e < n; ++e) {
        const Rec<AT, G> r = rec[e];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < kc) {
                const AT x = g(r.c, j);
#pragma unroll
                for (int t = 0; t < G; ++t) acc[t][u] = EXACT ? madd<AT>(acc[t][u], r.a[t], x) : fma(r.a[t], x, acc[t][u]);
            }
        }
    }
}

template <class AT, int G, int U, class Epi>
__device__ __forceinline__ void group_epilogue(int32_t r0, int kc, int lane, const Epi &ep, AT (&acc)[G][U],
                                               double (&red)[U][Epi::NC > 0 ? Epi::NC : 1]) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int j = lane + 32 * u;
        if (j < kc)
#pragma unroll
            for (int t = 0; t < G; ++t) ep.apply(r0 + t, j, acc[t][u], red[u]);
    }
}

template <class AT, int G, int U, bool EXACT, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                                        const AT *__restrict__ va, int32_t ngroups, int kc, Gather g,
                                                        Epi ep, const int *__restrict__ done, double *partials,
                                                        unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    __shared__ Rec<AT, G> srec[kWarps][32];
    constexpr int NC = Epi::NC > 0 ? Epi::NC : 1;
    double red[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[u][c] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Rec<AT, G> *rec = srec[warp];
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
        for (int32_t off = 0; off < len; off += 32) {
            const int n = min(32, len - off);
            if (lane < n) {
                Rec<AT, G> r;
                r.c = (uint32_t)__ldg(ci + s[0] + off + lane);
#pragma unroll
                for (int t = 0; t < G; ++t) r.a[t] = __ldg(va + s[t] + off + lane);
                rec[lane] = r;
            }
            __syncwarp();
            chunk_fma<AT, G, U, EXACT>(rec, n, kc, lane, g, acc);
            __syncwarp();
        }
        group_epilogue<AT, G, U>(r0, kc, lane, ep, acc, red);
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
    int nuniq;
};

__device__ __forceinline__ uint32_t load_vi(const void *v, int bits, uint32_t i) {
    if (bits == 8) return __ldg(static_cast<const uint8_t *>(v) + i);
    if (bits == 16) return __ldg(static_cast<const uint16_t *>(v) + i);
    return __ldg(static_cast<const uint32_t *>(v) + i);
}

// DuVi rows (DuViGeometricMultigrid.cl:84-98): a row is a run of blocks; the
// first entry byte of a block holds the count of its following entries, the
// others hold gap - 1; block start columns are in col_idx.  The G rows of a
// group share their block structure, so their value indices sit at the same
// offsets of their own entry ranges.  Chunk decode: block starts inside the
// chunk are found by hopping count bytes (one shuffle per block), then a
// segmented inclusive scan over the lanes gives every entry its column.
template <class AT, int G, int U, bool EXACT, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_duvi(BDuviArgs A, int32_t ngroups, int kc, Gather g, Epi ep,
                                                         const int *__restrict__ done, double *partials,
                                                         unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    __shared__ Rec<AT, G> srec[kWarps][32];
    __shared__ AT stab[256];
    constexpr int NC = Epi::NC > 0 ? Epi::NC : 1;
    const AT *gtab = static_cast<const AT *>(A.values);
    const bool smem_tab = A.vi_bits == 8;
    if (smem_tab) {
        for (int i = threadIdx.x; i < A.nuniq; i += blockDim.x) stab[i] = gtab[i];
        __syncthreads();
    }
    double red[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[u][c] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    Rec<AT, G> *rec = srec[warp];
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; grp < ngroups; grp += nw) {
        const int32_t r0 = grp * G;
        uint32_t d[G];
#pragma unroll
        for (int t = 0; t < G; ++t) d[t] = __ldg(A.row_to_dist + r0 + t);
        const uint32_t len = __ldg(A.row_to_dist + r0 + 1) - d[0];
        uint32_t bl = __ldg(A.row_to_col + r0);   // next block to start
        uint32_t rem = 0;                           // entries of the open block not yet decoded
        uint32_t ccur = 0;                          // column of the last decoded entry
        AT acc[G][U];
#pragma unroll
        for (int t = 0; t < G; ++t)
#pragma unroll
            for (int u = 0; u < U; ++u) acc[t][u] = AT(0);
        for (uint32_t off = 0; off < len; off += 32) {
            const int n = (int)min(32u, len - off);
            const bool act = lane < n;
            const uint32_t db = act ? (uint32_t)__ldg(A.dist + d[0] + off + lane) : 0u;
            // block starts of this chunk
            unsigned mask = 0;
            uint32_t p = rem;
            while (p < (uint32_t)n) {
                mask |= 1u << p;
                p += __shfl_sync(0xffffffffu, db, (int)p) + 1u;
            }
            rem = p - (uint32_t)n;
            const bool start = (mask >> lane) & 1u;
            const int nstart_le = __popc(mask & (below | (1u << lane)));   // starts at or before this lane
            // segmented scan: heads are block starts (their col_idx) and lane 0 (continuing the open block)
            uint32_t v;
            bool head;
            if (start) {
                v = __ldg(A.col_idx + bl + nstart_le - 1);
                head = true;
            } else {
                v = db + 1u + (lane == 0 ? ccur : 0u);
                head = lane == 0;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
                const bool hy = __shfl_up_sync(0xffffffffu, head, o);
                if (lane >= o && !head) {
                    v += y;
                    head = hy;
                }
            }
            bl += __popc(mask);
            ccur = __shfl_sync(0xffffffffu, v, n - 1);
            if (act) {
                Rec<AT, G> r;
                r.c = v;
#pragma unroll
                for (int t = 0; t < G; ++t) {
                    const uint32_t idx = load_vi(A.vidx, A.vi_bits, d[t] + off + lane);
                    r.a[t] = smem_tab ? stab[idx] : __ldg(gtab + idx);
                }
                rec[lane] = r;
            }
            __syncwarp();
            chunk_fma<AT, G, U, EXACT>(rec, n, kc, lane, g, acc);
            __syncwarp();
        }
        group_epilogue<AT, G, U>(r0, kc, lane, ep, acc, red);
    }
    if constexpr (Epi::NC > 0) col_reduce<Epi::NC, U>(red, kc, partials, ticket, ep.fin);
}

// Grid of a block product: one warp per group, at most max_blocks blocks
// (products that reduce use fewer blocks so the last block's sum stays short).
inline int bprod_blocks(const LaunchEnv &e, int64_t ngroups, bool reduces) {
    const int64_t want = (ngroups * 32 + kThreads - 1) / kThreads;
    const int64_t cap = reduces ? (int64_t)e.ctx->num_sms * kReduceBlocksPerSm : (int64_t)e.max_blocks;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

template <class AT, int G, int U, bool EXACT, class Gather, class Epi>
void launch_bprod_gu(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    const int32_t ngroups = m->n_rows / G;
    const int blocks = bprod_blocks(e, ngroups, Epi::NC > 0);
    if (m->format == DV_FORMAT_CSR) {
        k_bprod_csr<AT, G, U, EXACT, Gather, Epi><<<blocks, kThreads, 0, e.stream>>>(
            m->rowptr.as<int32_t>(), m->col.as<int32_t>(), static_cast<const AT *>(m->val.p), ngroups, kc, g, ep,
            e.done, e.partials, e.ticket);
    } else {
        BDuviArgs a{m->row_to_col.as<uint32_t>(), m->row_to_dist.as<uint32_t>(), m->col_idx.as<uint32_t>(),
                    m->dist.as<uint8_t>(), m->vidx.p, m->values.p, m->vi_bits, (int)m->nuniq};
        k_bprod_duvi<AT, G, U, EXACT, Gather, Epi><<<blocks, kThreads, 0, e.stream>>>(a, ngroups, kc, g, ep, e.done,
                                                                                      e.partials, e.ticket);
    }
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

// Y-epilogue product over kc <= kMaxCols columns; the matrix's values have type AT.
// Block product on the node-pattern layout (dvk::PatRec records staged in shared
// memory): one warp per node group, every record one broadcast shared load, lanes
// gather their right-hand-side columns.  No decode at all.  BASED: offsets from the
// group's first column (base[]); SHIFT: row d reads column + d.
template <class AT, int G, int U, bool EXACT, bool BASED, bool SHIFT, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_pattern(const uint16_t *__restrict__ pid,
                                                            const uint32_t *__restrict__ pstart,
                                                            const dvk::PatRec<AT> *__restrict__ grec,
                                                            const uint32_t *__restrict__ base, int32_t npat,
                                                            int32_t nrec, int32_t ngroups, int kc, Gather g, Epi ep,
                                                            const int *__restrict__ done, double *partials,
                                                            unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 bpat_smem[];
    dvk::PatRec<AT> *rec = reinterpret_cast<dvk::PatRec<AT> *>(bpat_smem);
    uint32_t *st = reinterpret_cast<uint32_t *>(rec + nrec);
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(grec);
        const int n16 = nrec * (int)(sizeof(dvk::PatRec<AT>) / 16);
        for (int i = threadIdx.x; i < n16; i += blockDim.x) bpat_smem[i] = __ldg(src + i);
        for (int i = threadIdx.x; i <= npat; i += blockDim.x) st[i] = __ldg(pstart + i);
    }
    __syncthreads();
    constexpr int NC = Epi::NC > 0 ? Epi::NC : 1;
    double red[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[u][c] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; grp < ngroups; grp += nw) {
        const uint32_t p = __ldg(pid + grp);
        const uint32_t b = st[p], e = st[p + 1];
        const int32_t r0 = grp * G;
        const uint32_t c0 = BASED ? __ldg(base + grp) : (uint32_t)r0;
        AT acc[G][U];
#pragma unroll
        for (int t = 0; t < G; ++t)
#pragma unroll
            for (int u = 0; u < U; ++u) acc[t][u] = AT(0);
#pragma unroll 2
        for (uint32_t k = b; k < e; ++k) {
            const dvk::PatRec<AT> q = rec[k];
            const uint32_t c = c0 + (uint32_t)q.off;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = lane + 32 * u;
                if (j < kc) {
                    if constexpr (SHIFT) {
#pragma unroll
                        for (int t = 0; t < G; ++t) {
                            const AT x = g(c + (uint32_t)t, j);
                            acc[t][u] = EXACT ? madd<AT>(acc[t][u], q.v[t], x) : fma(q.v[t], x, acc[t][u]);
                        }
                    } else {
                        const AT x = g(c, j);
#pragma unroll
                        for (int t = 0; t < G; ++t)
                            acc[t][u] = EXACT ? madd<AT>(acc[t][u], q.v[t], x) : fma(q.v[t], x, acc[t][u]);
                    }
                }
            }
        }
        group_epilogue<AT, G, U>(r0, kc, lane, ep, acc, red);
    }
    if constexpr (Epi::NC > 0) col_reduce<Epi::NC, U>(red, kc, partials, ticket, ep.fin);
}

template <class AT, int U, bool EXACT, bool BASED, bool SHIFT, class Gather, class Epi>
void launch_bprod_pattern_u(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    constexpr int G = 3;
    auto kern = k_bprod_pattern<AT, G, U, EXACT, BASED, SHIFT, Gather, Epi>;
    const size_t smem = sizeof(dvk::PatRec<AT>) * (size_t)m->pat_entries + 4 * ((size_t)m->pat_count + 1);
    static dvk::SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
    const int32_t ngroups = m->n_rows / G;
    const int blocks = bprod_blocks(e, ngroups, Epi::NC > 0);
    kern<<<blocks, kThreads, smem, e.stream>>>(m->pat_id.as<uint16_t>(), m->pat_start.as<uint32_t>(),
                                               static_cast<const dvk::PatRec<AT> *>(m->pat_rec.p),
                                               m->pat_base.as<uint32_t>(), m->pat_count, m->pat_entries, ngroups, kc,
                                               g, ep, e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

template <class AT, bool EXACT, bool BASED, bool SHIFT, class Gather, class Epi>
void launch_bprod_pattern(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    if (kc <= 32) launch_bprod_pattern_u<AT, 1, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
    else if (kc <= 64) launch_bprod_pattern_u<AT, 2, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
    else launch_bprod_pattern_u<AT, 4, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
}

// Matrix-free trilinear transfer (DV_FORMAT_TRILINEAR): one thread per (node, column j), the
// node's three rows summed from zero in column order like the stored kernels.
template <bool RESTRICT, class AT, class Gather, class Epi>
__global__ void __launch_bounds__(kThreads) k_bprod_tri(dvk::TriGeom G, int kc, Gather g, Epi ep,
                                                         const int *__restrict__ done) {
    static_assert(Epi::NC == 0, "transfers carry no reductions");
    if (done && *(volatile const int *)done) return;
    const int64_t work = G.nodes(RESTRICT) * kc;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < work; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t / kc;
        const int j = (int)(t - q * kc);
        AT s[3] = {AT(0), AT(0), AT(0)};
        dvk::tri_walk<RESTRICT, AT>(G, q, [&](uint32_t col, AT w) {
#pragma unroll
            for (int d = 0; d < 3; ++d) s[d] = madd<AT>(s[d], w, g(col + d, j));
        });
#pragma unroll
        for (int d = 0; d < 3; ++d) ep.apply((int32_t)(3 * q + d), j, s[d], nullptr);
    }
}

template <class AT, bool EXACT = true, class Gather, class Epi>
void launch_bprod(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    DV_REQUIRE(kc >= 1 && kc <= kMaxCols, DV_ERR_ARG, "block product of more than 128 columns");
    DV_REQUIRE(m->format != DV_FORMAT_HEX, DV_ERR_UNSUPPORTED, "block products need an assembled matrix");
    if constexpr (Epi::NC == 0) {
        if (m->format == DV_FORMAT_TRILINEAR) {
            const dvk::TriGeom G{m->tri_ne[0], m->tri_ne[1], m->tri_ne[2]};
            const int64_t work = G.nodes(m->tri_restrict) * kc;
            const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((work + kThreads - 1) / kThreads, e.max_blocks));
            if (m->tri_restrict) k_bprod_tri<true, AT><<<blocks, kThreads, 0, e.stream>>>(G, kc, g, ep, e.done);
            else k_bprod_tri<false, AT><<<blocks, kThreads, 0, e.stream>>>(G, kc, g, ep, e.done);
            DV_CUDA(cudaGetLastError());
            e.ctx->count();
            return;
        }
    }
    DV_REQUIRE(m->format == DV_FORMAT_CSR || m->format == DV_FORMAT_DUVI, DV_ERR_UNSUPPORTED,
               "block products need an assembled matrix");
    if (m->format == DV_FORMAT_DUVI && m->pat_ok && m->lanes_group == 3) {   // node patterns, 3-row groups
        if (!m->pat_based && !m->pat_shift) {
            launch_bprod_pattern<AT, EXACT, false, false>(e, m, kc, g, ep);
            return;
        }
        if (m->pat_based && m->pat_shift) {
            launch_bprod_pattern<AT, EXACT, true, true>(e, m, kc, g, ep);
            return;
        }
    }
    const bool g3 = m->row_group == 3;
    if (kc <= 32) {
        if (g3) launch_bprod_gu<AT, 3, 1, EXACT>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 1, EXACT>(e, m, kc, g, ep);
    } else if (kc <= 64) {
        if (g3) launch_bprod_gu<AT, 3, 2, EXACT>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 2, EXACT>(e, m, kc, g, ep);
    } else {
        if (g3) launch_bprod_gu<AT, 3, 4, EXACT>(e, m, kc, g, ep);
        else launch_bprod_gu<AT, 1, 4, EXACT>(e, m, kc, g, ep);
    }
}

}  // namespace dvb
