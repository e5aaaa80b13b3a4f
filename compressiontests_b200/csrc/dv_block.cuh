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
                                                            unsigned *ticket, const uint32_t *__restrict__ list) {
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
    for (int32_t gi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gi < ngroups; gi += nw) {
        const int32_t grp = list ? (int32_t)__ldg(list + gi) : gi;   // list: the groups to run (ngroups of them)
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
void launch_bprod_pattern_u(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep,
                            const uint32_t *list = nullptr, int64_t nlist = 0) {
    constexpr int G = 3;
    auto kern = k_bprod_pattern<AT, G, U, EXACT, BASED, SHIFT, Gather, Epi>;
    const size_t smem = sizeof(dvk::PatRec<AT>) * (size_t)m->pat_entries + 4 * ((size_t)m->pat_count + 1);
    static dvk::SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
    const int32_t ngroups = list ? (int32_t)nlist : m->n_rows / G;
    const int blocks = bprod_blocks(e, ngroups, Epi::NC > 0);
    kern<<<blocks, kThreads, smem, e.stream>>>(m->pat_id.as<uint16_t>(), m->pat_start.as<uint32_t>(),
                                               static_cast<const dvk::PatRec<AT> *>(m->pat_rec.p),
                                               m->pat_base.as<uint32_t>(), m->pat_count, m->pat_entries, ngroups, kc,
                                               g, ep, e.done, e.partials, e.ticket, list);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

template <int U, class Gather, class Epi>
void launch_bprod_boundary(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    launch_bprod_pattern_u<float, U, true, false, false>(e, m, kc, g, ep, m->grid_bnode.as<uint32_t>(), m->grid_nb);
}

template <class AT, bool EXACT, bool BASED, bool SHIFT, class Gather, class Epi>
void launch_bprod_pattern(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    if (kc <= 32) launch_bprod_pattern_u<AT, 1, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
    else if (kc <= 64) launch_bprod_pattern_u<AT, 2, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
    else launch_bprod_pattern_u<AT, 4, EXACT, BASED, SHIFT>(e, m, kc, g, ep);
}

// ---------------------------------------------------------------------------
// Block products on the grid-stencil layout (FP32 hex operators, epilogues without column
// reductions).  A block owns a tile of 8 x 4 interior nodes of a plane, streams a run of z planes
// and covers 32 right-hand sides (lane = column).  Each plane of the tile with its one-node halo
// (10 x 6 nodes, 3 dofs, 32 columns: 180 rows of 128 bytes) is copied into a ring of shared-memory
// slots with 16-byte cp.async copies, two planes ahead; warp w takes the 4 nodes x = 4 (w % 2) .. +3
// of tile row w / 2 and applies every staged value of the plane to the nodes it couples in z - 1,
// z and z + 1 (the streaming accumulators of k_duvi_grid) with the hex stencil's class values.
// Each row sums its terms in column order with one FMA each, as the pattern kernel does (the
// stencil's structural zeros skipped: they add exact zeros).  Face groups and interior groups of
// other patterns run on the pattern kernel over the boundary list.
// ---------------------------------------------------------------------------
// DV_BGRID=0 keeps the pattern kernel for block products on grid layouts (A/B comparisons).
inline bool bgrid_enabled() {
    const char *v = getenv("DV_BGRID");
    return !(v && v[0] == '0');
}
constexpr int kBgTX = 8, kBgTY = 4;                      // interior nodes of a tile
constexpr int kBgHX = kBgTX + 2, kBgHY = kBgTY + 2;      // with the halo
constexpr int kBgRows = kBgHX * kBgHY * 3;               // staged rows of a plane (node dofs)
constexpr int kBgStages = 3;
constexpr int kBgSlot = kBgRows * 32 + kBgRows;          // floats of a slot: the rows, then w (Jacobi from zero)

struct BGridGeom {
    int32_t lx, ly, lz, ntx, nty, zc, ntile, hot, all_hot;
};

template <class Gather>
struct BGridSrc;   // the block array a gather stages, and its per-row weight (w .* B)
template <class T>
struct BGridSrc<BGatherVec<T, T>> {
    static constexpr bool WB = false;
    static const T *block(const BGatherVec<T, T> &g) { return g.x; }
    __device__ static const T *weights(const BGatherVec<T, T> &) { return nullptr; }
};
template <class T>
struct BGridSrc<BGatherWB<T>> {
    static constexpr bool WB = true;
    static const T *block(const BGatherWB<T> &g) { return g.b; }
    __device__ static const T *weights(const BGatherWB<T> &g) { return g.w; }
};

template <class Gather>
__device__ __forceinline__ void bgrid_issue(const Gather &g, const float *__restrict__ X, int ld, float *slot, int x0,
                                            int y0, int z, const BGridGeom &G, int j0, int kc) {
    const bool zin = z >= 0 && z < G.lz;
    for (int c = threadIdx.x; c < kBgRows * 8; c += kThreads) {
        const int row = c >> 3, sub = c & 7, hn = row / 3, comp = row - 3 * hn;
        const int gx = x0 - 1 + hn % kBgHX, gy = y0 - 1 + hn / kBgHX;
        const bool v = zin && gx >= 0 && gx < G.lx && gy >= 0 && gy < G.ly && j0 + 4 * sub < kc;
        const int64_t grow = 3 * ((int64_t)gx + (int64_t)G.lx * (gy + (int64_t)G.ly * z)) + comp;
        dvk::cp_async_zfill<16>(slot + row * 32 + 4 * sub, v ? X + grow * ld + j0 + 4 * sub : X, v);
    }
    if constexpr (BGridSrc<Gather>::WB) {
        const float *w = BGridSrc<Gather>::weights(g);
        for (int row = threadIdx.x; row < kBgRows; row += kThreads) {
            const int hn = row / 3, comp = row - 3 * hn;
            const int gx = x0 - 1 + hn % kBgHX, gy = y0 - 1 + hn / kBgHX;
            const bool v = zin && gx >= 0 && gx < G.lx && gy >= 0 && gy < G.ly;
            const int64_t grow = 3 * ((int64_t)gx + (int64_t)G.lx * (gy + (int64_t)G.ly * z)) + comp;
            dvk::cp_async_zfill<4>(slot + kBgRows * 32 + row, v ? w + grow : w, v);
        }
    }
    dvk::cp_async_commit();
}

template <class Gather, class Epi>
__global__ void __launch_bounds__(kThreads, 3) k_bprod_grid(BGridGeom G, dvk::GridCoef<float> cf,
                                                             const uint16_t *__restrict__ pid, const float *__restrict__ X,
                                                             int ld, int kc, Gather g, Epi ep,
                                                             const int *__restrict__ done) {
    static_assert(Epi::NC == 0, "column reductions run on the pattern kernel");
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 bgrid_smem[];
    float *ring = reinterpret_cast<float *>(bgrid_smem);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int yw = warp >> 1, xs = (warp & 1) * 4;   // the warp's 4 nodes: tile x xs .. xs+3, tile row yw
    const int j0 = blockIdx.y * 32;
    const int64_t lxy = (int64_t)G.lx * G.ly;
    double nored[1];
    for (int t = blockIdx.x; t < G.ntile; t += gridDim.x) {
        const int txi = t % G.ntx, tyi = (t / G.ntx) % G.nty, tzi = t / (G.ntx * G.nty);
        const int x0 = 1 + txi * kBgTX, y0 = 1 + tyi * kBgTY, z0 = 1 + tzi * G.zc, z1 = min(G.lz - 1, z0 + G.zc);
        const int gy = y0 + yw;
        bool inxy[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) inxy[i] = x0 + xs + i <= G.lx - 2 && gy <= G.ly - 2;
        auto active = [&](int i, int z) {
            if (!inxy[i] || z < 1 || z > G.lz - 2) return false;
            return G.all_hot || (int)__ldg(pid + (x0 + xs + i) + (int64_t)G.lx * gy + lxy * z) == G.hot;
        };
        bgrid_issue(g, X, ld, ring, x0, y0, z0 - 1, G, j0, kc);
        if (z0 <= z1) bgrid_issue(g, X, ld, ring + kBgSlot, x0, y0, z0, G, j0, kc);
        else dvk::cp_async_commit();
        float a0[4][3], a1[4][3], a2[4][3];
        bool act0[4], act1[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            act0[i] = act1[i] = false;
#pragma unroll
            for (int d = 0; d < 3; ++d) a0[i][d] = a1[i][d] = a2[i][d] = 0.f;
        }
        for (int p = z0 - 1, k = 0; p <= z1; ++p, ++k) {
            dvk::cp_async_wait<kBgStages - 2>();
            __syncthreads();
            if (p + 2 <= z1) bgrid_issue(g, X, ld, ring + ((k + 2) % kBgStages) * kBgSlot, x0, y0, p + 2, G, j0, kc);
            else dvk::cp_async_commit();
            const float *pl = ring + (k % kBgStages) * kBgSlot;
            const bool di = p + 1 >= z0 && p + 1 < z1, dm = p >= z0 && p < z1, df = p - 1 >= z0 && p - 1 < z1;
            bool act2[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                act2[i] = di && active(i, p + 1);
#pragma unroll
                for (int d = 0; d < 3; ++d) a2[i][d] = 0.f;
            }
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int hx = 0; hx < 6; ++hx)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int row = ((yw + dy) * kBgHX + xs + hx) * 3 + c;
                        float v = pl[row * 32 + lane];
                        if constexpr (BGridSrc<Gather>::WB) v = pl[kBgRows * 32 + row] * v;
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int dx = hx - i;   // neighbour offset + 1
                            if (dx < 0 || dx > 2) continue;
                            const int e = 9 * dy + 3 * dx + c;
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                const int ci = dvk::hex_class(3 * e + d), cm = dvk::hex_class(3 * (27 + e) + d),
                                          cz = dvk::hex_class(3 * (54 + e) + d);
                                if (ci >= 0 && di) a2[i][d] = fmaf(cf.cls[ci], v, a2[i][d]);
                                if (cm >= 0 && dm) a1[i][d] = fmaf(cf.cls[cm], v, a1[i][d]);
                                if (cz >= 0 && df) a0[i][d] = fmaf(cf.cls[cz], v, a0[i][d]);
                            }
                        }
                    }
            if (df && lane < kc - j0) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (act0[i]) {
                        const int32_t r = (int32_t)(3 * ((x0 + xs + i) + G.lx * (int64_t)gy + lxy * (p - 1)));
#pragma unroll
                        for (int d = 0; d < 3; ++d) ep.apply(r + d, j0 + lane, a0[i][d], nored);
                    }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    a0[i][d] = a1[i][d];
                    a1[i][d] = a2[i][d];
                }
                act0[i] = act1[i];
                act1[i] = act2[i];
            }
        }
        dvk::cp_async_wait<0>();
        __syncthreads();
    }
}

template <class Gather>
struct bgrid_gather : std::false_type {};
template <>
struct bgrid_gather<BGatherVec<float, float>> : std::true_type {};
template <>
struct bgrid_gather<BGatherWB<float>> : std::true_type {};

// The grid-stencil block product and the boundary groups' pattern walk (two launches, disjoint rows).
template <class Gather, class Epi>
void launch_bprod_grid(const LaunchEnv &e, const dv_matrix *m, int kc, Gather g, Epi ep) {
    BGridGeom G;
    G.lx = m->grid_lx;
    G.ly = m->grid_ly;
    G.lz = m->grid_lz;
    G.ntx = std::max(0, (G.lx - 2 + kBgTX - 1) / kBgTX);   // tiles over the interior nodes 1 .. l-2
    G.nty = std::max(0, (G.ly - 2 + kBgTY - 1) / kBgTY);
    G.zc = 8;
    const int lzi = std::max(1, G.lz - 2);
    G.ntile = G.lz > 2 ? G.ntx * G.nty * ((lzi + G.zc - 1) / G.zc) : 0;
    G.hot = m->grid_hot;
    G.all_hot = m->grid_all_hot;
    dvk::GridCoef<float> cf;
    for (int k = 0; k < 81; ++k)
        for (int d = 0; d < 3; ++d) cf.v[k][d] = (float)m->grid_coef[3 * k + d];
    for (int c = 0; c < dvk::kHexClasses; ++c) cf.cls[c] = (float)m->grid_cls[c];
    if (G.ntile > 0) {
        auto kern = k_bprod_grid<Gather, Epi>;
        const size_t smem = sizeof(float) * (size_t)kBgStages * kBgSlot;
        static dvk::SmemLimit limit;   // per instantiation and device
        limit.raise(kern, smem, e.ctx->device);
        const dim3 grid((unsigned)G.ntile, (unsigned)((kc + 31) / 32));
        kern<<<grid, kThreads, smem, e.stream>>>(G, cf, m->pat_id.as<uint16_t>(), BGridSrc<Gather>::block(g), g.ld, kc,
                                                 g, ep, e.done);
        DV_CUDA(cudaGetLastError());
        e.ctx->count();
    }
    if (m->grid_nb > 0) {
        if (kc <= 32) launch_bprod_boundary<1>(e, m, kc, g, ep);
        else if (kc <= 64) launch_bprod_boundary<2>(e, m, kc, g, ep);
        else launch_bprod_boundary<4>(e, m, kc, g, ep);
    }
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
        const uint32_t q = (uint32_t)(t / kc);
        const int j = (int)(t - (int64_t)q * kc);
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
    if constexpr (Epi::NC == 0 && std::is_same<AT, float>::value && bgrid_gather<Gather>::value) {
        // FP32 hex operators on the grid-stencil layout; 16-byte copies need an aligned block and ld
        const void *xb = BGridSrc<Gather>::block(g);
        if (m->format == DV_FORMAT_DUVI && m->duvi_variant == 3 && m->grid_hex && m->precision == DV_F32 &&
            (reinterpret_cast<uintptr_t>(xb) & 15) == 0 && g.ld % 4 == 0 && bgrid_enabled()) {
            launch_bprod_grid(e, m, kc, g, ep);
            return;
        }
    }
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
