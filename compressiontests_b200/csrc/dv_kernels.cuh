// Device kernels of libduvigpu.so for sm_100a.
//
// The sparse path is HBM-bound integer/byte decode plus FMAs (about 0.1 flop
// per byte), so there are no tensor-core tiles here: the kernels are built
// around coalesced 16-byte staging of the index/byte streams into shared
// memory, L2-resident gathers of the vector, warp-shuffle reductions and
// epilogues that fuse the vector updates of each algorithm step into the
// pass over the matrix.
#pragma once

#include <cstddef>
#include <mutex>
#include <type_traits>
#include <utility>

#include "dv_internal.cuh"

#include <cuda_runtime.h>

namespace dvk {

constexpr int kThreads = 256;            // CSR and vector kernels
constexpr int kDuviWarps = 8;            // warps per block, staged DuVi kernel (8/16-bit indices)
constexpr int kDuviWarps32 = 4;          // 32-bit value indices (larger stage)
constexpr int kStageD = 3072;            // per-warp stage of entry bytes (>= kBundleBytes + 32)
constexpr int kStageC = 512;             // per-warp stage of block column starts (>= kBundleBlocks + 8)
constexpr int kMaxRed = 4;               // doubles per block in a grid reduction

static_assert(kStageD >= kBundleBytes + 32, "stage too small");
static_assert(kStageC >= kBundleBlocks + 8, "column stage too small");

// The dynamic shared memory a kernel may use is an attribute of each device: a
// launcher raises it to every new largest size on each device it launches on.
// Host threads may launch on several contexts at once: the caches of launch settings
// below are updated under one lock, so a raise never lowers a limit another thread set.
inline std::mutex &launch_cache_mutex() {
    static std::mutex m;
    return m;
}

constexpr int kMaxDevices = 64;
struct SmemLimit {
    size_t set[kMaxDevices] = {};
    template <class K>
    void raise(K kern, size_t smem, int device) {
        DV_REQUIRE(device >= 0 && device < kMaxDevices, DV_ERR_ARG, "device ordinal out of range");
        std::lock_guard<std::mutex> lock(launch_cache_mutex());
        if (smem > set[device]) {
            DV_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            set[device] = smem;
        }
    }
};

// Resident blocks per SM of a kernel at a dynamic shared-memory size on a device (occupancy
// query, remembered for the last few (device, size) pairs; the current device is `device`).
struct OccupancyCache {
    size_t smem[8] = {};
    int dev[8] = {};
    int blocks[8] = {};
    int next = 0;
    template <class K>
    int get(K kern, int threads, size_t smem_bytes, int device) {
        std::lock_guard<std::mutex> lock(launch_cache_mutex());
        for (int i = 0; i < 8; ++i)
            if (blocks[i] > 0 && smem[i] == smem_bytes && dev[i] == device) return blocks[i];
        int occ = 0;
        DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem_bytes));
        occ = std::max(occ, 1);
        smem[next] = smem_bytes;
        dev[next] = device;
        blocks[next] = occ;
        next = (next + 1) % 8;
        return occ;
    }
};

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Sum over aligned groups of W lanes (all lanes of a group must be converged).
template <int W, class T>
__device__ __forceinline__ T group_sum(T v) {
    if constexpr (W == 1) {
        return v;
    } else {
        const unsigned lane = threadIdx.x & 31u;
        const unsigned mask = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(unsigned)(W - 1)));
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
}

// Block reduction of N doubles: bit i of MAXMASK selects max instead of sum.
// Result valid in thread 0.  All threads of the block must call it.
template <int N, unsigned MAXMASK>
__device__ void block_reduce(double (&v)[N]) {
    __shared__ double sh[kMaxRed][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double t = ((MAXMASK >> i) & 1u) ? warp_max(v[i]) : warp_sum(v[i]);
        if (lane == 0) sh[i][warp] = t;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = lane < nw ? sh[i][lane] : 0.0;
            v[i] = ((MAXMASK >> i) & 1u) ? warp_max(t) : warp_sum(t);
        }
    }
    __syncthreads();
}

// Deterministic grid reduction: per-block partials, then the last block to
// arrive sums them in block order.  Returns true in thread 0 of the last block,
// with the totals in out.  Resets the ticket for the next launch.
template <int N, unsigned MAXMASK>
__device__ bool grid_reduce(double (&v)[N], double *partials, unsigned *ticket, double (&out)[N]) {
    block_reduce<N, MAXMASK>(v);
    __shared__ int is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) partials[(size_t)blockIdx.x * N + i] = v[i];
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc[N];
#pragma unroll
    for (int i = 0; i < N; ++i) acc[i] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double p = __ldcg(partials + (size_t)b * N + i);
            acc[i] = ((MAXMASK >> i) & 1u) ? fmax(acc[i], p) : acc[i] + p;
        }
    block_reduce<N, MAXMASK>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) out[i] = acc[i];
        *ticket = 0;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// gathers: value of the vector at a column (the x of y = A x)
// ---------------------------------------------------------------------------
template <class XT, class AT>
struct GatherVec {
    const XT *__restrict__ x;
    __device__ __forceinline__ AT operator()(uint32_t c) const { return (AT)__ldg(x + c); }
};
// x = w .* b on the fly: the first Jacobi sweep from a zero guess fused into the second.
template <class T>
struct GatherWB {
    const T *__restrict__ w;
    const T *__restrict__ b;
    __device__ __forceinline__ T operator()(uint32_t c) const { return __ldg(w + c) * __ldg(b + c); }
};

// Multiply-add policy: FP64 paths round the product and the sum separately
// (bit-identical to the reference's sequential kernels and to the .NET CPU
// code); FP32 V-cycle paths contract to FMA.
template <class AT>
__device__ __forceinline__ AT madd(AT acc, AT a, AT b);
template <>
__device__ __forceinline__ double madd<double>(double acc, double a, double b) { return __dadd_rn(acc, __dmul_rn(a, b)); }
template <>
__device__ __forceinline__ float madd<float>(float acc, float a, float b) { return fmaf(a, b, acc); }

// Epilogues that set FUSED = true accept one fused multiply-add per term in FP64
// (more accurate, half the FP64 operations); all others keep the reference's order
// of a rounded product followed by a rounded add.
template <class Op, class = void>
struct op_fused : std::false_type {};
template <class Op>
struct op_fused<Op, std::void_t<decltype(Op::FUSED)>> : std::integral_constant<bool, Op::FUSED> {};
template <class AT, bool FUSED>
__device__ __forceinline__ AT madd_op(AT acc, AT a, AT b) {
    if constexpr (FUSED) return fma(a, b, acc);
    else return madd<AT>(acc, a, b);
}

// ---------------------------------------------------------------------------
// epilogues (row operators).  Each has NRED reduction slots and MAXMASK.  An
// epilogue may define touch(r): a prefetch of what row() will read at rows r .. r+2,
// issued by the streaming kernels one step before they finish those rows.
// ---------------------------------------------------------------------------
struct NoRed {
    static constexpr int NRED = 0;
    static constexpr unsigned MAXMASK = 0;
    __device__ void finish(const double *) const {}
};

template <class T>
__device__ __forceinline__ void prefetch_l1(const T *p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
template <class Op, class = void>
struct op_touch : std::false_type {};
template <class Op>
struct op_touch<Op, std::void_t<decltype(std::declval<const Op &>().touch(0))>> : std::true_type {};
template <class Op>
__device__ __forceinline__ void touch_rows(const Op &op, int32_t r) {
    if constexpr (op_touch<Op>::value) op.touch(r);
}

// y = A x (clear) or y += A x, accumulating onto the old y in entry order.
template <class YT, class AT>
struct OpSpmv : NoRed {
    YT *__restrict__ y;
    int clear;
    __device__ __forceinline__ AT init(int32_t r) const { return clear ? AT(0) : (AT)y[r]; }
    __device__ __forceinline__ void row(int32_t r, AT s, double *) const { y[r] = (YT)s; }
    __device__ __forceinline__ void touch(int32_t) const {}
};

// y = A x (restriction into the next level's right-hand side) and wb = w .* y, the product the
// next level's first Jacobi sweep gathers
template <class T>
struct OpRestrictWB : NoRed {
    T *__restrict__ y;
    T *__restrict__ wb;
    const T *__restrict__ w;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t r, T s, double *) const {
        y[r] = s;
        wb[r] = w[r] * s;
    }
    __device__ __forceinline__ void touch(int32_t) const {}
};

// r = b - A x
template <class T>
struct OpResid : NoRed {
    const T *__restrict__ b;
    T *__restrict__ r;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t i, T s, double *) const { r[i] = b[i] - s; }
    __device__ __forceinline__ void touch(int32_t i) const { prefetch_l1(b + i); }
};

// y = x + w .* (b - A x)  (jacobi_iteration, CsrGeometricMultigrid.cl:176-194)
template <class T>
struct OpJacobi : NoRed {
    const T *__restrict__ x;
    const T *__restrict__ w;
    const T *__restrict__ b;
    T *__restrict__ y;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t i, T s, double *) const { y[i] = x[i] + w[i] * (b[i] - s); }
    __device__ __forceinline__ void touch(int32_t i) const {
        prefetch_l1(x + i);
        prefetch_l1(w + i);
        prefetch_l1(b + i);
    }
};
// Second sweep from a zero guess: x1 = w .* b, y = x1 + w .* (b - A x1).
template <class T>
struct OpJacobiFromZero : NoRed {
    const T *__restrict__ w;
    const T *__restrict__ b;
    T *__restrict__ y;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t i, T s, double *) const {
        T wi = w[i], bi = b[i];
        y[i] = wi * bi + wi * (bi - s);
    }
    __device__ __forceinline__ void touch(int32_t i) const {
        prefetch_l1(w + i);
        prefetch_l1(b + i);
    }
};

// Device scalars shared by the solver kernels of one solve.
struct SolverScalars {
    double rz, rz_new, pap, alpha, beta;   // Jacobi PCG
    double zr, zq, pq;                     // flexible CG
    double rr, bb, tol2, res_max, res_norm2;
    int it, max_it, done, converged, failed, restart, cycle, pad;
};

// Last Jacobi sweep of the finest level with the flexible-CG dot products of its
// result z fused in: z.q, z.r and beta = -(z.q)/(p.q) (0 on a restart), as k_fcg_red.
template <class T>
struct OpJacobiFcgRed {
    static constexpr int NRED = 2;
    static constexpr unsigned MAXMASK = 0;
    const T *__restrict__ x;
    const T *__restrict__ w;
    const T *__restrict__ b;
    T *__restrict__ y;
    const double *__restrict__ q;
    const double *__restrict__ r;
    SolverScalars *sc;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t i, T s, double *red) const {
        const T z = x[i] + w[i] * (b[i] - s);
        y[i] = z;
        red[0] += (double)z * q[i];
        red[1] += (double)z * r[i];
    }
    __device__ __forceinline__ void touch(int32_t i) const {
        prefetch_l1(x + i);
        prefetch_l1(w + i);
        prefetch_l1(b + i);
        prefetch_l1(q + i);
        prefetch_l1(r + i);
    }
    __device__ void finish(const double *t) const {
        sc->zq = t[0];
        sc->zr = t[1];
        sc->beta = sc->restart ? 0.0 : -t[0] / sc->pq;
        sc->restart = 0;
    }
};

// PCG: Ap = A p and p.Ap; alpha = rz / pAp (dot_finalize_and_calc_a, CsrCG.cl:223-241).
struct OpPcgAp {
    static constexpr int NRED = 1;
    static constexpr unsigned MAXMASK = 0;
    const double *__restrict__ p;
    double *__restrict__ ap;
    SolverScalars *sc;
    __device__ __forceinline__ double init(int32_t) const { return 0.0; }
    __device__ __forceinline__ void row(int32_t i, double s, double *red) const {
        ap[i] = s;
        red[0] = __dadd_rn(red[0], __dmul_rn(p[i], s));
    }
    __device__ void finish(const double *t) const {
        sc->pap = t[0];
        sc->alpha = sc->rz / t[0];
    }
};

// Flexible CG outer product: s = (A z)_i, q = s + beta q, p = z + beta p, p.q.
template <class ZT>
struct OpFcg {
    static constexpr int NRED = 1;
    static constexpr unsigned MAXMASK = 0;
    static constexpr bool FUSED = true;   // products may use fused multiply-adds (not a parity path)
    const ZT *__restrict__ z;
    double *__restrict__ p;
    double *__restrict__ q;
    SolverScalars *sc;
    double beta;   // unused placeholder: beta is read from sc in row()
    __device__ __forceinline__ double init(int32_t) const { return 0.0; }
    __device__ __forceinline__ void row(int32_t i, double s, double *red) const {
        double bt = sc->beta;
        double qi = s + bt * q[i];
        double pi = (double)z[i] + bt * p[i];
        q[i] = qi;
        p[i] = pi;
        red[0] += pi * qi;
    }
    __device__ __forceinline__ void touch(int32_t i) const {
        prefetch_l1(z + i);
        prefetch_l1(p + i);
        prefetch_l1(q + i);
    }
    __device__ void finish(const double *t) const {
        sc->pq = t[0];
        sc->alpha = sc->zr / t[0];
    }
};

// r = b - A x with the max-norm / NaN check of residual_with_check
// (CsrGeometricMultigrid.cl:121-141): converged when all |r_i| <= tol, failed
// on NaN or |r_i| > 1e50.  Also ||r||^2.  The last block updates the cycle
// counter and the stop decision of the V-cycle driver.
struct OpResidCheck {
    static constexpr int NRED = 3;
    static constexpr unsigned MAXMASK = 0b011;
    const double *__restrict__ b;
    double *__restrict__ r;
    SolverScalars *sc;
    double tol;
    __device__ __forceinline__ double init(int32_t) const { return 0.0; }
    __device__ __forceinline__ void row(int32_t i, double s, double *red) const {
        double ri = __dsub_rn(b[i], s);
        r[i] = ri;
        double c = fabs(ri);
        if (isnan(ri) || c > 1e50) red[1] = 1.0;
        else red[0] = fmax(red[0], c);
        red[2] += ri * ri;
    }
    __device__ void finish(const double *t) const {
        bool failed = t[1] != 0.0;
        bool converged = !failed && t[0] <= tol;
        sc->res_max = t[0];
        sc->res_norm2 = sqrt(t[2]);
        sc->converged = converged;
        sc->failed = failed;
        if (converged || failed || sc->cycle > sc->max_it) sc->done = 1;
        else sc->cycle += 1;
    }
};

// ---------------------------------------------------------------------------
// CSR row kernel: TPR threads per row, grid-stride over rows
// ---------------------------------------------------------------------------
template <int TPR, class MT, class AT, class Gather, class Op>
__global__ void __launch_bounds__(kThreads) k_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                                  const MT *__restrict__ va, int32_t n, Gather g, Op op,
                                                  const int *__restrict__ done, double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    constexpr int U = 4;   // entries per lane per step: all index/value loads, then all gathers, then the FMAs
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    const int sub = threadIdx.x % TPR;
    const int gpb = kThreads / TPR;
    for (int32_t row = blockIdx.x * gpb + threadIdx.x / TPR; row < n; row += gridDim.x * gpb) {
        const int32_t s0 = __ldg(rp + row), s1 = __ldg(rp + row + 1);
        AT s = (TPR == 1) ? op.init(row) : AT(0);
        for (int32_t base = s0 + sub; base < s1; base += TPR * U) {
            int32_t c[U];
            AT v[U], xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t k = base + u * TPR;
                c[u] = k < s1 ? __ldcs(ci + k) : 0;
                v[u] = k < s1 ? (AT)__ldcs(va + k) : AT(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = (base + u * TPR < s1) ? g((uint32_t)c[u]) : AT(0);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (base + u * TPR < s1) s = madd<AT>(s, v[u], xv[u]);
        }
        s = group_sum<TPR>(s);
        if (TPR > 1) s = op.init(row) + s;
        if (sub == 0) op.row(row, s, red);
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

// ---------------------------------------------------------------------------
// DuVi row-bundle kernel
//
// One warp per bundle of <= 32 consecutive rows.  The warp copies the
// bundle's entry bytes (Distances), value indices and block column starts into
// its shared-memory stage with 16-byte loads (ranges widened to 16-byte
// boundaries; device arrays carry tail padding), then each lane walks one row
// of the stage in the order of DuViGeometricMultigrid.cl:84-98.  Tables of at
// most 256 distinct values are staged per block.
// ---------------------------------------------------------------------------
struct DuviArgs {
    const uint32_t *__restrict__ row_to_col;
    const uint32_t *__restrict__ row_to_dist;
    const uint32_t *__restrict__ col_idx;
    const uint8_t *__restrict__ dist;
    const void *__restrict__ vidx;
    const void *__restrict__ values;
    const int32_t *__restrict__ bundles;
    int32_t nbundles;
    int32_t nuniq;
};

template <class VI>
__device__ __forceinline__ void copy16(void *dst, const void *src, int nbytes16, int lane) {
    const uint4 *s = static_cast<const uint4 *>(src);
    uint4 *d = static_cast<uint4 *>(dst);
    for (int i = lane; i < nbytes16; i += 32) d[i] = __ldg(s + i);
}

template <class VI, class AT, class Gather, class Op, int WARPS, int BATCH>
__global__ void __launch_bounds__(WARPS * 32, 2) k_duvi(DuviArgs A, Gather g, Op op, const int *__restrict__ done,
                                                     double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool kSmemTable = sizeof(VI) == 1;
    AT *tab = reinterpret_cast<AT *>(smem);
    unsigned char *wbase = smem + (kSmemTable ? 256 * sizeof(AT) : 0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *sdist = wbase + (size_t)warp * (kStageD + kStageD * sizeof(VI) + kStageC * 4);
    VI *svi = reinterpret_cast<VI *>(sdist + kStageD);
    uint32_t *scol = reinterpret_cast<uint32_t *>(sdist + kStageD + kStageD * sizeof(VI));
    const AT *gtab = static_cast<const AT *>(A.values);
    const VI *gvi = static_cast<const VI *>(A.vidx);
    if (kSmemTable) {
        for (int i = threadIdx.x; i < A.nuniq; i += blockDim.x) tab[i] = gtab[i];
        __syncthreads();
    }
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;

    for (int32_t bi = blockIdx.x * WARPS + warp; bi < A.nbundles; bi += gridDim.x * WARPS) {
        const int32_t r0 = __ldg(A.bundles + bi), r1 = __ldg(A.bundles + bi + 1);
        const int32_t rl = min(r0 + lane, r1);
        const uint32_t rd_l = __ldg(A.row_to_dist + rl), rc_l = __ldg(A.row_to_col + rl);
        const uint32_t d0 = __shfl_sync(0xffffffffu, rd_l, 0), c0 = __shfl_sync(0xffffffffu, rc_l, 0);
        const uint32_t d1 = __ldg(A.row_to_dist + r1), c1 = __ldg(A.row_to_col + r1);
        const int32_t row = r0 + lane;
        if (d1 - d0 <= (uint32_t)kBundleBytes && c1 - c0 <= (uint32_t)kBundleBlocks) {
            // stage
            const uint32_t a0 = d0 & ~15u;
            const int nd16 = (int)((d1 - a0 + 15u) >> 4);
            copy16<VI>(sdist, A.dist + a0, nd16, lane);
            const uint64_t vb0 = ((uint64_t)d0 * sizeof(VI)) & ~(uint64_t)15;
            const int nv16 = (int)(((uint64_t)d1 * sizeof(VI) - vb0 + 15u) >> 4);
            copy16<VI>(svi, reinterpret_cast<const unsigned char *>(gvi) + vb0, nv16, lane);
            const uint32_t ca0 = c0 & ~3u;
            const int nc16 = (int)((c1 - ca0 + 3u) >> 2);
            copy16<VI>(scol, A.col_idx + ca0, nc16, lane);
            __syncwarp();
            if (row < r1) {
                uint32_t di = rd_l - a0;
                uint32_t dv = rd_l - (uint32_t)(vb0 / sizeof(VI));
                const uint32_t b_end = __ldg(A.row_to_col + row + 1) - ca0;
                AT s = op.init(row);
                for (uint32_t b = rc_l - ca0; b < b_end; ++b) {
                    const uint32_t n = sdist[di] + 1u;   // entries of the block
                    uint32_t cc = scol[b];
                    uint32_t k = 0;
                    // batches of BATCH entries: column prefix from the gap bytes, then
                    // BATCH independent gathers, then the FMAs in entry order
                    for (; k + BATCH <= n; k += BATCH) {
                        uint32_t cols[BATCH];
                        AT vals[BATCH], xs[BATCH];
#pragma unroll
                        for (int u = 0; u < BATCH; ++u) {
                            cols[u] = cc;
                            cc += sdist[di + k + u + 1] + 1u;   // gap to the next entry (the last read is unused)
                            vals[u] = kSmemTable ? tab[svi[dv + k + u]] : __ldg(gtab + svi[dv + k + u]);
                        }
#pragma unroll
                        for (int u = 0; u < BATCH; ++u) xs[u] = g(cols[u]);
#pragma unroll
                        for (int u = 0; u < BATCH; ++u) s = madd<AT>(s, vals[u], xs[u]);
                    }
                    for (; k < n; ++k) {
                        const AT v = kSmemTable ? tab[svi[dv + k]] : __ldg(gtab + svi[dv + k]);
                        const AT xv = g(cc);
                        cc += sdist[di + k + 1] + 1u;
                        s = madd<AT>(s, v, xv);
                    }
                    di += n;
                    dv += n;
                }
                op.row(row, s, red);
            }
            __syncwarp();
        } else if (lane == 0) {
            // a row longer than the stage: walk it from global memory
            for (int32_t rr = r0; rr < r1; ++rr) {
                uint32_t di = __ldg(A.row_to_dist + rr);
                const uint32_t be = __ldg(A.row_to_col + rr + 1);
                AT s = op.init(rr);
                for (uint32_t b = __ldg(A.row_to_col + rr); b < be; ++b) {
                    uint32_t c = __ldg(A.col_idx + b);
                    int cnt = __ldg(A.dist + di);
                    s = madd<AT>(s, kSmemTable ? tab[__ldg(gvi + di)] : __ldg(gtab + __ldg(gvi + di)), g(c));
                    for (int k = 0; k < cnt; ++k) {
                        ++di;
                        c += __ldg(A.dist + di) + 1u;
                        s = madd<AT>(s, kSmemTable ? tab[__ldg(gvi + di)] : __ldg(gtab + __ldg(gvi + di)), g(c));
                    }
                    ++di;
                }
                op.row(rr, s, red);
            }
        }
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

template <class VI, class AT>
constexpr size_t duvi_smem_bytes(int warps) {
    return (sizeof(VI) == 1 ? 256 * sizeof(AT) : 0) + (size_t)warps * (kStageD + kStageD * sizeof(VI) + kStageC * 4);
}

// ---------------------------------------------------------------------------
// launch dispatch
// ---------------------------------------------------------------------------
struct LaunchEnv {
    dv_context *ctx;
    cudaStream_t stream;
    const int *done;
    double *partials;
    unsigned *ticket;
    int max_blocks;
};

// ---------------------------------------------------------------------------
// DuVi lane kernel (lane-interleaved derived layout, see DuviLanesHost)
//
// One warp per bundle of 32 row groups, one lane per group.  The loop over the
// bundle's 4-entry words is warp-uniform; each lane decodes its leader row's
// columns once (entry byte 255: next block column; otherwise column += byte + 1)
// and applies every gathered x value to the G rows of its group, which share
// the column structure.  Words whose 4 entries all belong to the lane take a
// path without per-entry predicates; only a lane's last word is predicated.
// With SCALED, 8-bit value indices are byte offsets into the shared-memory
// table (one byte extract and one shared load per value).  No staging: every
// stream load is a coalesced 128-byte warp transaction, issued one word ahead
// (register double buffer, streaming loads).  Each row still sums its entries
// in order, so FP64 results equal the reference walk bit for bit.
// ---------------------------------------------------------------------------
template <class VI> struct ViChunk;
template <> struct ViChunk<uint8_t> { using T = uint32_t; };
template <> struct ViChunk<uint16_t> { using T = uint2; };
template <> struct ViChunk<uint32_t> { using T = uint4; };

__device__ __forceinline__ uint32_t vi_get(uint32_t c, int k) { return __byte_perm(c, 0u, 0x4440u + (unsigned)k); }
__device__ __forceinline__ uint32_t vi_get(uint2 c, int k) { return ((k < 2 ? c.x : c.y) >> (16 * (k & 1))) & 0xFFFFu; }
__device__ __forceinline__ uint32_t vi_get(uint4 c, int k) { return k == 0 ? c.x : k == 1 ? c.y : k == 2 ? c.z : c.w; }

struct DuviLanesArgs {
    const uint32_t *__restrict__ meta;
    const uint32_t *__restrict__ dist;
    const void *__restrict__ vi;
    const uint32_t *__restrict__ cols;
    const uint32_t *__restrict__ nent;
    const void *__restrict__ values;
    const void *__restrict__ tuples;   // node-tuple mode: 4 values per tuple
    const int32_t *__restrict__ offsets;   // stencil mode: column - first row of the group
    int64_t ngroups;
    int32_t nbundles;
    int32_t nuniq;
    int32_t ntup;
    int32_t noff;
};

// the (up to) 3 row values of a node tuple: one 16-byte shared load (FP32) or two (FP64)
__device__ __forceinline__ void tup_get(const float *t, uint32_t idx, float (&v)[4]) {
    const float4 q = reinterpret_cast<const float4 *>(t)[idx];
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void tup_get(const double *t, uint32_t idx, double (&v)[4]) {
    const double2 *p = reinterpret_cast<const double2 *>(t) + 2 * idx;
    const double2 a = p[0], b = p[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <class AT, bool SCALED, bool SMEM, class Chunk>
__device__ __forceinline__ AT lane_value(const AT *tab, const AT *gtab, const Chunk &c, int k) {
    const uint32_t idx = vi_get(c, k);
    if constexpr (SCALED) return *reinterpret_cast<const AT *>(reinterpret_cast<const char *>(tab) + idx);
    else if constexpr (SMEM) return tab[idx];
    else return __ldg(gtab + idx);
}

template <class VI, class AT, class Gather, class Op, int G, bool SCALED, bool SHIFT, bool TUP, bool STEN>
__global__ void __launch_bounds__(256) k_duvi_lanes(DuviLanesArgs A, Gather g, Op op, const int *__restrict__ done,
                                                    double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    using Chunk = typename ViChunk<VI>::T;
    constexpr bool kSmemTable = sizeof(VI) == 1;
    constexpr int NV = TUP ? 1 : G;   // index chunks per word
    __shared__ __align__(16) AT tab[TUP ? 1024 : (kSmemTable ? 256 : 1)];
    const AT *gtab = static_cast<const AT *>(A.values);
    __shared__ int32_t soff[STEN ? 256 : 1];
    if constexpr (STEN)
        for (int i = threadIdx.x; i < A.noff; i += blockDim.x) soff[i] = A.offsets[i];
    if constexpr (TUP) {
        const AT *tg = static_cast<const AT *>(A.tuples);
        for (int i = threadIdx.x; i < 4 * A.ntup; i += blockDim.x) tab[i] = tg[i];
        __syncthreads();
    } else if (kSmemTable) {
        for (int i = threadIdx.x; i < A.nuniq; i += blockDim.x) tab[i] = gtab[i];
        __syncthreads();
    }
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const Chunk *vbase = static_cast<const Chunk *>(A.vi);
    for (int32_t bi = blockIdx.x * wpb + (threadIdx.x >> 5); bi < A.nbundles; bi += gridDim.x * wpb) {
        const uint32_t d_base = __ldg(A.meta + 5 * bi), v_base = __ldg(A.meta + 5 * bi + 1);
        const uint32_t c_base = __ldg(A.meta + 5 * bi + 2), words = __ldg(A.meta + 5 * bi + 3);
        const int64_t grp = (int64_t)bi * 32 + lane;
        const bool valid = grp < A.ngroups;
        const uint32_t ne = valid ? __ldg(A.nent + grp) : 0u;
        const uint32_t full = ne >> 2;   // words whose 4 entries are all this lane's
        const int32_t r0 = (int32_t)(grp * G);
        AT s[G];
#pragma unroll
        for (int d = 0; d < G; ++d) s[d] = valid ? op.init(r0 + d) : AT(0);
        const uint32_t *dp = A.dist + d_base + lane;
        const Chunk *vp = vbase + v_base + lane;
        const uint32_t *cp = A.cols + c_base + lane;
        uint32_t c = 0;
        // register double buffer: the streams of word w+1 are in flight while word w is decoded
        uint32_t dw_next = 0;
        Chunk vw_next[NV];
        if (words > 0) {
            dw_next = __ldcs(dp);
#pragma unroll
            for (int d = 0; d < NV; ++d) vw_next[d] = __ldcs(vp + (size_t)d * 32);
        }
        for (uint32_t w = 0; w < words; ++w) {
            const uint32_t dw = dw_next;
            Chunk vw[NV];
#pragma unroll
            for (int d = 0; d < NV; ++d) vw[d] = vw_next[d];
            if (w + 1 < words) {
                dw_next = __ldcs(dp + (size_t)(w + 1) * 32);
#pragma unroll
                for (int d = 0; d < NV; ++d) vw_next[d] = __ldcs(vp + ((size_t)(w + 1) * NV + d) * 32);
            }
            if (w < full) {
                uint32_t cols[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t byte = __byte_perm(dw, 0u, 0x4440u + (unsigned)k);
                    if constexpr (STEN) {
                        c = (uint32_t)(r0 + soff[byte]);
                    } else if (byte == 255u) {
                        c = __ldcs(cp);
                        cp += 32;
                    } else {
                        c += byte + 1u;
                    }
                    cols[k] = c;
                }
                if constexpr (SHIFT) {   // row d reads column + d
                    AT xs[4][G];
#pragma unroll
                    for (int k = 0; k < 4; ++k)
#pragma unroll
                        for (int d = 0; d < G; ++d) xs[k][d] = g(cols[k] + (uint32_t)d);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        AT tv[4];
                        if constexpr (TUP) tup_get(tab, vi_get(vw[0], k), tv);
#pragma unroll
                        for (int d = 0; d < G; ++d)
                            s[d] = madd<AT>(s[d], TUP ? tv[d] : lane_value<AT, SCALED, kSmemTable>(tab, gtab, vw[TUP ? 0 : d], k),
                                            xs[k][d]);
                    }
                } else {
                    AT xv[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) xv[k] = g(cols[k]);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        AT tv[4];
                        if constexpr (TUP) tup_get(tab, vi_get(vw[0], k), tv);
#pragma unroll
                        for (int d = 0; d < G; ++d)
                            s[d] = madd<AT>(s[d], TUP ? tv[d] : lane_value<AT, SCALED, kSmemTable>(tab, gtab, vw[TUP ? 0 : d], k),
                                            xv[k]);
                    }
                }
            } else if (w * 4 < ne) {   // the lane's last, partial word
                uint32_t cols[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t byte = __byte_perm(dw, 0u, 0x4440u + (unsigned)k);
                    if (w * 4 + k < ne) {
                        if constexpr (STEN) {
                            c = (uint32_t)(r0 + soff[byte]);
                        } else if (byte == 255u) {
                            c = __ldcs(cp);
                            cp += 32;
                        } else {
                            c += byte + 1u;
                        }
                    }
                    cols[k] = c;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (w * 4 + k < ne) {
                        const AT x0 = SHIFT ? AT(0) : g(cols[k]);
                        AT tv[4];
                        if constexpr (TUP) tup_get(tab, vi_get(vw[0], k), tv);
#pragma unroll
                        for (int d = 0; d < G; ++d)
                            s[d] = madd<AT>(s[d], TUP ? tv[d] : lane_value<AT, SCALED, kSmemTable>(tab, gtab, vw[TUP ? 0 : d], k),
                                            SHIFT ? g(cols[k] + (uint32_t)d) : x0);
                    }
                }
            }
        }
        if (valid) {
#pragma unroll
            for (int d = 0; d < G; ++d) op.row(r0 + d, s[d], red);
        }
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

template <class VI, class AT, class Gather, class Op, int G>
void launch_duvi_lanes_g(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    DuviLanesArgs a;
    a.meta = m->lanes_meta.as<uint32_t>();
    a.dist = m->lanes_dist.as<uint32_t>();
    a.vi = m->lanes_vi.p;
    a.cols = m->lanes_cols.as<uint32_t>();
    a.nent = m->lanes_nent.as<uint32_t>();
    a.values = m->values.p;
    a.tuples = m->lanes_tup.p;
    a.offsets = m->lanes_off.as<int32_t>();
    a.noff = m->lanes_noff;
    a.ngroups = m->lanes_groups;
    a.nbundles = (int32_t)m->lanes_bundles;
    a.nuniq = (int32_t)m->nuniq;
    a.ntup = m->lanes_ntup;
    int blocks = (int)((m->lanes_bundles + 7) / 8);
    if (blocks > e.max_blocks) blocks = e.max_blocks;
    if (blocks < 1) blocks = 1;
    const bool sh = G > 1 && m->lanes_shift;
    bool done_launch = false;
    if constexpr (sizeof(VI) == 1) {
        if constexpr (G > 1) {
            if (m->lanes_stencil) {
                k_duvi_lanes<VI, AT, Gather, Op, G, false, false, true, true><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
                done_launch = true;
            } else if (m->lanes_tuples) {
                if (sh) k_duvi_lanes<VI, AT, Gather, Op, G, false, true, true, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
                else k_duvi_lanes<VI, AT, Gather, Op, G, false, false, true, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
                done_launch = true;
            }
        }
        if (!done_launch && m->lanes_scaled) {
            if (sh) k_duvi_lanes<VI, AT, Gather, Op, G, true, G != 1, false, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
            else k_duvi_lanes<VI, AT, Gather, Op, G, true, false, false, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
            done_launch = true;
        }
    }
    if (!done_launch) {
        if (sh) k_duvi_lanes<VI, AT, Gather, Op, G, false, G != 1, false, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
        else k_duvi_lanes<VI, AT, Gather, Op, G, false, false, false, false><<<blocks, 256, 0, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
    }
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

template <class VI, class AT, class Gather, class Op>
void launch_duvi_lanes(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    if (m->lanes_group == 3) launch_duvi_lanes_g<VI, AT, Gather, Op, 3>(e, m, g, op);
    else if (m->lanes_group == 2) launch_duvi_lanes_g<VI, AT, Gather, Op, 2>(e, m, g, op);
    else launch_duvi_lanes_g<VI, AT, Gather, Op, 1>(e, m, g, op);
}


// ---------------------------------------------------------------------------
// DuVi node-pattern kernel (derived layout, see DuviPatternHost)
//
// One thread per node group.  The group's pattern id selects a run of records
// {column offset from the group's first row, the G row values} staged in shared
// memory; the thread gathers x at each offset and applies it to its G rows,
// summing every row in its entry order (FP64 results equal the reference walk
// bit for bit).  The matrix costs 2 bytes per group in DRAM; the product is
// bound by the x gathers.
// ---------------------------------------------------------------------------
template <class AT>
struct alignas(16) PatRec {
    int32_t off;
    AT v[3];
};
static_assert(sizeof(PatRec<float>) == 16 && offsetof(PatRec<float>, v) == 4, "FP32 pattern record layout");
static_assert(sizeof(PatRec<double>) == 32 && offsetof(PatRec<double>, v) == 8, "FP64 pattern record layout");

// Stages a pattern table (records and pattern starts) in shared memory.
template <class AT>
__device__ __forceinline__ void stage_patterns(uint4 *smem, const PatRec<AT> *__restrict__ grec,
                                               const uint32_t *__restrict__ pstart, int32_t npat, int32_t nrec) {
    uint32_t *st = reinterpret_cast<uint32_t *>(reinterpret_cast<PatRec<AT> *>(smem) + nrec);
    const uint4 *src = reinterpret_cast<const uint4 *>(grec);
    const int n16 = nrec * (int)(sizeof(PatRec<AT>) / 16);
    for (int i = threadIdx.x; i < n16; i += blockDim.x) smem[i] = __ldg(src + i);
    for (int i = threadIdx.x; i <= npat; i += blockDim.x) st[i] = __ldg(pstart + i);
}

// One node group from its pattern records (shared memory): every row summed in entry order.
// BASED: offsets from the group's first column (base[]), else from its first row;
// SHIFT: row d of the group reads column + d.
template <class AT, class Gather, class Op, int G, bool BASED, bool SHIFT>
__device__ __forceinline__ void pattern_group(int64_t gi, const PatRec<AT> *rec, const uint32_t *st,
                                              const uint16_t *__restrict__ pid, const uint32_t *__restrict__ base,
                                              const Gather &g, const Op &op, double *red) {
    const uint32_t p = __ldg(pid + gi);
    const uint32_t b = st[p], e = st[p + 1];
    const int32_t r0 = (int32_t)(gi * G);
    const int32_t c0 = BASED ? (int32_t)__ldg(base + gi) : r0;
    AT s[G];
#pragma unroll
    for (int d = 0; d < G; ++d) s[d] = op.init(r0 + d);
    uint32_t k = b;
    for (; k + 4 <= e; k += 4) {
        PatRec<AT> q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = rec[k + u];
        if constexpr (SHIFT) {
            AT x[4][G];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int d = 0; d < G; ++d) x[u][d] = g((uint32_t)(c0 + q[u].off + d));
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int d = 0; d < G; ++d) s[d] = madd_op<AT, op_fused<Op>::value>(s[d], q[u].v[d], x[u][d]);
        } else {
            AT x[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) x[u] = g((uint32_t)(c0 + q[u].off));
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int d = 0; d < G; ++d) s[d] = madd_op<AT, op_fused<Op>::value>(s[d], q[u].v[d], x[u]);
        }
    }
    for (; k < e; ++k) {
        const PatRec<AT> q = rec[k];
#pragma unroll
        for (int d = 0; d < G; ++d) s[d] = madd_op<AT, op_fused<Op>::value>(s[d], q.v[d], g((uint32_t)(c0 + q.off + (SHIFT ? d : 0))));
    }
#pragma unroll
    for (int d = 0; d < G; ++d) op.row(r0 + d, s[d], red);
}

template <class AT, class Gather, class Op, int G, bool BASED, bool SHIFT>
__global__ void __launch_bounds__(256) k_duvi_pattern(const uint16_t *__restrict__ pid, const uint32_t *__restrict__ pstart,
                                                      const PatRec<AT> *__restrict__ grec, const uint32_t *__restrict__ base,
                                                      int32_t npat, int32_t nrec, int64_t ngroups, Gather g, Op op,
                                                      const int *__restrict__ done, double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 pat_smem[];
    const PatRec<AT> *rec = reinterpret_cast<const PatRec<AT> *>(pat_smem);
    const uint32_t *st = reinterpret_cast<const uint32_t *>(rec + nrec);
    stage_patterns<AT>(pat_smem, grec, pstart, npat, nrec);
    __syncthreads();
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < ngroups; gi += (int64_t)gridDim.x * blockDim.x)
        pattern_group<AT, Gather, Op, G, BASED, SHIFT>(gi, rec, st, pid, base, g, op, red);
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

// ---------------------------------------------------------------------------
// DuVi grid-stencil kernel (derived layout, see DuviGridHost)
//
// Operators whose node groups sit on an lx x ly x lz box (x fastest, 3 rows per group) and
// whose interior groups share one pattern coupling the 27 box neighbours.  A block owns a
// tile of 32 x 8 groups of the xy plane and a run of zc planes; it streams the planes z0-1 ..
// z1 through shared memory (the tile plus a one-group halo, 3 values per group, double
// buffered, the next plane's loads in flight during the current plane's arithmetic).  Each
// staged value is read once per thread and applied to the three groups it couples to in z
// (the plane below, at and above it), so a group's three rows collect the 81 columns in
// column order: plane z-1, then z, then z+1, each plane by y, x and dof.  With the same
// multiply-add rounding this is the node-pattern kernel's sum bit for bit.  The interior
// pattern's values are kernel parameters (constant-bank operands of the FMAs): no record
// loads, one shared-memory load per staged value.  Groups on the box faces, and interior
// groups of other patterns, are listed and run through their pattern records by the first
// blocks of the same launch.
// ---------------------------------------------------------------------------

// Structure of the interior row block of an isotropic trilinear hexahedron operator on a uniform
// grid (3 rows of a node against its 27 neighbours x 3 dofs, entry k and row d at 3 k + d): the
// entries of one class are equal and class -1 entries are zero, for every modulus and Poisson
// ratio.  The equalities come from the element's reflection and rotation symmetries, the zeros
// from the cancellation of the 8 elements that share the node (90 of the 243 entries).  Ten
// values then describe the whole stencil.  A matrix is checked against this table when its
// grid layout is built and uses it only if every equality and zero holds exactly.
constexpr int kHexClasses = 10;
#define DV_HEX_CLASS_TABLE \
    0,  1,  1,  1,  0,  1,  1,  1,  0,  2, -1, -1, -1,  3,  4, -1,  4,  3,  0,  5,  5,  5,  0,  1,  5,  1,  0, \
    3, -1,  4, -1,  2, -1,  4, -1,  3,  6, -1, -1, -1,  6, -1, -1, -1,  7,  3, -1,  8, -1,  2, -1,  8, -1,  3, \
    0,  5,  1,  5,  0,  5,  1,  5,  0,  2, -1, -1, -1,  3,  8, -1,  8,  3,  0,  1,  5,  1,  0,  5,  5,  5,  0, \
    3,  4, -1,  4,  3, -1, -1, -1,  2,  6, -1, -1, -1,  7, -1, -1, -1,  6,  3,  8, -1,  8,  3, -1, -1, -1,  2, \
    7, -1, -1, -1,  6, -1, -1, -1,  6,  9, -1, -1, -1,  9, -1, -1, -1,  9,  7, -1, -1, -1,  6, -1, -1, -1,  6, \
    3,  8, -1,  8,  3, -1, -1, -1,  2,  6, -1, -1, -1,  7, -1, -1, -1,  6,  3,  4, -1,  4,  3, -1, -1, -1,  2, \
    0,  1,  5,  1,  0,  5,  5,  5,  0,  2, -1, -1, -1,  3,  8, -1,  8,  3,  0,  5,  1,  5,  0,  5,  1,  5,  0, \
    3, -1,  8, -1,  2, -1,  8, -1,  3,  6, -1, -1, -1,  6, -1, -1, -1,  7,  3, -1,  4, -1,  2, -1,  4, -1,  3, \
    0,  5,  5,  5,  0,  1,  5,  1,  0,  2, -1, -1, -1,  3,  4, -1,  4,  3,  0,  1,  1,  1,  0,  1,  1,  1,  0
// The same table in device and host memory: device code indexes the __device__ copy, which
// the compiler folds to constants after unrolling (a table local to a constexpr function
// would be rebuilt at every inlined call).
__device__ constexpr signed char kHexClassDev[243] = {DV_HEX_CLASS_TABLE};
constexpr signed char kHexClassHost[243] = {DV_HEX_CLASS_TABLE};
__host__ __device__ __forceinline__ constexpr int hex_class(int i) {
#ifdef __CUDA_ARCH__
    return kHexClassDev[i];
#else
    return kHexClassHost[i];
#endif
}

constexpr int kGridTX = 32, kGridTY = 8;   // tile of groups per block: one warp per row (of NY rows each)
constexpr int kGridPX = kGridTX + 2;       // with halo
template <int NY>
struct PlaneDims {
    static constexpr int TY = kGridTY * NY;             // tile rows
    static constexpr int PY = TY + 2;                   // with halo
    static constexpr int PLANE = kGridPX * PY * 3;      // staged values per plane
    static constexpr int LOADS = (PLANE + 255) / 256;   // staging slots per thread
};
constexpr int kGridPlane = PlaneDims<1>::PLANE;   // 1020
constexpr int kGridLoads = PlaneDims<1>::LOADS;   // 4

template <class AT>
struct GridCoef {
    AT v[81][3];           // interior pattern: entry k = 27 dz' + 9 dy' + 3 dx' + c (primes: offset + 1), row d
    AT cls[kHexClasses];   // its class values when it has the hex structure (hex_class)
};

struct GridGeom {
    int32_t lx, ly, lz;        // group box
    int32_t ntx, nty, zc;      // tiles per plane in x and y, planes per z run
    int32_t ntile;             // ntx * nty * ceil((lz - 2) / zc): tiles over the interior nodes
    int32_t bound_blocks;      // blocks [0, bound_blocks) run the boundary list, the rest the tiles
    int32_t hot, all_hot;      // interior pattern id; 1 when no interior group has another pattern
    int64_t nbound;
};

// One term of a stencil row: the coefficient of entry k, row d.  HEX takes it from the ten class
// values (zero entries skipped where SKIP0, i.e. wherever the result need not equal the sequential
// sum over every stored entry bit for bit: NaN or infinite x and the sign of a zero sum are the
// only differences), otherwise from the full table.
template <class AT, bool FUSED, bool HEX, bool SKIP0>
__device__ __forceinline__ AT grid_term(AT acc, const GridCoef<AT> &cf, int k, int d, AT v) {
    if constexpr (HEX) {
        const int c = hex_class(3 * k + d);
        if (c >= 0) return madd_op<AT, FUSED>(acc, cf.cls[c], v);
        if constexpr (SKIP0) return acc;
        else return madd_op<AT, FUSED>(acc, AT(0), v);
    } else {
        return madd_op<AT, FUSED>(acc, cf.v[k][d], v);
    }
}

// Asynchronous global -> shared copies (cp.async, zero fill when `valid` is false: no global read).
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void *dst, const void *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES), "r"(valid ? BYTES : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// How a gather is staged through shared memory: its source arrays (x; or w and b when the
// gathered value is w .* b) are copied plane by plane, and a staged value is formed from them
// (the same arithmetic as the gather, so results do not depend on the path).
template <class G>
struct StageSrc;
template <class XT, class AT>
struct StageSrc<GatherVec<XT, AT>> {
    using ST = XT;
    static constexpr int N = 1;
    __device__ static const XT *src(const GatherVec<XT, AT> &g, int) { return g.x; }
    template <int PLANE = kGridPlane>
    __device__ static AT value(const XT *pl, int i) { return (AT)pl[i]; }
};
template <class T>
struct StageSrc<GatherWB<T>> {
    using ST = T;
    static constexpr int N = 2;
    __device__ static const T *src(const GatherWB<T> &g, int k) { return k == 0 ? g.w : g.b; }
    template <int PLANE = kGridPlane>
    __device__ static T value(const T *pl, int i) { return pl[i] * pl[i + PLANE]; }
};
constexpr int kGridStages = 4;   // staged planes in flight per block (a plane is consumed 3 steps after its copy)

// Staging slots of a thread: plane value k = threadIdx.x + 256 j is node (sx, sy) of the halo tile
// (offsets from the tile's first node), dof sc; sy = -1000000 past the plane.
template <int NY = 1>
struct StageSlots {
    static constexpr int LOADS = PlaneDims<NY>::LOADS, PLANE = PlaneDims<NY>::PLANE;
    int sx[LOADS], sy[LOADS], sc[LOADS];
    __device__ StageSlots() {
#pragma unroll
        for (int j = 0; j < LOADS; ++j) {
            const int k = threadIdx.x + 256 * j;
            const int row = k / (kGridPX * 3), col = k - row * (kGridPX * 3);
            sx[j] = col / 3 - 1;
            sc[j] = col - 3 * (col / 3);
            sy[j] = k < PLANE ? row - 1 : -1000000;
        }
    }
    // per tile: offset of each slot inside a plane of the lx x ly node box (-1: outside the box)
    __device__ void plane_offsets(int x0, int y0, int lx, int ly, int32_t (&poff)[LOADS]) const {
#pragma unroll
        for (int j = 0; j < LOADS; ++j) {
            const int xn = x0 + sx[j], yn = y0 + sy[j];
            poff[j] = (xn >= 0 && xn < lx && yn >= 0 && yn < ly) ? 3 * (xn + lx * yn) + sc[j] : -1;
        }
    }
    // copies plane z (zero outside 0 <= z < lz) of every source of the gather into one ring slot
    template <class SS, class Gather>
    __device__ void issue(const Gather &g, typename SS::ST *slot, const int32_t (&poff)[LOADS], int z, int lz,
                          int32_t plane_len, int64_t origin = 0) const {
        const bool zin = z >= 0 && z < lz;
        const int64_t base = zin ? origin + (int64_t)z * plane_len : 0;
#pragma unroll
        for (int k = 0; k < SS::N; ++k) {
            const typename SS::ST *src = SS::src(g, k);
#pragma unroll
            for (int j = 0; j < LOADS; ++j)
                if (sy[j] > -2) {
                    const bool v = zin && poff[j] >= 0;
                    cp_async_zfill<sizeof(typename SS::ST)>(slot + k * PLANE + threadIdx.x + 256 * j,
                                                            v ? src + base + poff[j] : src, v);
                }
        }
        cp_async_commit();
    }
};

// One staged plane applied to the three accumulated groups of each of the thread's NY nodes
// (rows q = 0 .. NY-1 of its column of the tile): below (DI: group p+1 takes the plane as its
// dz = -1 neighbours), at (DM: group p, dz = 0) and above (DF: group p-1, dz = +1).  A staged
// value of plane row r is loaded once and serves every node q with r - q in 0 .. 2.
template <class AT, class SS, int NY, bool FUSED, bool HEX, bool SKIP0, bool DI, bool DM, bool DF>
__device__ __forceinline__ void grid_plane_step(const typename SS::ST *__restrict__ pl, int tx, int ty,
                                                const GridCoef<AT> &cf, AT (&a0)[NY][3], AT (&a1)[NY][3],
                                                AT (&a2)[NY][3]) {
    constexpr int PLANE = PlaneDims<NY>::PLANE;
#pragma unroll
    for (int r = 0; r < NY + 2; ++r)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const AT v = SS::template value<PLANE>(pl, ((NY * ty + r) * kGridPX + tx + dx) * 3 + c);
#pragma unroll
                for (int q = 0; q < NY; ++q) {
                    const int dy = r - q;
                    if (dy < 0 || dy > 2) continue;
                    const int k = 9 * dy + 3 * dx + c;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        if (DI) a2[q][d] = grid_term<AT, FUSED, HEX, SKIP0>(a2[q][d], cf, k, d, v);
                        if (DM) a1[q][d] = grid_term<AT, FUSED, HEX, SKIP0>(a1[q][d], cf, 27 + k, d, v);
                        if (DF) a0[q][d] = grid_term<AT, FUSED, HEX, SKIP0>(a0[q][d], cf, 54 + k, d, v);
                    }
                }
            }
}

template <class AT, class Gather, class Op, bool HEX, int NY>
__global__ void __launch_bounds__(256, 3)   // 3 blocks an SM: FP64 fits 80 registers without spills
    k_duvi_grid(GridGeom G, GridCoef<AT> cf, const uint16_t *__restrict__ pid, const uint32_t *__restrict__ pstart,
                const PatRec<AT> *__restrict__ grec, const uint32_t *__restrict__ bnode, int32_t npat, int32_t nrec,
                Gather g, Op op, const int *__restrict__ done, double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 grid_smem[];
    constexpr bool FU = op_fused<Op>::value;
    constexpr bool S0 = FU || sizeof(AT) == 4;   // FP64 parity epilogues multiply the zeros too
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    if ((int32_t)blockIdx.x < G.bound_blocks) {
        // boundary groups from their pattern records
        const PatRec<AT> *rec = reinterpret_cast<const PatRec<AT> *>(grid_smem);
        const uint32_t *st = reinterpret_cast<const uint32_t *>(rec + nrec);
        stage_patterns<AT>(grid_smem, grec, pstart, npat, nrec);
        __syncthreads();
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G.nbound;
             i += (int64_t)G.bound_blocks * blockDim.x)
            pattern_group<AT, Gather, Op, 3, false, false>((int64_t)__ldg(bnode + i), rec, st, pid, nullptr, g, op, red);
    } else {
        using SS = StageSrc<Gather>;
        using ST = typename SS::ST;
        using SL = StageSlots<NY>;
        constexpr int SLOT = SS::N * SL::PLANE;
        ST *ring = reinterpret_cast<ST *>(grid_smem);   // kGridStages slots of SS::N staged planes
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
        const SL slots;
        const int64_t lxy = (int64_t)G.lx * G.ly;
        const int32_t plane_len = (int32_t)(3 * lxy);
        const int nblk = (int)gridDim.x - G.bound_blocks;
        for (int t = (int)blockIdx.x - G.bound_blocks; t < G.ntile; t += nblk) {
            const int txi = t % G.ntx, tyi = (t / G.ntx) % G.nty, tzi = t / (G.ntx * G.nty);
            // tiles cover the interior nodes 1 .. l-2 of each axis (the faces are boundary groups)
            const int x0 = 1 + txi * kGridTX, y0 = 1 + tyi * PlaneDims<NY>::TY, z0 = 1 + tzi * G.zc,
                      z1 = min(G.lz - 1, z0 + G.zc);
            const int ix = x0 + tx;
            int32_t col_xy[NY];   // group index in its plane of the thread's nodes
            bool inxy[NY];
#pragma unroll
            for (int q = 0; q < NY; ++q) {
                const int iy = y0 + NY * ty + q;
                col_xy[q] = ix + G.lx * iy;
                inxy[q] = ix >= 1 && ix <= G.lx - 2 && iy >= 1 && iy <= G.ly - 2;
            }
            int32_t poff[SL::LOADS];
            slots.plane_offsets(x0, y0, G.lx, G.ly, poff);
            // a stencil group (off the faces, interior pattern) that this thread finishes
            auto active = [&](int q, int z) {
                if (!inxy[q] || z < 1 || z > G.lz - 2) return false;
                return G.all_hot || (int)__ldg(pid + col_xy[q] + lxy * z) == G.hot;
            };
#pragma unroll
            for (int s2 = 0; s2 < kGridStages - 1; ++s2) {
                if (z0 - 1 + s2 <= z1) slots.template issue<SS>(g, ring + s2 * SLOT, poff, z0 - 1 + s2, G.lz, plane_len);
                else cp_async_commit();
            }
            AT a0[NY][3], a1[NY][3], a2[NY][3];
            bool act0[NY], act1[NY];
#pragma unroll
            for (int q = 0; q < NY; ++q) {
                act0[q] = act1[q] = false;
#pragma unroll
                for (int d = 0; d < 3; ++d) a0[q][d] = a1[q][d] = a2[q][d] = AT(0);
            }
            for (int p = z0 - 1, k = 0; p <= z1; ++p, ++k) {
                cp_async_wait<kGridStages - 2>();   // plane p has landed (this thread's copies)
                __syncthreads();                     // ... and everyone's; the slot of plane p-1 is free
                if (p + kGridStages - 1 <= z1)
                    slots.template issue<SS>(g, ring + ((k + kGridStages - 1) % kGridStages) * SLOT, poff,
                                             p + kGridStages - 1, G.lz, plane_len);
                else
                    cp_async_commit();
                const ST *pl = ring + (k % kGridStages) * SLOT;
                const bool di = p + 1 >= z0 && p + 1 < z1, dm = p >= z0 && p < z1, df = p - 1 >= z0 && p - 1 < z1;
                bool act2[NY];
#pragma unroll
                for (int q = 0; q < NY; ++q) {
                    act2[q] = di && active(q, p + 1);
                    if (di) {
                        const int32_t r = (int32_t)(3 * (col_xy[q] + lxy * (p + 1)));
#pragma unroll
                        for (int d = 0; d < 3; ++d) a2[q][d] = act2[q] ? op.init(r + d) : AT(0);
                    }
                    if (dm && act1[q]) touch_rows(op, (int32_t)(3 * (col_xy[q] + lxy * p)));   // finished next step
                }
                if (di && dm && df) grid_plane_step<AT, SS, NY, FU, HEX, S0, true, true, true>(pl, tx, ty, cf, a0, a1, a2);
                else if (di && dm) grid_plane_step<AT, SS, NY, FU, HEX, S0, true, true, false>(pl, tx, ty, cf, a0, a1, a2);
                else if (dm && df) grid_plane_step<AT, SS, NY, FU, HEX, S0, false, true, true>(pl, tx, ty, cf, a0, a1, a2);
                else if (di) grid_plane_step<AT, SS, NY, FU, HEX, S0, true, false, false>(pl, tx, ty, cf, a0, a1, a2);
                else if (dm) grid_plane_step<AT, SS, NY, FU, HEX, S0, false, true, false>(pl, tx, ty, cf, a0, a1, a2);
                else if (df) grid_plane_step<AT, SS, NY, FU, HEX, S0, false, false, true>(pl, tx, ty, cf, a0, a1, a2);
#pragma unroll
                for (int q = 0; q < NY; ++q) {
                    if (df && act0[q]) {
                        const int32_t r = (int32_t)(3 * (col_xy[q] + lxy * (p - 1)));
#pragma unroll
                        for (int d = 0; d < 3; ++d) op.row(r + d, a0[q][d], red);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        a0[q][d] = a1[q][d];
                        a1[q][d] = a2[q][d];
                    }
                    act0[q] = act1[q];
                    act1[q] = act2[q];
                }
            }
            cp_async_wait<0>();
            __syncthreads();   // the next tile refills the ring
        }
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

// Planes per z run of a streaming tile: the run that minimises (waves of tiles) x (plane steps
// per tile), with `conc` tiles resident at once; ties go to the longer run.  Runs of 2, 4, .. 64
// planes: measured at 128^3, the run that fits every tile into one wave (13 planes, 320 tiles) left
// SMs with fewer resident blocks and was slower (FP32 residual 54 against 46 us) than 512 tiles of 8;
// runs of 2 give the coarse levels more tiles (mixed solve 8.45 -> 8.30 ms).
inline int stream_run_length(int64_t plane_tiles, int lz, int64_t conc) {
    int best = 2;
    int64_t best_cost = INT64_MAX;
    for (int zc = 2; zc <= 64; zc *= 2) {
        const int64_t tiles = plane_tiles * ((lz + zc - 1) / zc);
        const int64_t cost = ((tiles + conc - 1) / conc) * (int64_t)(std::min(zc, lz) + 2);
        if (cost <= best_cost) {
            best_cost = cost;
            best = zc;
        }
    }
    return best;
}

// Grid-stencil launch: boundary blocks first (they run alongside the tiles), then tile blocks over
// runs of zc planes.
template <class AT, class Gather, class Op, bool HEX>
void launch_duvi_grid_h(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    // FP32: two nodes per thread in y (staged rows shared, per-step work amortised); FP64: one
    // (registers)
    constexpr int NY = sizeof(AT) == 4 ? 2 : 1;
    auto kern = k_duvi_grid<AT, Gather, Op, HEX, NY>;
    using SS = StageSrc<Gather>;
    const size_t smem = std::max(sizeof(typename SS::ST) * SS::N * kGridStages * (size_t)PlaneDims<NY>::PLANE,
                                 sizeof(PatRec<AT>) * (size_t)m->pat_entries + 4 * ((size_t)m->pat_count + 1));
    static SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
    static OccupancyCache occupancy;   // per instantiation
    const int occ = occupancy.get(kern, 256, smem, e.ctx->device);
    GridCoef<AT> cf;
    for (int k = 0; k < 81; ++k)
        for (int d = 0; d < 3; ++d) cf.v[k][d] = (AT)m->grid_coef[3 * k + d];
    for (int c = 0; c < kHexClasses; ++c) cf.cls[c] = HEX ? (AT)m->grid_cls[c] : AT(0);
    GridGeom G;
    G.lx = m->grid_lx;
    G.ly = m->grid_ly;
    G.lz = m->grid_lz;
    G.ntx = std::max(0, (G.lx - 2 + kGridTX - 1) / kGridTX);   // tiles over the interior nodes 1 .. l-2
    G.nty = std::max(0, (G.ly - 2 + PlaneDims<NY>::TY - 1) / PlaneDims<NY>::TY);
    G.hot = m->grid_hot;
    G.all_hot = m->grid_all_hot;
    G.nbound = m->grid_nb;
    const int64_t wave = (int64_t)e.ctx->num_sms * occ;
    // one boundary group a thread: more per thread puts the boundary blocks on the critical path
    // (measured: two or four a thread slowed the solve by 6 and 14 %)
    G.bound_blocks = G.nbound == 0 ? 0
                     : (int32_t)std::min<int64_t>((G.nbound + 255) / 256, std::max<int64_t>(1, e.max_blocks / 4));
    const int64_t plane_tiles = (int64_t)G.ntx * G.nty;
    const int lzi = std::max(1, G.lz - 2);
    G.zc = stream_run_length(plane_tiles, lzi, std::max<int64_t>(1, wave - G.bound_blocks / 2));
    G.ntile = G.lz > 2 ? (int32_t)(plane_tiles * ((lzi + G.zc - 1) / G.zc)) : 0;
    const int64_t tile_blocks = std::min<int64_t>(G.ntile, std::max<int64_t>(1, e.max_blocks - G.bound_blocks));
    const int blocks = (int)std::max<int64_t>(1, G.bound_blocks + tile_blocks);
    kern<<<blocks, 256, smem, e.stream>>>(G, cf, m->pat_id.as<uint16_t>(), m->pat_start.as<uint32_t>(),
                                          static_cast<const PatRec<AT> *>(m->pat_rec.p), m->grid_bnode.as<uint32_t>(),
                                          m->pat_count, m->pat_entries, g, op, e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

template <class AT, class Gather, class Op, int G, bool BASED, bool SHIFT>
void launch_duvi_pattern_gbs(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    auto kern = k_duvi_pattern<AT, Gather, Op, G, BASED, SHIFT>;
    const size_t smem = sizeof(PatRec<AT>) * (size_t)m->pat_entries + 4 * ((size_t)m->pat_count + 1);
    // Raise the kernel's dynamic shared-memory limit to every new largest size: epilogues
    // that reduce add static shared memory, so even tables under 48 KB can need it.
    static SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
    // Whole waves: past one wave of resident blocks (SMs x blocks per SM at this table size
    // and register count), a multiple of it, so that the last wave is not a partial one.
    static OccupancyCache occupancy;   // per instantiation
    const int occ = occupancy.get(kern, 256, smem, e.ctx->device);
    const int64_t ng = m->n_rows / G;
    const int64_t need = std::max<int64_t>(1, (ng + 255) / 256), wave = (int64_t)e.ctx->num_sms * occ;
    const int64_t cap = std::min<int64_t>(need, e.max_blocks);
    const int blocks = (int)(cap <= wave ? cap : cap / wave * wave);
    kern<<<blocks, 256, smem, e.stream>>>(m->pat_id.as<uint16_t>(), m->pat_start.as<uint32_t>(),
                                          static_cast<const PatRec<AT> *>(m->pat_rec.p), m->pat_base.as<uint32_t>(),
                                          m->pat_count, m->pat_entries, ng, g, op, e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}


template <class AT, class Gather, class Op, int G>
void launch_duvi_pattern_g(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op);

// The hex-structured stencil when the matrix has it; the general stencil (243 coefficients) in
// FP32 otherwise.  FP64 matrices without the hex structure keep the node patterns (grid_ok is
// not set for them); the fallback below only guards against a stale variant.
template <class AT, class Gather, class Op>
void launch_duvi_grid(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    if (m->grid_hex) launch_duvi_grid_h<AT, Gather, Op, true>(e, m, g, op);
    else if constexpr (sizeof(AT) == 4) launch_duvi_grid_h<AT, Gather, Op, false>(e, m, g, op);
    else launch_duvi_pattern_g<AT, Gather, Op, 3>(e, m, g, op);
}

template <class AT, class Gather, class Op, int G>
void launch_duvi_pattern_g(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    if (!m->pat_based) launch_duvi_pattern_gbs<AT, Gather, Op, G, false, false>(e, m, g, op);
    else if (G > 1 && m->pat_shift) launch_duvi_pattern_gbs<AT, Gather, Op, G, true, (G > 1)>(e, m, g, op);
    else launch_duvi_pattern_gbs<AT, Gather, Op, G, true, false>(e, m, g, op);
}

template <class AT, class Gather, class Op>
void launch_duvi_pattern(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    if (m->lanes_group == 3) launch_duvi_pattern_g<AT, Gather, Op, 3>(e, m, g, op);
    else if (m->lanes_group == 2) launch_duvi_pattern_g<AT, Gather, Op, 2>(e, m, g, op);
    else launch_duvi_pattern_g<AT, Gather, Op, 1>(e, m, g, op);
}

template <class VI, class AT, class Gather, class Op, int BATCH>
void launch_duvi_vi(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    constexpr int W = sizeof(VI) == 4 ? kDuviWarps32 : kDuviWarps;
    const size_t smem = duvi_smem_bytes<VI, AT>(W);
    auto kern = k_duvi<VI, AT, Gather, Op, W, BATCH>;
    static SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
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
    int blocks = (m->nbundles + W - 1) / W;
    if (blocks > e.max_blocks) blocks = e.max_blocks;
    if (blocks < 1) blocks = 1;
    kern<<<blocks, W * 32, smem, e.stream>>>(a, g, op, e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

template <int TPR, class AT, class Gather, class Op>
void launch_csr_tpr(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    const int gpb = kThreads / TPR;
    int blocks = (m->n_rows + gpb - 1) / gpb;
    if (blocks > e.max_blocks) blocks = e.max_blocks;
    if (blocks < 1) blocks = 1;
    k_csr<TPR, AT, AT, Gather, Op><<<blocks, kThreads, 0, e.stream>>>(
        m->rowptr.as<int32_t>(), m->col.as<int32_t>(), static_cast<const AT *>(m->val.p), m->n_rows, g, op, e.done,
        e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

// ---------------------------------------------------------------------------
// Matrix-free hexahedral operator (DV_FORMAT_HEX): y = K(E) x with K = sum_e f_e Ke on a
// structured grid of unit-cube trilinear hexahedra, f_e = scale * E_e per element, the
// nodes of the x = 0 face clamped (FemCantileverBase.cs:87-158, FemCantilever3D.cs:27-132).
//
// Nothing of the matrix is stored: a product reads the element factors (one value per
// element), x and writes y.  A block owns a tile of 32 x 8 free nodes of the xy plane and a
// run of zc planes and streams node planes of x and layers of element factors through
// shared memory (x planes double buffered, factor layers triple buffered because each layer
// is read in two consecutive steps).  At plane p every thread loads its 3 x 3 x 3
// neighbourhood of x once and forms, for the 8 elements around its node column, the
// element rows Ke(a, b) x_b of the corners b in plane p, scaled by the element factor, into
// the three nodes it accumulates (planes p + 1, p, p - 1).  Elements outside the mesh have
// factor 0 and clamped or outside nodes have x = 0, so face and edge nodes need no special
// case.  Ke enters through its 14 value classes (ke_class): equal entries share one
// register-resident value.  The sum order differs from the assembled operator's, so FP64
// products agree with the assembled matrix to rounding (not bit for bit).
// ---------------------------------------------------------------------------

// Value classes of the 24 x 24 unit-cube hexahedron stiffness (VTK corner order, 3 dofs per
// corner, entry (3 a + d, 3 b + c) at 24 (3 a + d) + 3 b + c): entries of one class are equal
// for every modulus and Poisson ratio (the element's symmetries; no entry is structurally
// zero).  Checked against Ke when an operator is created.
constexpr int kKeClasses = 14;
#define DV_KE_CLASS_TABLE \
    0,  1,  1,  2,  3,  3,  4,  5,  6,  7,  8,  9,  7,  9,  8,  4,  6,  5, 10, 11, 11, 12, 13, 13, \
    1,  0,  1,  8,  7,  9,  5,  4,  6,  3,  2,  3,  9,  7,  8, 13, 12, 13, 11, 10, 11,  6,  4,  5, \
    1,  1,  0,  8,  9,  7, 13, 13, 12,  9,  8,  7,  3,  3,  2,  5,  6,  4, 11, 11, 10,  6,  5,  4, \
    2,  8,  8,  0,  5,  5,  7,  3, 11,  4,  1, 13,  4, 13,  1,  7, 11,  3, 12,  6,  6, 10,  9,  9, \
    3,  7,  9,  5,  0,  1,  8,  2,  3,  1,  4,  6,  6, 12, 13, 11,  7,  8, 13,  4,  5,  9, 10, 11, \
    3,  9,  7,  5,  1,  0, 11,  8,  7,  6, 13, 12,  1,  6,  4,  8,  3,  2, 13,  5,  4,  9, 11, 10, \
    4,  5, 13,  7,  8, 11,  0,  1,  5,  2,  3,  8, 10, 11,  9, 12, 13,  6,  7,  9,  3,  4,  6,  1, \
    5,  4, 13,  3,  2,  8,  1,  0,  5,  8,  7, 11, 11, 10,  9,  6,  4,  1,  9,  7,  3, 13, 12,  6, \
    6,  6, 12, 11,  3,  7,  5,  5,  0,  3, 11,  7,  9,  9, 10, 13,  1,  4,  8,  8,  2,  1, 13,  4, \
    7,  3,  9,  4,  1,  6,  2,  8,  3,  0,  5,  1, 12,  6, 13, 10,  9, 11,  4, 13,  5,  7, 11,  8, \
    8,  2,  8,  1,  4, 13,  3,  7, 11,  5,  0,  5, 13,  4,  1,  9, 10,  9,  6, 12,  6, 11,  7,  3, \
    9,  3,  7, 13,  6, 12,  8, 11,  7,  1,  5,  0,  6,  1,  4, 11,  9, 10,  5, 13,  4,  3,  8,  2, \
    7,  9,  3,  4,  6,  1, 10, 11,  9, 12, 13,  6,  0,  1,  5,  2,  3,  8,  4,  5, 13,  7,  8, 11, \
    9,  7,  3, 13, 12,  6, 11, 10,  9,  6,  4,  1,  1,  0,  5,  8,  7, 11,  5,  4, 13,  3,  2,  8, \
    8,  8,  2,  1, 13,  4,  9,  9, 10, 13,  1,  4,  5,  5,  0,  3, 11,  7,  6,  6, 12, 11,  3,  7, \
    4, 13,  5,  7, 11,  8, 12,  6, 13, 10,  9, 11,  2,  8,  3,  0,  5,  1,  7,  3,  9,  4,  1,  6, \
    6, 12,  6, 11,  7,  3, 13,  4,  1,  9, 10,  9,  3,  7, 11,  5,  0,  5,  8,  2,  8,  1,  4, 13, \
    5, 13,  4,  3,  8,  2,  6,  1,  4, 11,  9, 10,  8, 11,  7,  1,  5,  0,  9,  3,  7, 13,  6, 12, \
    10, 11, 11, 12, 13, 13,  7,  9,  8,  4,  6,  5,  4,  5,  6,  7,  8,  9,  0,  1,  1,  2,  3,  3, \
    11, 10, 11,  6,  4,  5,  9,  7,  8, 13, 12, 13,  5,  4,  6,  3,  2,  3,  1,  0,  1,  8,  7,  9, \
    11, 11, 10,  6,  5,  4,  3,  3,  2,  5,  6,  4, 13, 13, 12,  9,  8,  7,  1,  1,  0,  8,  9,  7, \
    12,  6,  6, 10,  9,  9,  4, 13,  1,  7, 11,  3,  7,  3, 11,  4,  1, 13,  2,  8,  8,  0,  5,  5, \
    13,  4,  5,  9, 10, 11,  6, 12, 13, 11,  7,  8,  8,  2,  3,  1,  4,  6,  3,  7,  9,  5,  0,  1, \
    13,  5,  4,  9, 11, 10,  1,  6,  4,  8,  3,  2, 11,  8,  7,  6, 13, 12,  3,  9,  7,  5,  1,  0
// The same table in device and host memory: device code indexes the __device__ copy, which
// the compiler folds to constants after unrolling (a table local to a constexpr function
// would be rebuilt at every inlined call).
__device__ constexpr signed char kKeClassDev[576] = {DV_KE_CLASS_TABLE};
constexpr signed char kKeClassHost[576] = {DV_KE_CLASS_TABLE};
__host__ __device__ __forceinline__ constexpr int ke_class(int i) {
#ifdef __CUDA_ARCH__
    return kKeClassDev[i];
#else
    return kKeClassHost[i];
#endif
}

template <class AT>
struct KeCoef {
    AT cls[kKeClasses];
};

// One mesh of a (possibly batched) matrix-free operator: its element counts, the tiles it is
// streamed in, its first tile in the launch, and where its rows and element factors start.
struct HexMesh {
    int32_t ne0, ne1, ne2;     // elements per axis (free-node box: ne0 x (ne1 + 1) x (ne2 + 1))
    int32_t ntx, nty, zc;      // tiles per plane in x and y, planes per z run
    int32_t tile0, pad;        // first tile of this mesh
    int64_t row0, fac0;        // first row, first element factor
};

constexpr int kHexEX = kGridTX + 1, kHexEY = kGridTY + 1;   // element tile per layer (33 x 9)
constexpr int kHexLayer = kHexEX * kHexEY;                  // 297 factors
constexpr int kHexLayerLoads = (kHexLayer + 255) / 256;     // per thread (2)

// Contributions of one element layer to the two accumulated nodes of the thread's column that
// its elements contain.  L = 0: the layer above plane p (elements between p and p + 1; their
// corners in plane p are lower corners), which holds node p + 1 as an upper corner (UP, into
// au) and node p as a lower corner (DN, into ad).  L = 1: the layer below (p - 1 .. p; corners
// in plane p are upper corners), holding node p as an upper corner and node p - 1 as a lower
// one.  Each staged x value is scaled by the element factor once and applied to both nodes.
template <class AT, bool FUSED, int L, bool UP, bool DN>
__device__ __forceinline__ void hex_layer_terms(const AT (&xv)[27], const AT *__restrict__ el, int tx, int ty,
                                                const KeCoef<AT> &kc, AT (&au)[3], AT (&ad)[3]) {
    constexpr int vtk[8] = {0, 1, 3, 2, 4, 5, 7, 6};
    constexpr int bz = L == 0 ? 0 : 1;
#pragma unroll
    for (int eyo = 0; eyo < 2; ++eyo)
#pragma unroll
        for (int exo = 0; exo < 2; ++exo) {
            const AT f = el[(tx + exo) + kHexEX * (ty + eyo)];
            const int a_up = vtk[(1 - exo) + 2 * (1 - eyo) + 4];   // the node as the element's upper corner
            const int a_dn = vtk[(1 - exo) + 2 * (1 - eyo)];       // and as its lower corner
#pragma unroll
            for (int by = 0; by < 2; ++by)
#pragma unroll
                for (int bx = 0; bx < 2; ++bx) {
                    const int b = vtk[bx + 2 * by + 4 * bz];
                    const int dxs = exo + bx - 1, dys = eyo + by - 1;   // source node offset in the plane
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const AT w = f * xv[9 * (dys + 1) + 3 * (dxs + 1) + c];
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            if (UP) au[d] = madd_op<AT, FUSED>(au[d], kc.cls[ke_class(24 * (3 * a_up + d) + 3 * b + c)], w);
                            if (DN) ad[d] = madd_op<AT, FUSED>(ad[d], kc.cls[ke_class(24 * (3 * a_dn + d) + 3 * b + c)], w);
                        }
                    }
                }
        }
}

// One plane step: layer p feeds nodes p + 1 (DI) and p (DM), layer p - 1 nodes p (DM) and p - 1 (DF).
template <class AT, bool FUSED, bool DI, bool DM, bool DF>
__device__ __forceinline__ void hex_plane_step(const AT (&xv)[27], const AT *lay_up, const AT *lay_dn, int tx, int ty,
                                               const KeCoef<AT> &kc, AT (&a0)[3], AT (&a1)[3], AT (&a2)[3]) {
    if constexpr (DI || DM) hex_layer_terms<AT, FUSED, 0, DI, DM>(xv, lay_up, tx, ty, kc, a2, a1);
    if constexpr (DM || DF) hex_layer_terms<AT, FUSED, 1, DM, DF>(xv, lay_dn, tx, ty, kc, a1, a0);
}

template <class AT, class Gather, class Op>
__global__ void __launch_bounds__(256, sizeof(AT) == 8 ? 1 : 3)
    k_hex_elem(const HexMesh *__restrict__ meshes, int32_t nmesh, int32_t ntile, KeCoef<AT> kc,
               const AT *__restrict__ ef_all, Gather g, Op op, const int *__restrict__ done, double *partials,
               unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    extern __shared__ uint4 hex_smem[];
    constexpr bool FU = op_fused<Op>::value;
    using SS = StageSrc<Gather>;
    using ST = typename SS::ST;
    constexpr int SLOT = SS::N * kGridPlane;
    constexpr int NL = kGridStages + 1;              // factor layers: each is read in two consecutive steps
    ST *ring = reinterpret_cast<ST *>(hex_smem);     // kGridStages slots of node planes
    AT *layer = reinterpret_cast<AT *>(ring + kGridStages * SLOT);   // NL slots of element factors
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const StageSlots<1> slots;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
        int lo = 0, hi = nmesh - 1;   // the mesh of tile t: the last with tile0 <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (meshes[mid].tile0 <= t) lo = mid;
            else hi = mid - 1;
        }
        const HexMesh G = meshes[lo];
        const int32_t lx = G.ne0, ly = G.ne1 + 1, lz = G.ne2 + 1;
        const int64_t lxy = (int64_t)lx * ly;
        const int32_t plane_len = (int32_t)(3 * lxy), layer_len = G.ne0 * G.ne1;
        const AT *ef = ef_all + G.fac0;
        const int tl = t - G.tile0;
        const int txi = tl % G.ntx, tyi = (tl / G.ntx) % G.nty, tzi = tl / (G.ntx * G.nty);
        const int x0 = txi * kGridTX, y0 = tyi * kGridTY, z0 = tzi * G.zc, z1 = min(lz, z0 + G.zc);
        const int ix = x0 + tx, iy = y0 + ty;
        const bool inxy = ix < lx && iy < ly;
        const int64_t col_xy = G.row0 / 3 + ix + (int64_t)lx * iy;   // node index in the batch
        int32_t poff[kGridLoads], loff[kHexLayerLoads];
        slots.plane_offsets(x0, y0, lx, ly, poff);
#pragma unroll
        for (int j = 0; j < kHexLayerLoads; ++j) {   // element (ex, ey) of the layer tile (x index 0 is clamped)
            const int k = threadIdx.x + 256 * j;
            const int ex = x0 + k % kHexEX, ey = y0 - 1 + k / kHexEX;
            loff[j] = (k < kHexLayer && ex < G.ne0 && ey >= 0 && ey < G.ne1) ? ex + G.ne0 * ey : (k < kHexLayer ? -1 : -2);
        }
        // node plane z and element layer z (elements between planes z and z + 1), one copy group
        auto issue = [&](int z, int k) {
            const bool lin = z >= 0 && z < G.ne2;
            const int32_t lbase = lin ? z * layer_len : 0;
            AT *ld = layer + (k % NL) * kHexLayer;
#pragma unroll
            for (int j = 0; j < kHexLayerLoads; ++j)
                if (loff[j] > -2) {
                    const bool v = lin && loff[j] >= 0;
                    cp_async_zfill<sizeof(AT)>(ld + threadIdx.x + 256 * j, v ? ef + lbase + loff[j] : ef, v);
                }
            slots.template issue<SS>(g, ring + (k % kGridStages) * SLOT, poff, z, lz, plane_len, G.row0);   // commits
        };
#pragma unroll
        for (int q = 0; q < kGridStages - 1; ++q) {
            if (z0 - 1 + q <= z1) issue(z0 - 1 + q, q);
            else cp_async_commit();
        }
        AT a0[3], a1[3], a2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) a0[d] = a1[d] = a2[d] = AT(0);
        for (int p = z0 - 1, k = 0; p <= z1; ++p, ++k) {
            cp_async_wait<kGridStages - 2>();
            __syncthreads();
            if (p + kGridStages - 1 <= z1) issue(p + kGridStages - 1, k + kGridStages - 1);
            else cp_async_commit();
            const ST *pl = ring + (k % kGridStages) * SLOT;
            const AT *lay_up = layer + (k % NL) * kHexLayer;             // layer p
            const AT *lay_dn = layer + ((k + NL - 1) % NL) * kHexLayer;  // layer p - 1
            const bool di = p + 1 >= z0 && p + 1 < z1, dm = p >= z0 && p < z1, df = p - 1 >= z0 && p - 1 < z1;
            if (di) {
                const int32_t r = (int32_t)(3 * (col_xy + lxy * (p + 1)));
#pragma unroll
                for (int d = 0; d < 3; ++d) a2[d] = inxy ? op.init(r + d) : AT(0);
            }
            if (dm && inxy) touch_rows(op, (int32_t)(3 * (col_xy + lxy * p)));   // finished next step
            AT xv[27];
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                    for (int c = 0; c < 3; ++c) xv[9 * dy + 3 * dx + c] = SS::value(pl, ((ty + dy) * kGridPX + tx + dx) * 3 + c);
            if (di && dm && df) hex_plane_step<AT, FU, true, true, true>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            else if (di && dm) hex_plane_step<AT, FU, true, true, false>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            else if (dm && df) hex_plane_step<AT, FU, false, true, true>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            else if (di) hex_plane_step<AT, FU, true, false, false>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            else if (dm) hex_plane_step<AT, FU, false, true, false>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            else if (df) hex_plane_step<AT, FU, false, false, true>(xv, lay_up, lay_dn, tx, ty, kc, a0, a1, a2);
            if (df && inxy) {
                const int32_t r = (int32_t)(3 * (col_xy + lxy * (p - 1)));
#pragma unroll
                for (int d = 0; d < 3; ++d) op.row(r + d, a0[d], red);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                a0[d] = a1[d];
                a1[d] = a2[d];
            }
        }
        cp_async_wait<0>();
        __syncthreads();   // the next tile refills the rings
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

template <class AT, class Gather, class Op>
void launch_hex_elem(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    auto kern = k_hex_elem<AT, Gather, Op>;
    using SS = StageSrc<Gather>;
    const size_t smem = sizeof(typename SS::ST) * SS::N * kGridStages * (size_t)kGridPlane +
                        sizeof(AT) * (kGridStages + 1) * (size_t)kHexLayer;
    static SmemLimit limit;   // per instantiation and device
    limit.raise(kern, smem, e.ctx->device);
    KeCoef<AT> kc;
    for (int c = 0; c < kKeClasses; ++c) kc.cls[c] = (AT)m->hex_cls[c];
    const int blocks = (int)std::min<int64_t>(m->hex_ntile, e.max_blocks);
    kern<<<blocks, 256, smem, e.stream>>>(m->hex_meshes.as<HexMesh>(), m->hex_nmesh, m->hex_ntile, kc,
                                          static_cast<const AT *>(m->hex_factor.p), g, op, e.done, e.partials,
                                          e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

// ---------------------------------------------------------------------------
// Trilinear transfers without a matrix (DV_FORMAT_TRILINEAR): the factor-2 coarsening of an even
// structured grid (coarse nodes at the even fine nodes, x = 0 clamped), prolongation y_f = P x_c
// (a fine node takes 1 or 2 coarse nodes per axis, weights 1 or 1/2) and restriction y_c = P^T x_f
// (a coarse node takes the fine nodes at -1, 0, +1 per axis, weights 1/2, 1, 1/2).  Each row sums
// its columns in increasing order with the same multiply-add rounding as a stored matrix, so the
// products equal those of the assembled P and P^T (dv_hex_trilinear) bit for bit.
// ---------------------------------------------------------------------------
struct TriGeom {
    int32_t f0, f1, f2;   // fine element counts (even)
    __host__ __device__ int64_t nodes(bool restrict_) const {   // rows / 3
        return restrict_ ? (int64_t)(f0 / 2) * (f1 / 2 + 1) * (f2 / 2 + 1) : (int64_t)f0 * (f1 + 1) * (f2 + 1);
    }
};

// Calls f(first column, weight) for the coarse nodes of fine free node q (prolongation, a row of P)
// or the fine nodes of coarse free node q (restriction, a row of P^T), in increasing column order.
template <bool RESTRICT, class AT, class F>
__device__ __forceinline__ void tri_walk(const TriGeom &G, uint32_t q, F &&f) {
    // 32-bit index arithmetic throughout: rows and columns are below 2^31
    const uint32_t ny = G.f1 + 1, cx = G.f0 / 2, cy = G.f1 / 2 + 1;
    if constexpr (!RESTRICT) {
        const uint32_t t = q / (uint32_t)G.f0, Zy = t / ny;
        const int32_t X = (int32_t)(q - t * (uint32_t)G.f0) + 1, Y = (int32_t)(t - Zy * ny), Z = (int32_t)Zy;
        const int nx_ = (X & 1) ? 2 : 1, ny_ = (Y & 1) ? 2 : 1, nz_ = (Z & 1) ? 2 : 1;
        const AT w = (nx_ == 2 ? AT(0.5) : AT(1)) * (ny_ == 2 ? AT(0.5) : AT(1)) * (nz_ == 2 ? AT(0.5) : AT(1));
        for (int c = 0; c < nz_; ++c)
            for (int b = 0; b < ny_; ++b)
                for (int a = 0; a < nx_; ++a) {
                    const int32_t xc = X / 2 + a;
                    if (xc == 0) continue;   // clamped coarse node
                    f(3u * ((uint32_t)(xc - 1) + cx * ((uint32_t)(Y / 2 + b) + cy * (uint32_t)(Z / 2 + c))), w);
                }
    } else {
        const uint32_t t = q / cx, Zc_ = t / cy;
        const int32_t Xc = (int32_t)(q - t * cx) + 1, Yc = (int32_t)(t - Zc_ * cy), Zc = (int32_t)Zc_;
        for (int c = -1; c <= 1; ++c) {
            const int32_t Z = 2 * Zc + c;
            if (Z < 0 || Z > G.f2) continue;
            for (int b = -1; b <= 1; ++b) {
                const int32_t Y = 2 * Yc + b;
                if (Y < 0 || Y > G.f1) continue;
                for (int a = -1; a <= 1; ++a) {
                    const int32_t X = 2 * Xc + a;
                    if (X > G.f0) continue;   // X >= 1 always (Xc >= 1)
                    const AT w = (a ? AT(0.5) : AT(1)) * (b ? AT(0.5) : AT(1)) * (c ? AT(0.5) : AT(1));
                    f(3u * ((uint32_t)(X - 1) + (uint32_t)G.f0 * ((uint32_t)Y + ny * (uint32_t)Z)), w);
                }
            }
        }
    }
}

// One thread per node: its three rows (dof d takes column d of each node).
template <bool RESTRICT, class AT, class Gather, class Op>
__global__ void __launch_bounds__(256) k_tri(TriGeom G, Gather g, Op op, const int *__restrict__ done,
                                             double *partials, unsigned *ticket) {
    if (done && *(volatile const int *)done) return;
    constexpr bool FU = op_fused<Op>::value;
    double red[Op::NRED > 0 ? Op::NRED : 1];
#pragma unroll
    for (int i = 0; i < (Op::NRED > 0 ? Op::NRED : 1); ++i) red[i] = 0.0;
    const uint32_t nodes = (uint32_t)G.nodes(RESTRICT);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nodes; q += gridDim.x * blockDim.x) {
        const int32_t r0 = (int32_t)(3 * q);
        AT s[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) s[d] = op.init(r0 + d);
        tri_walk<RESTRICT, AT>(G, q, [&](uint32_t col, AT w) {
#pragma unroll
            for (int d = 0; d < 3; ++d) s[d] = madd_op<AT, FU>(s[d], w, g(col + d));
        });
#pragma unroll
        for (int d = 0; d < 3; ++d) op.row(r0 + d, s[d], red);
    }
    if constexpr (Op::NRED > 0) {
        double tot[Op::NRED];
        if (grid_reduce<Op::NRED, Op::MAXMASK>(red, partials, ticket, tot)) op.finish(tot);
    }
}

template <class AT, class Gather, class Op>
void launch_trilinear(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    const TriGeom G{m->tri_ne[0], m->tri_ne[1], m->tri_ne[2]};
    const int64_t nodes = m->n_rows / 3;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nodes + 255) / 256, e.max_blocks));
    if (m->tri_restrict) k_tri<true, AT, Gather, Op><<<blocks, 256, 0, e.stream>>>(G, g, op, e.done, e.partials, e.ticket);
    else k_tri<false, AT, Gather, Op><<<blocks, 256, 0, e.stream>>>(G, g, op, e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    e.ctx->count();
}

// Runs op over every row of m with the accumulator type AT (= value precision).
template <class AT, class Gather, class Op>
void launch_rows(const LaunchEnv &e, const dv_matrix *m, Gather g, Op op) {
    if (m->format == DV_FORMAT_HEX) {
        launch_hex_elem<AT>(e, m, g, op);
        return;
    }
    if (m->format == DV_FORMAT_TRILINEAR) {
        launch_trilinear<AT>(e, m, g, op);
        return;
    }
    if (m->format == DV_FORMAT_DUVI && m->duvi_variant == 3) {
        launch_duvi_grid<AT>(e, m, g, op);
        return;
    }
    if (m->format == DV_FORMAT_DUVI && m->duvi_variant == 2) {
        launch_duvi_pattern<AT>(e, m, g, op);
        return;
    }
    if (m->format == DV_FORMAT_DUVI && m->duvi_variant == 1) {
        if (m->vi_bits == 8) launch_duvi_lanes<uint8_t, AT>(e, m, g, op);
        else if (m->vi_bits == 16) launch_duvi_lanes<uint16_t, AT>(e, m, g, op);
        else launch_duvi_lanes<uint32_t, AT>(e, m, g, op);
        return;
    }
    if (m->format == DV_FORMAT_DUVI) {
        // batch width matched to the dominant block length (chosen at upload)
        if (m->duvi_batch == 9) {
            if (m->vi_bits == 8) launch_duvi_vi<uint8_t, AT, Gather, Op, 9>(e, m, g, op);
            else if (m->vi_bits == 16) launch_duvi_vi<uint16_t, AT, Gather, Op, 9>(e, m, g, op);
            else launch_duvi_vi<uint32_t, AT, Gather, Op, 9>(e, m, g, op);
        } else {
            if (m->vi_bits == 8) launch_duvi_vi<uint8_t, AT, Gather, Op, 4>(e, m, g, op);
            else if (m->vi_bits == 16) launch_duvi_vi<uint16_t, AT, Gather, Op, 4>(e, m, g, op);
            else launch_duvi_vi<uint32_t, AT, Gather, Op, 4>(e, m, g, op);
        }
        return;
    }
    switch (m->csr_tpr) {
        case 1: launch_csr_tpr<1, AT>(e, m, g, op); break;
        case 4: launch_csr_tpr<4, AT>(e, m, g, op); break;
        case 8: launch_csr_tpr<8, AT>(e, m, g, op); break;
        case 16: launch_csr_tpr<16, AT>(e, m, g, op); break;
        default: launch_csr_tpr<32, AT>(e, m, g, op); break;
    }
}

// ---------------------------------------------------------------------------
// vector kernels
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_scale(const T *__restrict__ w, const T *__restrict__ b, T *__restrict__ x, int32_t n,
                        const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = w[i] * b[i];
}
template <class T>
__global__ void k_copy(const T *__restrict__ a, T *__restrict__ b, int32_t n, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}
template <class T>
__global__ void k_fill(T *__restrict__ a, T v, int32_t n, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}
template <class A, class B>
__global__ void k_convert(const A *__restrict__ a, B *__restrict__ b, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (B)a[i];
}
// x += y
template <class T>
__global__ void k_axpy1(const T *__restrict__ y, T *__restrict__ x, int32_t n, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = x[i] + y[i];
}

// Dense y = Ainv b (coarse solve), one warp per row.
template <class T>
__global__ void k_dense_gemv(const T *__restrict__ a, const T *__restrict__ b, T *__restrict__ y, int32_t n,
                             const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const T *ar = a + (size_t)r * n;
        T s = 0;
        for (int32_t k = lane; k < n; k += 32) s += ar[k] * __ldg(b + k);
        s = warp_sum(s);
        if (lane == 0) y[r] = s;
    }
}

// Dense y = Ainv b with one block of 128 threads per row (the coarse solve of the MG-PCG V-cycle):
// every row's products split over 4 warps, two partial sums per thread, a shared-memory sum.
template <class T>
__global__ void __launch_bounds__(128) k_dense_gemv_rows(const T *__restrict__ a, const T *__restrict__ b,
                                                         T *__restrict__ y, int32_t n, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    __shared__ T part[4];
    for (int32_t r = blockIdx.x; r < n; r += gridDim.x) {
        const T *ar = a + (size_t)r * n;
        T s0 = 0, s1 = 0;
        int32_t k = threadIdx.x;
        for (; k + 128 < n; k += 256) {
            s0 += ar[k] * __ldg(b + k);
            s1 += ar[k + 128] * __ldg(b + k + 128);
        }
        if (k < n) s0 += ar[k] * __ldg(b + k);
        T v = warp_sum(s0 + s1);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) y[r] = (part[0] + part[1]) + (part[2] + part[3]);
        __syncthreads();
    }
}

}  // namespace dvk
