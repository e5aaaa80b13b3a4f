// Multi-right-hand-side multigrid-preconditioned flexible CG.
//
// k load cases solved together on the hierarchy of a dv_mgpcg solver.  All
// vectors are n x k row-interleaved blocks, every operator application is a
// block product (dv_block.cuh: the matrix is decoded once per k vectors) and
// every vector step is one fused pass over the block.  Each right-hand side
// keeps its own alpha, beta and relative stop test ||r_j|| <= tol ||b_j||
// (per-column deterministic reductions); a converged column is frozen
// (alpha_j = 0) while the others continue.  After the recurrence stops, the
// FP64 true residual of every column is verified and columns that drifted are
// restarted from it (iterative refinement), as in the single-vector driver.
// The reference solves several right-hand sides one after another
// (PcgSolver2.InverseSystemMatrixTimesOtherMatrix, PcgSolver2.cs:92-136).
#include "dv_block.cuh"
#include "dv_mgpcg.cuh"

#include <cmath>
#include <cstring>
#include <type_traits>

namespace {

constexpr int kMaxK = dvb::kMaxCols;
constexpr int kMaxRefinements = 4;

// per-column solver scalars (device)
struct ColScalars {
    double zr, zq, pq, alpha, beta, rr, bb;
    int converged, restart, pad0, pad1;
};

// ---------------------------------------------------------------------------
// epilogue of the outer product: q = A z + beta q, p = z + beta p, p.q per column
// ---------------------------------------------------------------------------
struct FinFcg {
    ColScalars *cs;
    __device__ void operator()(int j, const double *t) const {
        cs[j].pq = t[0];
        cs[j].alpha = cs[j].converged ? 0.0 : cs[j].zr / t[0];
    }
};
template <class ZT>
struct BEpiFcg {
    static constexpr int NC = 1;
    const ZT *z;
    double *p, *q;
    const ColScalars *cs;
    int ld;
    FinFcg fin;
    __device__ __forceinline__ void apply(int32_t i, int j, double s, double *red) const {
        const size_t o = (size_t)i * ld + j;
        const double bt = cs[j].beta;
        const double qi = s + bt * q[o];
        const double pi = (double)z[o] + bt * p[o];
        q[o] = qi;
        p[o] = pi;
        red[0] += pi * qi;
    }
};

// ---------------------------------------------------------------------------
// vector kernels over blocks: one warp per row, lanes over columns
// ---------------------------------------------------------------------------
struct FinRed {   // beta_j = -(z.q)/(p.q) (FCG(1)), 0 on a restart or a frozen column
    ColScalars *cs;
    __device__ void operator()(int j, const double *t) const {
        cs[j].zq = t[0];
        cs[j].zr = t[1];
        cs[j].beta = (cs[j].restart || cs[j].converged) ? 0.0 : -t[0] / cs[j].pq;
        cs[j].restart = 0;
    }
};
template <class ZT, int U>
__global__ void __launch_bounds__(dvb::kThreads) k_bfcg_red(const ZT *__restrict__ z, const double *__restrict__ q,
                                                            const double *__restrict__ r, int32_t n, int k,
                                                            ColScalars *cs, const int *__restrict__ done,
                                                            double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    double red[U][2];
#pragma unroll
    for (int u = 0; u < U; ++u) red[u][0] = red[u][1] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < k) {
                const size_t o = (size_t)i * k + j;
                const double zi = (double)z[o];
                red[u][0] += zi * q[o];
                red[u][1] += zi * r[o];
            }
        }
    dvb::col_reduce<2, U>(red, k, partials, ticket, FinRed{cs});
}

struct FinUpdate {   // ||r_j||^2 and the per-column stop test
    ColScalars *cs;
    double tol2;
    __device__ void operator()(int j, const double *t) const {
        cs[j].rr = t[0];
        if (!cs[j].converged && t[0] <= tol2 * cs[j].bb) cs[j].converged = 1;
    }
};
// x += alpha p; r -= alpha q; rlow = r (mixed); ||r||^2 per column
template <class RT, int U>
__global__ void __launch_bounds__(dvb::kThreads) k_bfcg_update(double *__restrict__ x, double *__restrict__ r,
                                                               RT *__restrict__ rlow, const double *__restrict__ p,
                                                               const double *__restrict__ q, int32_t n, int k,
                                                               ColScalars *cs, double tol2, const int *__restrict__ done,
                                                               double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    double red[U][1];
#pragma unroll
    for (int u = 0; u < U; ++u) red[u][0] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    double al[U];
#pragma unroll
    for (int u = 0; u < U; ++u) al[u] = (lane + 32 * u < k) ? cs[lane + 32 * u].alpha : 0.0;
    for (int32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < k) {
                const size_t o = (size_t)i * k + j;
                x[o] = x[o] + al[u] * p[o];
                const double ri = r[o] - al[u] * q[o];
                r[o] = ri;
                if (rlow) rlow[o] = (RT)ri;
                red[u][0] += ri * ri;
            }
        }
    dvb::col_reduce<1, U>(red, k, partials, ticket, FinUpdate{cs, tol2});
}

// stop decision after an update: every column converged, a NaN, or the iteration limit
__global__ void k_bfcg_stop(const ColScalars *cs, int k, dvk::SolverScalars *sc) {
    if (sc->done) return;
    int all = 1, bad = 0;
    for (int j = 0; j < k; ++j) {
        all &= cs[j].converged;
        bad |= isnan(cs[j].rr) ? 1 : 0;
    }
    sc->it += 1;
    if (all || bad || sc->it >= sc->max_it) {
        sc->done = 1;
        sc->converged = all && !bad;
        sc->failed = bad;
    }
}

// ||v_j||^2 per column into bb (slot 0; a zero load case is converged at once) or rr (slot 1)
struct FinNorm {
    ColScalars *cs;
    int slot;
    __device__ void operator()(int j, const double *t) const {
        if (slot == 0) {
            cs[j].bb = t[0];
            if (t[0] == 0.0) cs[j].converged = 1;   // x_j = 0 is exact
        } else {
            cs[j].rr = t[0];
        }
    }
};
template <int U>
__global__ void __launch_bounds__(dvb::kThreads) k_bnorm(const double *__restrict__ v, int32_t n, int k, ColScalars *cs,
                                                         int slot, double *partials, unsigned *ticket) {
    double red[U][1];
#pragma unroll
    for (int u = 0; u < U; ++u) red[u][0] = 0.0;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = lane + 32 * u;
            if (j < k) {
                const double a = v[(size_t)i * k + j];
                red[u][0] += a * a;
            }
        }
    dvb::col_reduce<1, U>(red, k, partials, ticket, FinNorm{cs, slot});
}

template <class T>
__global__ void k_bscale(const T *__restrict__ w, const T *__restrict__ b, T *__restrict__ x, int32_t n, int k,
                         const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    const size_t tot = (size_t)n * k;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x)
        x[q] = w[q / k] * b[q];
}

// Y = Ainv B on the coarsest level (dense inverse, nc x nc row-major, times
// nc x k): a block computes 8 rows x 32 columns, one output per thread, over
// 32-wide tiles of Ainv and B staged in shared memory.
template <class T>
__global__ void __launch_bounds__(256) k_bcoarse(const T *__restrict__ a, const T *__restrict__ b, T *__restrict__ y,
                                                 int32_t nc, int k, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    __shared__ T As[8][33];
    __shared__ T Bs[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int32_t row = blockIdx.x * 8 + ty;
    const int col = blockIdx.y * 32 + tx;
    T s = 0;
    for (int32_t c0 = 0; c0 < nc; c0 += 32) {
        As[ty][tx] = (row < nc && c0 + tx < nc) ? a[(size_t)row * nc + c0 + tx] : T(0);
        for (int q = ty; q < 32; q += 8) Bs[q][tx] = (c0 + q < nc && col < k) ? b[(size_t)(c0 + q) * k + col] : T(0);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 32; ++q) s += As[ty][q] * Bs[q][tx];
        __syncthreads();
    }
    if (row < nc && col < k) y[(size_t)row * k + col] = s;
}

// ---------------------------------------------------------------------------
// block V-cycle on the levels of a VCycle<T>
// ---------------------------------------------------------------------------
template <class T>
struct BlockLevels {
    std::vector<DevMem> x, t, r, b;   // per level, n_l x k
    DevMem bc, xc;                    // coarsest level
};

inline int vec_grid(dv_context *ctx, size_t tot) {
    return (int)std::max<size_t>(1, std::min<size_t>((tot + 255) / 256, (size_t)ctx->num_sms * 8));
}

template <class T>
T *block_vcycle(const LaunchEnv &e, VCycle<T> &vc, BlockLevels<T> &W, size_t l, const T *b, int k) {
    using namespace dvb;
    cudaStream_t s = e.stream;
    dv_context *ctx = vc.ctx;
    if (l == vc.lv.size()) {
        k_bcoarse<T><<<dim3((vc.nc + 7) / 8, (k + 31) / 32), 256, 0, s>>>(vc.ainv.template as<T>(), b,
                                                                          W.xc.template as<T>(), vc.nc, k, e.done);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        return W.xc.template as<T>();
    }
    VLevel<T> &L = vc.lv[l];
    T *x = W.x[l].template as<T>(), *t = W.t[l].template as<T>();
    const T *w = L.w.template as<T>();
    if (vc.nu == 1) {
        k_bscale<T><<<vec_grid(ctx, (size_t)L.n * k), 256, 0, s>>>(w, b, x, L.n, k, e.done);
        DV_CUDA(cudaGetLastError());
        ctx->count();
    } else {
        launch_bprod<T>(e, L.A.get(), k, BGatherWB<T>{w, b, k}, BEpiJacobiFromZero<T>{w, b, x, k, {}});
        for (int q = 2; q < vc.nu; ++q) {
            launch_bprod<T>(e, L.A.get(), k, BGatherVec<T, T>{x, k}, BEpiJacobi<T>{x, w, b, t, k, {}});
            std::swap(x, t);
        }
    }
    T *r = W.r[l].template as<T>();
    launch_bprod<T>(e, L.A.get(), k, BGatherVec<T, T>{x, k}, BEpiResid<T>{b, r, k, {}});
    T *bn = l + 1 < vc.lv.size() ? W.b[l + 1].template as<T>() : W.bc.template as<T>();
    launch_bprod<T>(e, L.R.get(), k, BGatherVec<T, T>{r, k}, BEpiSpmm<T>{bn, k, 1, {}});
    T *xn = block_vcycle<T>(e, vc, W, l + 1, bn, k);
    launch_bprod<T>(e, L.P.get(), k, BGatherVec<T, T>{xn, k}, BEpiSpmm<T>{x, k, 0, {}});
    for (int q = 0; q < vc.nu; ++q) {
        launch_bprod<T>(e, L.A.get(), k, BGatherVec<T, T>{x, k}, BEpiJacobi<T>{x, w, b, t, k, {}});
        std::swap(x, t);
    }
    return x;
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
template <class T>
struct MultiState {
    int k = 0;
    BlockLevels<T> W;
    DevMem B, X, R, Rlow, Pv, Q, cols;
    DevMem red;   // ticket + per-column partials
    std::unique_ptr<SolverWs> ws;
};

template <class T>
void multi_solve(dv_mgpcg *s, VCycle<T> &vc, MultiState<T> &M, int k, const double *dB, double *dX,
                 int32_t *col_converged, dv_stats *stats) {
    using namespace dvb;
    dv_context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int32_t n = s->n;
    const size_t nk = (size_t)n * k;
    constexpr bool kMixed = std::is_same<T, float>::value;
    if (M.k != k) {   // (re)size the block buffers
        M = MultiState<T>();
        M.k = k;
        for (auto &L : vc.lv) {
            const size_t b = sizeof(T) * (size_t)L.n * k;
            M.W.x.emplace_back(b);
            M.W.t.emplace_back(b);
            M.W.r.emplace_back(b);
            M.W.b.emplace_back(b);
        }
        M.W.bc.alloc(sizeof(T) * (size_t)vc.nc * k);
        M.W.xc.alloc(sizeof(T) * (size_t)vc.nc * k);
        M.B.alloc(8 * nk);
        M.X.alloc(8 * nk);
        M.R.alloc(8 * nk);
        M.Pv.alloc(8 * nk);
        M.Q.alloc(8 * nk);
        if (kMixed) M.Rlow.alloc(4 * nk);
        M.cols.alloc(sizeof(ColScalars) * (size_t)k);
        M.red.alloc(64 + sizeof(double) * 2 * (size_t)kMaxK * ctx->num_sms * dvb::kReduceBlocksPerSm);
        M.ws = std::make_unique<SolverWs>(ctx);
    }
    SolverWs &ws = *M.ws;
    ws.reset_graph();
    ws.warmed = false;
    dvk::SolverScalars &h = *ws.host_scal;
    std::memset(&h, 0, sizeof(h));
    h.max_it = s->cfg.max_iterations;
    h.tol2 = s->cfg.tol * s->cfg.tol;
    ws.push();
    LaunchEnv e0 = ws.env(false);
    e0.ticket = M.red.template as<unsigned>();
    e0.partials = reinterpret_cast<double *>(M.red.template as<char>() + 64);
    LaunchEnv ed = e0;
    ed.done = &ws.sc()->done;
    ColScalars *cs = M.cols.template as<ColScalars>();
    const int gw = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n * 32 + 255) / 256,
                                                                (int64_t)ctx->num_sms * dvb::kReduceBlocksPerSm));
    auto norms = [&](const double *v, int slot) {
        if (k <= 32) k_bnorm<1><<<gw, dvb::kThreads, 0, st>>>(v, n, k, cs, slot, e0.partials, e0.ticket);
        else if (k <= 64) k_bnorm<2><<<gw, dvb::kThreads, 0, st>>>(v, n, k, cs, slot, e0.partials, e0.ticket);
        else k_bnorm<4><<<gw, dvb::kThreads, 0, st>>>(v, n, k, cs, slot, e0.partials, e0.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
    };
    std::vector<ColScalars> hc(k);
    for (auto &c : hc) {
        std::memset(&c, 0, sizeof(c));
        c.restart = 1;
        c.pq = 1.0;
    }
    DV_CUDA(cudaMemcpyAsync(cs, hc.data(), sizeof(ColScalars) * k, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(M.B.p, dB, 8 * nk, cudaMemcpyDeviceToDevice, st));
    norms(M.B.template as<double>(), 0);
    DV_CUDA(cudaMemsetAsync(M.X.p, 0, 8 * nk, st));
    DV_CUDA(cudaMemcpyAsync(M.R.p, M.B.p, 8 * nk, cudaMemcpyDeviceToDevice, st));
    DV_CUDA(cudaMemsetAsync(M.Pv.p, 0, 8 * nk, st));
    DV_CUDA(cudaMemsetAsync(M.Q.p, 0, 8 * nk, st));
    T *rin = kMixed ? reinterpret_cast<T *>(M.Rlow.p) : reinterpret_cast<T *>(M.R.p);
    auto to_low = [&] {
        if (kMixed) {
            dvk::k_convert<double, float><<<vec_grid(ctx, nk), 256, 0, st>>>(M.R.template as<double>(),
                                                                             M.Rlow.template as<float>(), (int32_t)nk);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
    };
    to_low();
    const T *z = block_vcycle<T>(ed, vc, M.W, 0, rin, k);
    const int per = s->cfg.iterations_per_sync > 0 ? s->cfg.iterations_per_sync : 4;
    const double tol2 = h.tol2;
    const T *zfinal = z;
    double *Xd = M.X.template as<double>(), *Rd = M.R.template as<double>();
    double *Pd = M.Pv.template as<double>(), *Qd = M.Q.template as<double>();
    auto launch_red = [&](const T *zz) {
        if (k <= 32) k_bfcg_red<T, 1><<<gw, dvb::kThreads, 0, st>>>(zz, Qd, Rd, n, k, cs, ed.done, ed.partials, ed.ticket);
        else if (k <= 64) k_bfcg_red<T, 2><<<gw, dvb::kThreads, 0, st>>>(zz, Qd, Rd, n, k, cs, ed.done, ed.partials, ed.ticket);
        else k_bfcg_red<T, 4><<<gw, dvb::kThreads, 0, st>>>(zz, Qd, Rd, n, k, cs, ed.done, ed.partials, ed.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
    };
    auto launch_update = [&] {
        T *rl = kMixed ? reinterpret_cast<T *>(M.Rlow.p) : nullptr;
        if (k <= 32) k_bfcg_update<T, 1><<<gw, dvb::kThreads, 0, st>>>(Xd, Rd, rl, Pd, Qd, n, k, cs, tol2, ed.done, ed.partials, ed.ticket);
        else if (k <= 64) k_bfcg_update<T, 2><<<gw, dvb::kThreads, 0, st>>>(Xd, Rd, rl, Pd, Qd, n, k, cs, tol2, ed.done, ed.partials, ed.ticket);
        else k_bfcg_update<T, 4><<<gw, dvb::kThreads, 0, st>>>(Xd, Rd, rl, Pd, Qd, n, k, cs, tol2, ed.done, ed.partials, ed.ticket);
        DV_CUDA(cudaGetLastError());
        k_bfcg_stop<<<1, 1, 0, st>>>(cs, k, ws.sc());
        DV_CUDA(cudaGetLastError());
        ctx->count(2);
    };
    auto body = [&] {
        const T *zz = z;
        for (int it = 0; it < per; ++it) {
            launch_red(zz);
            launch_bprod<double, false>(ed, s->Aout.get(), k, BGatherVec<T, double>{zz, k},
                                 BEpiFcg<T>{zz, Pd, Qd, cs, k, FinFcg{cs}});
            launch_update();
            zz = block_vcycle<T>(ed, vc, M.W, 0, rin, k);
        }
        zfinal = zz;
    };
    auto true_residual = [&] {   // into Pd (free once the recurrence stopped)
        launch_bprod<double>(e0, s->Aout.get(), k, BGatherVec<double, double>{Xd, k},
                             BEpiResid<double>{M.B.template as<double>(), Pd, k, {}});
        norms(Pd, 1);
        DV_CUDA(cudaMemcpyAsync(hc.data(), cs, sizeof(ColScalars) * k, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    };
    int refinements = 0;
    bool verified = false;   // the last true_residual() was taken on the final iterate
    for (;;) {
        ws.run_chunk(body, s->cfg.use_graphs != 0, 0);
        DV_REQUIRE(zfinal == z, DV_ERR_ARG, "block V-cycle output buffer is not stable across iterations");
        ws.pull();
        if (!h.done) continue;
        if (!h.converged) break;
        // FP64 verification of every column's true residual; restart from it if any column drifted
        true_residual();
        int bad = 0;
        for (int j = 0; j < k; ++j)
            if (!(hc[j].rr <= tol2 * hc[j].bb)) {
                hc[j].converged = 0;
                ++bad;
            }
        if (bad == 0 || refinements >= kMaxRefinements || h.it >= h.max_it) {
            verified = true;
            break;
        }
        ++refinements;
        for (int j = 0; j < k; ++j) hc[j].restart = 1;   // every direction restarts from the new residual
        DV_CUDA(cudaMemcpyAsync(cs, hc.data(), sizeof(ColScalars) * k, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaMemcpyAsync(Rd, Pd, 8 * nk, cudaMemcpyDeviceToDevice, st));
        to_low();
        h.done = 0;
        h.converged = 0;
        ws.push();
        z = block_vcycle<T>(ed, vc, M.W, 0, rin, k);
    }
    // final FP64 true residual of every column (already taken when the loop ended on a verification)
    if (!verified) true_residual();
    DV_CUDA(cudaMemcpyAsync(dX, Xd, 8 * nk, cudaMemcpyDeviceToDevice, st));
    DV_CUDA(cudaStreamSynchronize(st));
    double worst = 0.0, worst_abs = 0.0;
    int all = 1;
    for (int j = 0; j < k; ++j) {
        const double rel = hc[j].bb > 0 ? std::sqrt(hc[j].rr / hc[j].bb) : std::sqrt(hc[j].rr);
        const int ok = hc[j].rr <= tol2 * hc[j].bb;
        all &= ok;
        if (col_converged) col_converged[j] = ok;
        worst = std::max(worst, rel);
        worst_abs = std::max(worst_abs, std::sqrt(hc[j].rr));
    }
    if (stats) {
        stats->iterations = h.it;
        stats->converged = all && !h.failed;
        stats->failed = h.failed;
        stats->reserved = 0;
        stats->residual_max = NAN;
        stats->residual_norm2 = worst_abs;
        stats->relative_residual = worst;
        stats->solve_ms = NAN;
    }
}

}  // namespace

struct MultiHolder {
    MultiState<float> f;
    MultiState<double> d;
};

void dv_mgpcg_multi_release(MultiHolder *m) { delete m; }

extern "C" DV_API int dv_mgpcg_solve_multi_device(dv_mgpcg *s, int32_t k, const double *d_B, double *d_X,
                                                  int32_t *converged_per_rhs, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "solver not created");
        DV_REQUIRE(d_B && d_X, DV_ERR_ARG, "null argument");
        DV_REQUIRE(k >= 1 && k <= kMaxK, DV_ERR_ARG, "number of right-hand sides must be 1..128");
        dv_ctx_check(s->ctx);
        if (!s->multi) s->multi = new MultiHolder();
        cudaStream_t st = s->ctx->stream;
        cudaEvent_t e0, e1;
        DV_CUDA(cudaEventCreate(&e0));
        DV_CUDA(cudaEventCreate(&e1));
        DV_CUDA(cudaEventRecord(e0, st));
        if (s->v32) multi_solve<float>(s, *s->v32, s->multi->f, k, d_B, d_X, converged_per_rhs, stats);
        else multi_solve<double>(s, *s->v64, s->multi->d, k, d_B, d_X, converged_per_rhs, stats);
        DV_CUDA(cudaEventRecord(e1, st));
        DV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (stats) stats->solve_ms = ms;
    });
}

extern "C" DV_API int dv_mgpcg_solve_multi(dv_mgpcg *s, int32_t k, const double *B, double *X,
                                           int32_t *converged_per_rhs, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "solver not created");
        DV_REQUIRE(B && X, DV_ERR_ARG, "null argument");
        DV_REQUIRE(k >= 1 && k <= kMaxK, DV_ERR_ARG, "number of right-hand sides must be 1..128");
        dv_ctx_check(s->ctx);
        const size_t bytes = 8 * (size_t)s->n * k;
        DevMem dB(bytes), dX(bytes);
        cudaStream_t st = s->ctx->stream;
        DV_CUDA(cudaMemcpyAsync(dB.p, B, bytes, cudaMemcpyHostToDevice, st));
        const int rc = dv_mgpcg_solve_multi_device(s, k, dB.as<double>(), dX.as<double>(), converged_per_rhs, stats);
        DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
        DV_CUDA(cudaMemcpyAsync(X, dX.p, bytes, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    });
}
