// Solvers of libduvigpu.so: Jacobi PCG (OpenCLCsrPcgSolver semantics) and the
// multigrid-preconditioned flexible CG in FP64 or mixed precision.
//
// Every solver keeps its scalars (alpha, beta, dot products, stop flags) in
// device memory: no kernel result goes through the host inside an iteration.
// A chunk of iterations is captured once into a CUDA graph and replayed; each
// kernel returns at entry once the device-side `done` flag is set, so the
// iterate is frozen at the iteration that met the stop test and the host reads
// the flag once per chunk.
#include "dv_kernels.cuh"
#include "dv_solvers.cuh"
#include "dv_mgpcg.cuh"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <type_traits>

using namespace dvk;

dvk::LaunchEnv dv_default_env(dv_context *ctx);

// ---------------------------------------------------------------------------
// shared pieces
// ---------------------------------------------------------------------------
SolverWs::SolverWs(dv_context *c) : ctx(c) {
    red.alloc(sizeof(double) * kMaxRed * c->num_sms * 16 + 64);
    scal.alloc(sizeof(SolverScalars));
    DV_CUDA(cudaMallocHost(&host_scal, sizeof(SolverScalars)));
}
SolverWs::~SolverWs() {
    for (auto &c : chunks) cudaGraphExecDestroy(c.exec);
    if (host_scal) cudaFreeHost(host_scal);
}
LaunchEnv SolverWs::env(bool with_done) const {
    LaunchEnv e;
    e.ctx = ctx;
    e.stream = ctx->stream;
    e.done = with_done ? &sc()->done : nullptr;
    e.ticket = reinterpret_cast<unsigned *>(red.as<char>());
    e.partials = reinterpret_cast<double *>(red.as<char>() + 64);
    e.max_blocks = ctx->num_sms * 16;
    return e;
}
void SolverWs::pull() {
    DV_CUDA(cudaMemcpyAsync(host_scal, scal.p, sizeof(SolverScalars), cudaMemcpyDeviceToHost, ctx->stream));
    DV_CUDA(cudaStreamSynchronize(ctx->stream));
}
void SolverWs::push() {
    DV_CUDA(cudaMemcpyAsync(scal.p, host_scal, sizeof(SolverScalars), cudaMemcpyHostToDevice, ctx->stream));
}
// Runs `body` once eagerly (first call: sets kernel attributes, validates) and
// afterwards through the graph of the same launches captured for `key`.
void SolverWs::run_chunk(const std::function<void()> &body, bool use_graph, int key) {
    cudaStream_t s = ctx->stream;
    if (!use_graph || !warmed) {
        body();
        warmed = true;
        return;
    }
    const Chunk *c = nullptr;
    for (const auto &g : chunks)
        if (g.key == key) c = &g;
    if (!c) {
        cudaGraph_t g;
        int64_t launches = 0;
        {
            CountScope capture(ctx, dv_context::kCountCapture);   // counted when the graph runs
            const int64_t before = ctx->captured_launches;
            DV_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                body();
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                throw;
            }
            DV_CUDA(cudaStreamEndCapture(s, &g));
            launches = ctx->captured_launches - before;
        }
        cudaGraphExec_t exec;
        const cudaError_t err = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        DV_CUDA(err);
        chunks.push_back({key, exec, launches});
        c = &chunks.back();
    }
    DV_CUDA(cudaGraphLaunch(c->exec, s));
    graph_launches = c->launches;
    ctx->count(c->launches);
}


// ---------------------------------------------------------------------------
// vector kernels with reductions
// ---------------------------------------------------------------------------
// z = M r; p = z; rz = r.z   (initialize0 + dot, CsrCG.cl:165-176)
__global__ void k_pcg_init(const double *__restrict__ M, const double *__restrict__ r, double *__restrict__ z,
                           double *__restrict__ p, int32_t n, SolverScalars *sc, double *partials, unsigned *ticket) {
    double red[1] = {0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double zi = M[i] * r[i];
        z[i] = zi;
        p[i] = zi;
        red[0] += r[i] * zi;
    }
    double tot[1];
    if (grid_reduce<1, 0>(red, partials, ticket, tot)) sc->rz = tot[0];
}

// x += a p; r -= a Ap; z = M r; convergence flags; r.z (update_x_r_z_check_r,
// CsrCG.cl:257-277, then dot_finalize_and_calc_b, :289-301).  The stop test is the
// reference's max |r_i| <= tol, or with rel_l2 ||r||_2 <= tol ||b||_2 (sc->bb = ||b||^2).
__global__ void k_pcg_update(const double *__restrict__ M, const double *__restrict__ ap, const double *__restrict__ p,
                             double *__restrict__ x, double *__restrict__ r, double *__restrict__ z, int32_t n,
                             double tol, int rel_l2, SolverScalars *sc, const int *__restrict__ done,
                             double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    const double a = sc->alpha;
    double red[4] = {0.0, 0.0, 0.0, 0.0};   // max|r|, failed flag, r.z, r.r
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = x[i] + a * p[i];
        double ri = r[i] - a * ap[i];
        r[i] = ri;
        double zi = M[i] * ri;
        z[i] = zi;
        double c = fabs(ri);
        if (isnan(ri) || c > 1e50) red[1] = 1.0;
        else red[0] = fmax(red[0], c);
        red[2] += ri * zi;
        red[3] += ri * ri;
    }
    double t[4];
    if (grid_reduce<4, 0b0011>(red, partials, ticket, t)) {
        bool failed = t[1] != 0.0;
        bool converged = !failed && (rel_l2 ? t[3] <= tol * tol * sc->bb : t[0] <= tol);
        sc->res_max = t[0];
        sc->res_norm2 = sqrt(t[3]);
        sc->converged = converged;
        sc->failed = failed;
        if (converged || failed || sc->it > sc->max_it) {
            sc->done = 1;
        } else {
            sc->beta = t[2] / sc->rz;
            sc->rz = t[2];
            sc->it += 1;
        }
    }
}

// p = z + beta p (update_p, CsrCG.cl:311-320)
__global__ void k_pcg_p(const double *__restrict__ z, double *__restrict__ p, int32_t n, const SolverScalars *sc,
                        const int *__restrict__ done) {
    if (*(volatile const int *)done) return;
    const double b = sc->beta;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = z[i] + b * p[i];
}

// Flexible CG: beta = -(z.q)/(p.q) (FCG(1) orthogonalisation), z.r for alpha.
template <class ZT>
__global__ void k_fcg_red(const ZT *__restrict__ z, const double *__restrict__ q, const double *__restrict__ r,
                          int32_t n, SolverScalars *sc, const int *__restrict__ done, double *partials,
                          unsigned *ticket) {
    if (*(volatile const int *)done) return;
    double red[2] = {0.0, 0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double zi = (double)z[i];
        red[0] += zi * q[i];
        red[1] += zi * r[i];
    }
    double t[2];
    if (grid_reduce<2, 0>(red, partials, ticket, t)) {
        sc->zq = t[0];
        sc->zr = t[1];
        sc->beta = sc->restart ? 0.0 : -t[0] / sc->pq;
        sc->restart = 0;
    }
}

// x += alpha p; r -= alpha q; r32 = r and wb = w0 .* r32 (mixed: the V-cycle's first sweep gathers
// wb); ||r||^2 and the stop decision.
template <class RT>
__global__ void k_fcg_update(double *__restrict__ x, double *__restrict__ r, RT *__restrict__ rlow,
                             const RT *__restrict__ w0, RT *__restrict__ wb, const double *__restrict__ p,
                             const double *__restrict__ q, int32_t n, SolverScalars *sc, const int *__restrict__ done,
                             double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    const double a = sc->alpha;
    double red[1] = {0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = x[i] + a * p[i];
        double ri = r[i] - a * q[i];
        r[i] = ri;
        if (rlow) {
            const RT rl = (RT)ri;
            rlow[i] = rl;
            if (wb) wb[i] = w0[i] * rl;
        }
        red[0] += ri * ri;
    }
    double t[1];
    if (grid_reduce<1, 0>(red, partials, ticket, t)) {
        sc->rr = t[0];
        sc->it += 1;
        if (!(t[0] <= sc->tol2 * sc->bb) && !isnan(t[0])) {
            if (sc->it >= sc->max_it) sc->done = 1;
        } else {
            sc->done = 1;
            sc->converged = !isnan(t[0]);
            sc->failed = isnan(t[0]);
        }
    }
}

// ||v||^2 into sc->bb (slot 0) or sc->rr (slot 1)
__global__ void k_norm2(const double *__restrict__ v, int32_t n, SolverScalars *sc, int slot, double *partials,
                        unsigned *ticket) {
    double red[1] = {0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) red[0] += v[i] * v[i];
    double t[1];
    if (grid_reduce<1, 0>(red, partials, ticket, t)) {
        if (slot == 0) sc->bb = t[0];
        else sc->rr = t[0];
    }
}

// Power-method step for the spectral radius of D^-1 A: y = D^-1 A x (epilogue) and ||y||^2.
template <class T>
struct OpPower {
    static constexpr int NRED = 1;
    static constexpr unsigned MAXMASK = 0;
    const double *__restrict__ diag;
    T *__restrict__ y;
    SolverScalars *sc;
    __device__ __forceinline__ T init(int32_t) const { return T(0); }
    __device__ __forceinline__ void row(int32_t i, T s, double *red) const {
        T v = (T)((double)s / diag[i]);
        y[i] = v;
        red[0] += (double)v * (double)v;
    }
    __device__ void finish(const double *t) const { sc->rr = t[0]; }
};
template <class T>
__global__ void k_power_normalize(const T *__restrict__ y, T *__restrict__ x, int32_t n, const SolverScalars *sc) {
    const double s = 1.0 / sqrt(sc->rr);
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = (T)(y[i] * s);
}

template <class T>
__global__ void k_make_weights(const double *__restrict__ diag, T *__restrict__ w, double omega, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w[i] = (T)(omega / diag[i]);
}

// Spectral radius estimate of D^-1 A by the power method (iters steps from a
// fixed pseudo-random start); returns ||D^-1 A x|| for the last unit x.
double dv_power_estimate(dv_context *ctx, SolverWs &ws, dv_matrix *A, int iters) {
    int32_t n = A->n_rows;
    const bool f64 = A->precision == DV_F64;
    const size_t vs = f64 ? 8 : 4;
    DevMem x(vs * n), y(vs * n);
    std::vector<double> h(n);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    double nn = 0;
    for (int32_t i = 0; i < n; ++i) {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        h[i] = 0.5 + (double)(st >> 11) * (1.0 / 9007199254740992.0);
        nn += h[i] * h[i];
    }
    for (auto &v : h) v /= std::sqrt(nn);
    cudaStream_t s = ctx->stream;
    if (f64) DV_CUDA(cudaMemcpyAsync(x.p, h.data(), 8 * n, cudaMemcpyHostToDevice, s));
    else {
        std::vector<float> f(h.begin(), h.end());
        DV_CUDA(cudaMemcpyAsync(x.p, f.data(), 4 * n, cudaMemcpyHostToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
    }
    LaunchEnv e = ws.env(false);
    for (int it = 0; it < iters; ++it) {
        if (f64) {
            OpPower<double> op{A->diag.as<double>(), y.as<double>(), ws.sc()};
            launch_rows<double>(e, A, GatherVec<double, double>{x.as<double>()}, op);
            k_power_normalize<double><<<grid_for(ctx, n), kThreads, 0, s>>>(y.as<double>(), x.as<double>(), n, ws.sc());
        } else {
            OpPower<float> op{A->diag.as<double>(), y.as<float>(), ws.sc()};
            launch_rows<float>(e, A, GatherVec<float, float>{x.as<float>()}, op);
            k_power_normalize<float><<<grid_for(ctx, n), kThreads, 0, s>>>(y.as<float>(), x.as<float>(), n, ws.sc());
        }
        DV_CUDA(cudaGetLastError());
        ctx->count();
    }
    ws.pull();
    return std::sqrt(ws.host_scal->rr);
}

// ---------------------------------------------------------------------------
// Jacobi PCG (OpenCLCsrPcgSolver)
// ---------------------------------------------------------------------------
struct dv_pcg {
    dv_context *ctx = nullptr;
    std::unique_ptr<dv_matrix> A;
    std::unique_ptr<SolverWs> ws;
    int32_t n = 0, max_iter = 0;
    double tol = 0;
    int32_t tol_kind = DV_TOL_ABS_MAX;
    DevMem M, b, x, r, z, p, ap;
};

extern "C" DV_API int dv_pcg_set_tolerance_kind(dv_pcg *s, int32_t tol_kind) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "You must call Initialize(model) first");
        DV_REQUIRE(tol_kind == DV_TOL_ABS_MAX || tol_kind == DV_TOL_REL_L2, DV_ERR_ARG,
                   "tol_kind must be DV_TOL_ABS_MAX or DV_TOL_REL_L2");
        s->tol_kind = tol_kind;
    });
}

extern "C" DV_API int dv_pcg_create(dv_context *ctx, const dv_csr_host *A, int32_t format, int32_t max_iter,
                                    double tol, dv_pcg **out) {
    return dv_guard([&] {
        DV_REQUIRE(A && out, DV_ERR_ARG, "null argument");
        DV_REQUIRE(A->n_rows == A->n_cols, DV_ERR_ARG, "matrix must be square");
        DV_REQUIRE(max_iter >= 0 && tol >= 0, DV_ERR_ARG, "bad iteration limit or tolerance");
        auto s = std::make_unique<dv_pcg>();
        s->ctx = ctx;
        s->A.reset(dv_matrix_build(ctx, *A, format, DV_F64, 0, 1e-10));
        s->ws = std::make_unique<SolverWs>(ctx);
        s->n = A->n_rows;
        s->max_iter = max_iter;
        s->tol = tol;
        std::vector<double> minv(s->n);
        for (int32_t i = 0; i < s->n; ++i) {
            DV_REQUIRE(s->A->host_diag[i] != 0.0, DV_ERR_SINGULAR, "zero diagonal entry");
            minv[i] = 1 / s->A->host_diag[i];   // JacobiPreconditioner (GeometricMultigridSolver.cs:128-134)
        }
        size_t nb = 8 * (size_t)s->n;
        s->M.alloc(nb);
        DV_CUDA(cudaMemcpyAsync(s->M.p, minv.data(), nb, cudaMemcpyHostToDevice, ctx->stream));
        s->b.alloc(nb); s->x.alloc(nb); s->r.alloc(nb); s->z.alloc(nb); s->p.alloc(nb); s->ap.alloc(nb);
        DV_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = s.release();
    });
}

extern "C" DV_API int dv_pcg_solve(dv_pcg *s, const double *b, const double *x0, double *xout, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "You must call Initialize(model) first");
        DV_REQUIRE(b && xout, DV_ERR_ARG, "null argument");
        dv_context *ctx = s->ctx;
        dv_ctx_check(ctx);
        cudaStream_t st = ctx->stream;
        const int32_t n = s->n;
        const size_t nb = 8 * (size_t)n;
        cudaEvent_t e0, e1;
        DV_CUDA(cudaEventCreate(&e0));
        DV_CUDA(cudaEventCreate(&e1));
        DV_CUDA(cudaMemcpyAsync(s->b.p, b, nb, cudaMemcpyHostToDevice, st));
        if (x0) DV_CUDA(cudaMemcpyAsync(s->x.p, x0, nb, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaEventRecord(e0, st));
        LaunchEnv e = s->ws->env(false);
        SolverScalars &h = *s->ws->host_scal;
        std::memset(&h, 0, sizeof(h));
        h.max_it = s->max_iter;
        s->ws->push();
        if (x0) {   // initialize: r = b - A x0 (CsrCG.cl:191-211)
            OpResid<double> op{{}, s->b.as<double>(), s->r.as<double>()};
            launch_rows<double>(e, s->A.get(), GatherVec<double, double>{s->x.as<double>()}, op);
        } else {
            DV_CUDA(cudaMemsetAsync(s->x.p, 0, nb, st));
            DV_CUDA(cudaMemcpyAsync(s->r.p, s->b.p, nb, cudaMemcpyDeviceToDevice, st));
        }
        const int g = grid_for(ctx, n);
        k_norm2<<<g, kThreads, 0, st>>>(s->b.as<double>(), n, s->ws->sc(), 0, e.partials, e.ticket);   // ||b||^2
        DV_CUDA(cudaGetLastError());
        k_pcg_init<<<g, kThreads, 0, st>>>(s->M.as<double>(), s->r.as<double>(), s->z.as<double>(), s->p.as<double>(), n,
                                          s->ws->sc(), e.partials, e.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count(2);
        const int rel_l2 = s->tol_kind == DV_TOL_REL_L2;
        LaunchEnv ed = s->ws->env(true);
        const int chunk = 16;
        auto body = [&] {
            for (int k = 0; k < chunk; ++k) {
                OpPcgAp op{s->p.as<double>(), s->ap.as<double>(), s->ws->sc()};
                launch_rows<double>(ed, s->A.get(), GatherVec<double, double>{s->p.as<double>()}, op);
                k_pcg_update<<<g, kThreads, 0, st>>>(s->M.as<double>(), s->ap.as<double>(), s->p.as<double>(),
                                                     s->x.as<double>(), s->r.as<double>(), s->z.as<double>(), n, s->tol,
                                                     rel_l2, s->ws->sc(), ed.done, ed.partials, ed.ticket);
                DV_CUDA(cudaGetLastError());
                k_pcg_p<<<g, kThreads, 0, st>>>(s->z.as<double>(), s->p.as<double>(), n, s->ws->sc(), ed.done);
                DV_CUDA(cudaGetLastError());
                ctx->count(2);
            }
        };
        for (;;) {
            s->ws->run_chunk(body, true, 3 * chunk);
            s->ws->pull();
            if (h.done) break;
        }
        DV_CUDA(cudaEventRecord(e1, st));
        DV_CUDA(cudaMemcpyAsync(xout, s->x.p, nb, cudaMemcpyDeviceToHost, st));
        // relative residual of the returned x, recomputed in FP64: z = b - A x, ||z||^2
        {
            OpResid<double> op{{}, s->b.as<double>(), s->z.as<double>()};
            launch_rows<double>(e, s->A.get(), GatherVec<double, double>{s->x.as<double>()}, op);
            k_norm2<<<g, kThreads, 0, st>>>(s->z.as<double>(), n, s->ws->sc(), 1, e.partials, e.ticket);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
        s->ws->pull();
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (stats) {
            stats->iterations = h.it;
            stats->converged = h.converged;
            stats->failed = h.failed;
            stats->reserved = 0;
            stats->residual_max = h.res_max;
            stats->residual_norm2 = h.res_norm2;
            stats->relative_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : (h.rr > 0 ? INFINITY : 0.0);
            stats->solve_ms = ms;
        }
    });
}

extern "C" DV_API int dv_pcg_destroy(dv_pcg *s) {
    return dv_guard([&] {
        if (!s) return;
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
        delete s;
    });
}

// ---------------------------------------------------------------------------
// multigrid-preconditioned flexible CG
// ---------------------------------------------------------------------------
// prebuilt: operators of levels 0 .. L-2 already on the device (A[l] then only gives the shape).
// tri: element counts of levels 0 .. L-2 (all even); the transfers are then the matrix-free
// trilinear ones (P[l] only gives the shape).
template <class T>
static std::unique_ptr<VCycle<T>> build_vcycle(dv_context *ctx, SolverWs &ws, int32_t L, const dv_csr_host *A,
                                               const dv_csr_host *P, const dv_mgpcg_config &cfg,
                                               std::vector<double> &omega_eff, const DuviHost *encoded0,
                                               std::vector<std::unique_ptr<dv_matrix>> *prebuilt = nullptr,
                                               const std::array<int32_t, 3> *tri = nullptr) {
    auto v = std::make_unique<VCycle<T>>();
    v->ctx = ctx;
    v->nu = cfg.nu;
    v->smoother = cfg.smoother;
    const int prec = sizeof(T) == 8 ? DV_F64 : DV_F32;
    cudaStream_t s = ctx->stream;
    v->lv.resize(L - 1);
    for (int32_t l = 0; l < L - 1; ++l) {
        VLevel<T> &lv = v->lv[l];
        DV_REQUIRE(A[l].n_rows == A[l].n_cols, DV_ERR_ARG, "level operators must be square");
        DV_REQUIRE(P[l].n_rows == A[l].n_rows && P[l].n_cols == A[l + 1].n_rows, DV_ERR_ARG,
                   "prolongation shape does not match the levels");
        lv.n = A[l].n_rows;
        if (prebuilt) lv.A = std::move((*prebuilt)[l]);
        else lv.A.reset(dv_matrix_build(ctx, A[l], cfg.format, prec, 0, 1e-10, l == 0 ? encoded0 : nullptr));
        DV_REQUIRE(lv.A->n_rows == lv.n && lv.A->precision == prec, DV_ERR_ARG, "level operator does not match");
        if (tri) {
            lv.P.reset(dv_trilinear_build(ctx, tri[l].data(), 0, prec));
            lv.R.reset(dv_trilinear_build(ctx, tri[l].data(), 1, prec));
            DV_REQUIRE(lv.P->n_rows == P[l].n_rows && lv.P->n_cols == P[l].n_cols, DV_ERR_ARG, "transfer shape mismatch");
        } else {
            lv.P.reset(dv_matrix_build(ctx, P[l], cfg.format, prec, 0, 1e-10));
            std::vector<int32_t> rp, ci;
            std::vector<double> va;
            dv_csr_transpose(P[l], rp, ci, va);
            dv_csr_host rt{P[l].n_cols, P[l].n_rows, rp.data(), ci.data(), va.data()};
            lv.R.reset(dv_matrix_build(ctx, rt, cfg.format, prec, 0, 1e-10));
        }
        for (double d : lv.A->host_diag) DV_REQUIRE(d != 0.0, DV_ERR_SINGULAR, "zero diagonal entry");
        double om = cfg.omega;
        if (cfg.omega_mode == DV_OMEGA_SPECTRAL) {
            double lam = dv_power_estimate(ctx, ws, lv.A.get(), 40);
            om = cfg.omega * 2.0 / (1.1 * lam);
        }
        omega_eff.push_back(om);
        const size_t vs = sizeof(T) * (size_t)lv.n;
        lv.w.alloc(vs); lv.b.alloc(vs); lv.x.alloc(vs); lv.t.alloc(vs); lv.r.alloc(vs);
        if (l > 0 && cfg.smoother == DV_SMOOTHER_JACOBI && cfg.nu > 1) lv.wb.alloc(vs);
        if (cfg.smoother != DV_SMOOTHER_JACOBI) gs_build_order(A[l], cfg.smoother == DV_SMOOTHER_GS_LEX, s, lv.gs);
        k_make_weights<T><<<grid_for(ctx, lv.n), kThreads, 0, s>>>(lv.A->diag.template as<double>(), lv.w.template as<T>(), om, lv.n);
        DV_CUDA(cudaGetLastError());
    }
    const dv_csr_host &Ac = A[L - 1];
    v->nc = Ac.n_rows;
    DV_REQUIRE(v->nc <= 16384, DV_ERR_UNSUPPORTED, "coarsest level above 16384 dofs (dense inverse)");
    std::vector<double> dense((size_t)v->nc * v->nc, 0.0);
    for (int32_t r = 0; r < v->nc; ++r)
        for (int32_t k = Ac.rowptr[r]; k < Ac.rowptr[r + 1]; ++k) dense[(size_t)r * v->nc + Ac.col[k]] = Ac.val[k];
    DV_REQUIRE(dv_dense_inverse(v->nc, dense, 1e-300), DV_ERR_SINGULAR, "coarse matrix is singular");
    v->ainv.alloc(sizeof(T) * dense.size());
    if (sizeof(T) == 8) {
        DV_CUDA(cudaMemcpyAsync(v->ainv.p, dense.data(), 8 * dense.size(), cudaMemcpyHostToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<float> f(dense.begin(), dense.end());
        DV_CUDA(cudaMemcpyAsync(v->ainv.p, f.data(), 4 * f.size(), cudaMemcpyHostToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
    }
    v->bc.alloc(sizeof(T) * v->nc);
    v->xc.alloc(sizeof(T) * v->nc);
    return v;
}

static void check_mgpcg_config(const dv_mgpcg_config *cfg) {
    DV_REQUIRE(cfg->precision == DV_F64 || cfg->precision == DV_MIXED, DV_ERR_ARG, "precision must be DV_F64 or DV_MIXED");
    DV_REQUIRE(cfg->nu >= 1 && cfg->max_iterations >= 1 && cfg->tol > 0, DV_ERR_ARG, "bad smoothing or stop parameters");
    DV_REQUIRE(cfg->smoother >= DV_SMOOTHER_JACOBI && cfg->smoother <= DV_SMOOTHER_GS_COLOR, DV_ERR_ARG, "unknown smoother");
}

extern "C" DV_API int dv_mgpcg_create_hex(dv_context *ctx, const int32_t *ne, double E, double nu, int32_t coarse_ne,
                                          const dv_mgpcg_config *cfg, dv_mgpcg **out) {
    return dv_guard([&] {
        DV_REQUIRE(ne && cfg && out, DV_ERR_ARG, "null argument");
        check_mgpcg_config(cfg);
        DV_REQUIRE(cfg->format == DV_FORMAT_DUVI && cfg->outer_format == DV_FORMAT_DUVI && cfg->smoother == DV_SMOOTHER_JACOBI,
                   DV_ERR_UNSUPPORTED, "the device-built hierarchy is DuVi with the Jacobi smoother");
        DV_REQUIRE(coarse_ne >= 1, DV_ERR_ARG, "coarse_ne must be positive");
        dv_ctx_check(ctx);
        cudaStream_t st = ctx->stream;
        // levels of the factor-2 re-discretised hierarchy: element size 2^l, K_l = 2^l sum_e E Ke
        std::vector<std::array<int32_t, 3>> dims;
        std::array<int32_t, 3> cur = {ne[0], ne[1], ne[2]};
        for (;;) {
            dims.push_back(cur);
            if (std::min(cur[0], std::min(cur[1], cur[2])) <= coarse_ne || (cur[0] | cur[1] | cur[2]) & 1) break;
            for (auto &c : cur) c /= 2;
        }
        const int32_t L = (int32_t)dims.size();
        DV_REQUIRE(L >= 2, DV_ERR_ARG, "mesh too small for a hierarchy");
        auto s = std::make_unique<dv_mgpcg>();
        s->ctx = ctx;
        s->cfg = *cfg;
        s->ws = std::make_unique<SolverWs>(ctx);
        const int prec = cfg->precision == DV_MIXED ? DV_F32 : DV_F64;
        std::vector<std::unique_ptr<dv_matrix>> prebuilt;
        std::vector<dv_csr_host> Ash(L);
        struct Owned { std::vector<int32_t> rp, ci; std::vector<double> va; };
        std::vector<Owned> hostP(L - 1);   // empty with matrix-free transfers
        std::vector<std::array<int32_t, 2>> pshape(L - 1);
        Owned coarse;
        const char *mft = getenv("DV_MATRIX_FREE_TRANSFERS");
        const bool free_transfers = !(mft && mft[0] == '0');
        double scale = 1.0;
        for (int32_t l = 0; l < L; ++l, scale *= 2.0) {
            int32_t nr;
            int64_t nnz;
            int rc = dv_hex_csr_size(dims[l].data(), &nr, &nnz);
            DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
            if (l == L - 1) {   // the coarsest level: host CSR for the dense inverse
                coarse.rp.resize((size_t)nr + 1);
                coarse.ci.resize(nnz);
                coarse.va.resize(nnz);
                rc = dv_hex_assemble(dims[l].data(), nullptr, scale, E, nu, coarse.rp.data(), coarse.ci.data(),
                                     coarse.va.data());
                DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
                Ash[l] = dv_csr_host{nr, nr, coarse.rp.data(), coarse.ci.data(), coarse.va.data()};
                break;
            }
            DevMem rp(4 * ((size_t)nr + 1)), ci(4 * (size_t)nnz), va(8 * (size_t)nnz);
            rc = dv_hex_assemble_device(ctx, dims[l].data(), nullptr, scale, E, nu, rp.as<int32_t>(), ci.as<int32_t>(),
                                        va.as<double>());
            DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
            auto build = [&](int p) {
                auto m = std::make_unique<dv_matrix>();
                m->ctx = ctx;
                m->n_rows = m->n_cols = nr;
                m->nnz = nnz;
                m->format = DV_FORMAT_DUVI;
                m->precision = p;
                dv_duvi_from_device_csr(m.get(), rp.as<int32_t>(), ci.as<int32_t>(), va.as<double>(), 0, 1e-10);
                dv_autotune(m.get());
                return m;
            };
            if (l == 0) s->Aout = build(DV_F64);
            prebuilt.push_back(build(prec));
            Ash[l] = dv_csr_host{nr, nr, nullptr, nullptr, nullptr};
            // trilinear prolongation to this level from the next: matrix-free, or host CSR when
            // DV_MATRIX_FREE_TRANSFERS=0 (A/B comparisons)
            int32_t pr, pc;
            int64_t pnnz;
            rc = dv_hex_trilinear_size(dims[l].data(), &pr, &pc, &pnnz);
            DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
            pshape[l] = {pr, pc};
            if (free_transfers) continue;
            Owned &P = hostP[l];
            P.rp.resize((size_t)pr + 1);
            P.ci.resize(pnnz);
            P.va.resize(pnnz);
            rc = dv_hex_trilinear(dims[l].data(), P.rp.data(), P.ci.data(), P.va.data());
            DV_REQUIRE(rc == DV_OK, rc, dv_last_error());
        }
        std::vector<dv_csr_host> Psh(L - 1);
        for (int32_t l = 0; l < L - 1; ++l)
            Psh[l] = dv_csr_host{pshape[l][0], pshape[l][1], hostP[l].rp.data(), hostP[l].ci.data(), hostP[l].va.data()};
        s->n = Ash[0].n_rows;
        const std::array<int32_t, 3> *tri = free_transfers ? dims.data() : nullptr;
        if (cfg->precision == DV_MIXED)
            s->v32 = build_vcycle<float>(ctx, *s->ws, L, Ash.data(), Psh.data(), *cfg, s->omega_eff, nullptr, &prebuilt, tri);
        else
            s->v64 = build_vcycle<double>(ctx, *s->ws, L, Ash.data(), Psh.data(), *cfg, s->omega_eff, nullptr, &prebuilt, tri);
        const size_t nb = 8 * (size_t)s->n;
        s->b.alloc(nb); s->x.alloc(nb); s->r.alloc(nb); s->p.alloc(nb); s->q.alloc(nb);
        if (cfg->precision == DV_MIXED) {
            s->r32.alloc(4 * (size_t)s->n);
            s->wb32.alloc(4 * (size_t)s->n);
        }
        DV_CUDA(cudaStreamSynchronize(st));
        *out = s.release();
    });
}

extern "C" DV_API int dv_mgpcg_create(dv_context *ctx, int32_t L, const dv_csr_host *A, const dv_csr_host *P,
                                      const dv_mgpcg_config *cfg, dv_mgpcg **out) {
    return dv_guard([&] {
        DV_REQUIRE(A && cfg && out && L >= 1 && (L == 1 || P), DV_ERR_ARG, "null argument");
        check_mgpcg_config(cfg);
        DV_REQUIRE(L >= 2, DV_ERR_ARG, "need at least two levels");
        dv_ctx_check(ctx);
        auto s = std::make_unique<dv_mgpcg>();
        s->ctx = ctx;
        s->cfg = *cfg;
        s->ws = std::make_unique<SolverWs>(ctx);
        s->n = A[0].n_rows;
        // the finest operator is encoded once for the outer matrix and the V-cycle's level 0
        const bool outer_duvi = cfg->outer_format == DV_FORMAT_DUVI, inner_duvi = cfg->format == DV_FORMAT_DUVI;
        DuviHost h0;
        if (outer_duvi && inner_duvi) {
            dv_check_csr(A[0]);
            dv_encode_duvi(A[0], 1e-10, 0, h0);
        }
        const DuviHost *shared = outer_duvi && inner_duvi ? &h0 : nullptr;
        s->Aout.reset(dv_matrix_build(ctx, A[0], cfg->outer_format, DV_F64, 0, 1e-10, shared));
        if (cfg->precision == DV_MIXED) s->v32 = build_vcycle<float>(ctx, *s->ws, L, A, P, *cfg, s->omega_eff, shared);
        else s->v64 = build_vcycle<double>(ctx, *s->ws, L, A, P, *cfg, s->omega_eff, shared);
        const size_t nb = 8 * (size_t)s->n;
        s->b.alloc(nb); s->x.alloc(nb); s->r.alloc(nb); s->p.alloc(nb); s->q.alloc(nb);
        if (cfg->precision == DV_MIXED) {
            s->r32.alloc(4 * (size_t)s->n);
            s->wb32.alloc(4 * (size_t)s->n);
        }
        DV_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = s.release();
    });
}

// One outer iteration of FCG(1) given z (the V-cycle output of the previous
// step), then the V-cycle for the next z.  Returns the buffer of the new z.
template <class T>
static const T *fcg_step(dv_mgpcg *s, const LaunchEnv &e, VCycle<T> &vc, const T *z, T *rin) {
    cudaStream_t st = e.stream;
    const int g = grid_for(s->ctx, s->n);
    if (!vc.fused_red()) {   // otherwise z.q, z.r and beta came with the V-cycle's last sweep
        k_fcg_red<T><<<g, kThreads, 0, st>>>(z, s->q.as<double>(), s->r.as<double>(), s->n, s->ws->sc(), e.done,
                                             e.partials, e.ticket);
        DV_CUDA(cudaGetLastError());
        s->ctx->count();
    }
    OpFcg<T> op{z, s->p.as<double>(), s->q.as<double>(), s->ws->sc(), 0.0};
    launch_rows<double>(e, s->Aout.get(), GatherVec<T, double>{z}, op);
    const bool mixed = std::is_same<T, float>::value;
    T *rl = mixed ? reinterpret_cast<T *>(s->r32.p) : nullptr;
    const bool form_wb = mixed && vc.nu > 1 && vc.smoother == DV_SMOOTHER_JACOBI && !vc.lv.empty();
    T *wb = form_wb ? reinterpret_cast<T *>(s->wb32.p) : nullptr;
    const T *w0 = wb ? vc.lv[0].w.template as<T>() : nullptr;
    k_fcg_update<T><<<g, kThreads, 0, st>>>(s->x.as<double>(), s->r.as<double>(), rl, w0, wb, s->p.as<double>(),
                                            s->q.as<double>(), s->n, s->ws->sc(), e.done, e.partials, e.ticket);
    DV_CUDA(cudaGetLastError());
    s->ctx->count();
    vc.wb0 = wb;
    const T *zn = vc.run(e, rin);
    vc.wb0 = nullptr;   // the first cycle and the restarts form w .* b in the sweep
    return zn;
}

// Outer iterations to run before the next host read of the stop flag: as many as the
// convergence rate of the last chunk (||r||^2 from r2_0 at iteration it_0 to r2 at it)
// needs to bring ||r||^2 down to target, at least 1 and at most per.  Iterations after
// convergence only launch kernels that return at once; a short last chunk avoids most
// of them.  Without a measurable rate the chunk stays at per.
static int next_chunk_length(int per, int it_0, double r2_0, int it, double r2, double target) {
    if (per <= 1 || it <= it_0 || !(r2 > 0.0) || !(r2_0 > r2) || !(target > 0.0)) return per;
    const double log_rate = std::log(r2 / r2_0) / (double)(it - it_0);   // < 0
    const double need = std::log(target / r2) / log_rate;                // iterations left
    if (!(need > 0.0)) return 1;
    return (int)std::min<double>((double)per, std::max(1.0, std::ceil(need)));
}

template <class T>
static void mgpcg_solve_impl(dv_mgpcg *s, VCycle<T> &vc, dv_stats *stats) {
    dv_context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int32_t n = s->n;
    const size_t nb = 8 * (size_t)n;
    SolverWs &ws = *s->ws;
    SolverScalars &h = *ws.host_scal;
    LaunchEnv e0 = ws.env(false), ed = ws.env(true);
    cudaEvent_t ev0, ev1;
    DV_CUDA(cudaEventCreate(&ev0));
    DV_CUDA(cudaEventCreate(&ev1));
    DV_CUDA(cudaEventRecord(ev0, st));
    std::memset(&h, 0, sizeof(h));
    h.max_it = s->cfg.max_iterations;
    h.tol2 = s->cfg.tol * s->cfg.tol;
    h.restart = 1;
    h.pq = 1.0;
    ws.push();
    const int g = grid_for(ctx, n);
    vc.fuse_q = s->q.as<double>();
    vc.fuse_r = s->r.as<double>();
    vc.fuse_sc = ws.sc();
    k_norm2<<<g, kThreads, 0, st>>>(s->b.as<double>(), n, ws.sc(), 0, e0.partials, e0.ticket);
    DV_CUDA(cudaGetLastError());
    ctx->count();
    DV_CUDA(cudaMemsetAsync(s->x.p, 0, nb, st));
    DV_CUDA(cudaMemcpyAsync(s->r.p, s->b.p, nb, cudaMemcpyDeviceToDevice, st));
    T *rin;
    if (std::is_same<T, float>::value) {
        k_convert<double, float><<<g, kThreads, 0, st>>>(s->b.as<double>(), s->r32.as<float>(), n);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        rin = reinterpret_cast<T *>(s->r32.p);
    } else {
        rin = reinterpret_cast<T *>(s->r.p);
    }
    const T *z = vc.run(ed, rin);
    const int per = s->cfg.iterations_per_sync > 0 ? s->cfg.iterations_per_sync : 4;
    int len = per;   // outer iterations in the next chunk (one captured graph per length)
    const T *zfinal = z;
    auto body = [&] {
        const T *zz = z;
        for (int k = 0; k < len; ++k) zz = fcg_step<T>(s, ed, vc, zz, rin);
        zfinal = zz;
    };
    int refinements = 0;
    bool verified = false;   // p = b - A x and rr already hold the final x's true residual
    int it0 = 0;             // iteration count and ||r||^2 at the previous host read
    double rr0 = -1.0;       // (-1: ||b||^2, known on the host after the first read)
    for (;;) {
        ws.run_chunk(body, s->cfg.use_graphs != 0, len);
        DV_REQUIRE(zfinal == z, DV_ERR_ARG, "V-cycle output buffer is not stable across iterations");
        ws.pull();
        if (!h.done) {
            len = next_chunk_length(per, it0, rr0 < 0 ? h.bb : rr0, h.it, h.rr, h.tol2 * h.bb);
            it0 = h.it;
            rr0 = h.rr;
            continue;
        }
        if (!h.converged) break;
        // FP64 verification of the true residual; restart from it if the
        // recurrence drifted (iterative refinement).
        OpResid<double> orr{{}, s->b.as<double>(), s->p.as<double>()};
        launch_rows<double>(e0, s->Aout.get(), GatherVec<double, double>{s->x.as<double>()}, orr);
        k_norm2<<<g, kThreads, 0, st>>>(s->p.as<double>(), n, ws.sc(), 1, e0.partials, e0.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        ws.pull();
        if (h.rr <= h.tol2 * h.bb || refinements >= 4 || h.it >= h.max_it) {
            verified = true;
            break;
        }
        ++refinements;
        DV_CUDA(cudaMemcpyAsync(s->r.p, s->p.p, nb, cudaMemcpyDeviceToDevice, st));
        if (std::is_same<T, float>::value) {
            k_convert<double, float><<<g, kThreads, 0, st>>>(s->r.as<double>(), s->r32.as<float>(), n);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
        h.done = 0;
        h.converged = 0;
        h.restart = 1;
        ws.push();
        z = vc.run(ed, rin);
        len = per;
        it0 = h.it;
        rr0 = h.rr;
    }
    if (!verified) {   // final true residual (FP64) of a solve that stopped without converging
        OpResid<double> orr{{}, s->b.as<double>(), s->p.as<double>()};
        launch_rows<double>(e0, s->Aout.get(), GatherVec<double, double>{s->x.as<double>()}, orr);
        k_norm2<<<g, kThreads, 0, st>>>(s->p.as<double>(), n, ws.sc(), 1, e0.partials, e0.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
    }
    DV_CUDA(cudaEventRecord(ev1, st));
    ws.pull();
    // converged: the recurrence stopped below the tolerance and the true residual confirms it
    h.converged = h.converged && h.rr <= h.tol2 * h.bb;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (stats) {
        stats->iterations = h.it;
        stats->converged = h.converged;
        stats->failed = h.failed;
        stats->reserved = 0;
        stats->residual_max = NAN;
        stats->residual_norm2 = std::sqrt(h.rr);
        stats->relative_residual = std::sqrt(h.rr / h.bb);
        stats->solve_ms = ms;
    }
}

extern "C" DV_API int dv_mgpcg_solve_device(dv_mgpcg *s, const double *d_b, double *d_x, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "solver not created");
        DV_REQUIRE(d_b && d_x, DV_ERR_ARG, "null argument");
        dv_ctx_check(s->ctx);
        cudaStream_t st = s->ctx->stream;
        const size_t nb = 8 * (size_t)s->n;
        DV_CUDA(cudaMemcpyAsync(s->b.p, d_b, nb, cudaMemcpyDeviceToDevice, st));
        if (s->v32) mgpcg_solve_impl<float>(s, *s->v32, stats);
        else mgpcg_solve_impl<double>(s, *s->v64, stats);
        DV_CUDA(cudaMemcpyAsync(d_x, s->x.p, nb, cudaMemcpyDeviceToDevice, st));
        DV_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" DV_API int dv_mgpcg_solve(dv_mgpcg *s, const double *b, double *x, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(s != nullptr, DV_ERR_NOT_INITIALIZED, "solver not created");
        DV_REQUIRE(b && x, DV_ERR_ARG, "null argument");
        dv_ctx_check(s->ctx);
        cudaStream_t st = s->ctx->stream;
        const size_t nb = 8 * (size_t)s->n;
        DV_CUDA(cudaMemcpyAsync(s->b.p, b, nb, cudaMemcpyHostToDevice, st));
        if (s->v32) mgpcg_solve_impl<float>(s, *s->v32, stats);
        else mgpcg_solve_impl<double>(s, *s->v64, stats);
        DV_CUDA(cudaMemcpyAsync(x, s->x.p, nb, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" DV_API int dv_mgpcg_omega(const dv_mgpcg *s, int32_t level, double *omega) {
    return dv_guard([&] {
        DV_REQUIRE(s && omega, DV_ERR_ARG, "null argument");
        DV_REQUIRE(level >= 0 && level < (int32_t)s->omega_eff.size(), DV_ERR_ARG, "level out of range");
        *omega = s->omega_eff[level];
    });
}

extern "C" DV_API int dv_mgpcg_destroy(dv_mgpcg *s) {
    return dv_guard([&] {
        if (!s) return;
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
        delete s;
    });
}
