// Stationary geometric multigrid with the semantics of the reference solvers:
// OpenCL{Csr,DuVi}GeometricMultigridSolver.Solve (OpenCLCsrGeometricMultigridSolver.cs:334-536)
// and the CPU GeometricMultigridSolver.Solve (GeometricMultigridSolver.cs:297-418).
//
// The level path comes from MakePath (GeometricMultigridSolver.cs:178-201).
// Smoothers: weighted Jacobi x += w D^-1 (b - A x) exactly as the CPU code;
// forward Gauss-Seidel in the reference's own row order (level-scheduled, one
// launch per dependency level, each row summed sequentially in column order so
// the result equals the CPU sweep of GaussSeidelIterationCsrDuVi.cs:22-50 bit
// for bit); and multicolor Gauss-Seidel (node blocks of equal color updated in
// parallel, rows inside a block in order) as the fast ordering.  The OpenCL
// "gauss_seidel_iteration" kernel (CsrGeometricMultigrid.cl:207-225) updates x
// in place while other work-items read it, which is a data race; it is not
// reproduced.
#include "dv_gs.cuh"
#include "dv_kernels.cuh"
#include "dv_solvers.cuh"

#include <algorithm>
#include <cmath>

using namespace dvk;

double dv_power_bound_ref(const dv_csr_host &a, const std::vector<double> &inv_diag);

static int grid_n(dv_context *ctx, int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, ctx->num_sms * 8));
}

// ||v||^2 into sc->bb (slot 0) or sc->rr (slot 1), for the exit check of a solve.
static __global__ void k_gmg_norm2(const double *__restrict__ v, int32_t n, SolverScalars *sc, int slot,
                                   double *partials, unsigned *ticket) {
    double red[1] = {0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) red[0] += v[i] * v[i];
    double t[1];
    if (grid_reduce<1, 0>(red, partials, ticket, t)) {
        if (slot == 0) sc->bb = t[0];
        else sc->rr = t[0];
    }
}

// ---------------------------------------------------------------------------
// solver object
// ---------------------------------------------------------------------------
struct GLevel {
    std::unique_ptr<dv_matrix> A, R, P;
    DevMem D, b, x, t, r;
    int32_t n = 0;
    double omega = 1.0;
    GsOrder gs;   // Gauss-Seidel row groups (forward-sweep levels or colors)
};

struct dv_gmg {
    dv_context *ctx = nullptr;
    std::unique_ptr<SolverWs> ws;
    int smoother = DV_SMOOTHER_JACOBI;
    int32_t max_cycles = 0;
    double tol = 0;
    std::vector<uint8_t> path;
    int32_t total_levels = 0, first_level = 0;
    std::vector<int32_t> level_iter;
    std::vector<GLevel> lv;   // total_levels - 1 smoothed levels
    int32_t nc = 0;
    DevMem ainv, bc, xc;
    int cycles_per_sync = 16;
};

static void smooth(dv_gmg *g, const LaunchEnv &e, GLevel &L, int sweeps) {
    cudaStream_t s = e.stream;
    dv_context *ctx = g->ctx;
    if (g->smoother == DV_SMOOTHER_JACOBI) {
        double *x = L.x.as<double>(), *t = L.t.as<double>();
        for (int k = 0; k < sweeps; ++k) {
            OpJacobi<double> op{{}, x, L.D.as<double>(), L.b.as<double>(), t};
            launch_rows<double>(e, L.A.get(), GatherVec<double, double>{x}, op);
            std::swap(x, t);
        }
        if (x != L.x.as<double>()) {
            k_copy<double><<<grid_n(ctx, L.n), kThreads, 0, s>>>(x, L.x.as<double>(), L.n, e.done);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
        return;
    }
    for (int k = 0; k < sweeps; ++k) gs_sweep<double>(e, L.A.get(), L.gs, L.b.as<double>(), L.x.as<double>());
}

// One V-cycle pass over the path (the step loop of Solve).
static void cycle(dv_gmg *g, const LaunchEnv &e) {
    cudaStream_t s = e.stream;
    dv_context *ctx = g->ctx;
    const int32_t TL = g->total_levels;
    int32_t cur = g->first_level;
    for (size_t step = 0; step < g->path.size(); ++step) {
        if (cur == TL - 1) {
            GLevel &Lp = g->lv[cur - 1];
            k_dense_gemv<double><<<std::max(1, std::min(g->nc / 8 + 1, ctx->num_sms * 8)), kThreads, 0, s>>>(
                g->ainv.as<double>(), g->bc.as<double>(), g->xc.as<double>(), g->nc, e.done);
            DV_CUDA(cudaGetLastError());
            ctx->count();
            OpSpmv<double, double> op;
            op.y = Lp.x.as<double>();
            op.clear = 0;
            launch_rows<double>(e, Lp.P.get(), GatherVec<double, double>{g->xc.as<double>()}, op);
        } else {
            GLevel &L = g->lv[cur];
            int32_t li = g->level_iter[std::min<size_t>(cur, g->level_iter.size() - 1)];
            smooth(g, e, L, li);
            if (g->path[step]) {
                if (cur == 0) {
                    OpResidCheck op{L.b.as<double>(), L.r.as<double>(), g->ws->sc(), g->tol};
                    launch_rows<double>(e, L.A.get(), GatherVec<double, double>{L.x.as<double>()}, op);
                } else {
                    OpResid<double> op{{}, L.b.as<double>(), L.r.as<double>()};
                    launch_rows<double>(e, L.A.get(), GatherVec<double, double>{L.x.as<double>()}, op);
                }
                double *bn = cur + 1 < TL - 1 ? g->lv[cur + 1].b.as<double>() : g->bc.as<double>();
                OpSpmv<double, double> op;
                op.y = bn;
                op.clear = 1;
                launch_rows<double>(e, L.R.get(), GatherVec<double, double>{L.r.as<double>()}, op);
                if (cur < TL - 2) {
                    GLevel &N = g->lv[cur + 1];
                    k_fill<double><<<grid_n(ctx, N.n), kThreads, 0, s>>>(N.x.as<double>(), 0.0, N.n, e.done);
                    DV_CUDA(cudaGetLastError());
                    ctx->count();
                }
            } else {
                GLevel &Lp = g->lv[cur - 1];
                OpSpmv<double, double> op;
                op.y = Lp.x.as<double>();
                op.clear = 0;
                launch_rows<double>(e, Lp.P.get(), GatherVec<double, double>{L.x.as<double>()}, op);
            }
        }
        cur += g->path[step] ? 1 : -1;
    }
}

// MakePath (GeometricMultigridSolver.cs:178-201).
static void make_path(std::vector<uint8_t> &ld, int32_t &total, int32_t &first) {
    int32_t cur = 0;
    total = 1;
    first = 0;
    for (uint8_t d : ld) {
        if (d) { ++cur; if (cur == total) ++total; }
        else if (cur == 0) { ++first; ++total; }
        else --cur;
    }
    if (cur > first) ld.insert(ld.end(), cur - first, 0);
    else if (cur < first) ld.insert(ld.end(), first - cur, 1);
}

extern "C" DV_API int dv_gmg_create(dv_context *ctx, int32_t n_levels, const dv_csr_host *A, const dv_csr_host *R,
                                    const dv_csr_host *P, const dv_gmg_config *cfg, dv_gmg **out) {
    return dv_guard([&] {
        DV_REQUIRE(A && cfg && out && n_levels >= 2 && R && P, DV_ERR_ARG, "null argument or fewer than two levels");
        DV_REQUIRE(cfg->smoother >= DV_SMOOTHER_JACOBI && cfg->smoother <= DV_SMOOTHER_GS_COLOR, DV_ERR_ARG, "unknown smoother");
        DV_REQUIRE(cfg->max_cycles >= 0 && cfg->tol >= 0, DV_ERR_ARG, "bad stop parameters");
        dv_ctx_check(ctx);
        auto g = std::make_unique<dv_gmg>();
        g->ctx = ctx;
        g->ws = std::make_unique<SolverWs>(ctx);
        g->smoother = cfg->smoother;
        g->max_cycles = cfg->max_cycles;
        g->tol = cfg->tol;
        g->cycles_per_sync = cfg->cycles_per_sync > 0 ? cfg->cycles_per_sync : 16;
        if (cfg->n_steps > 0) {
            DV_REQUIRE(cfg->level_down != nullptr, DV_ERR_ARG, "null level_down");
            g->path.assign(cfg->level_down, cfg->level_down + cfg->n_steps);
        } else {
            g->path.assign(n_levels - 1, 1);
            g->path.insert(g->path.end(), n_levels - 1, 0);
        }
        make_path(g->path, g->total_levels, g->first_level);
        DV_REQUIRE(g->first_level == 0, DV_ERR_UNSUPPORTED, "firstLevel != 0 is not implemented");
        DV_REQUIRE(g->total_levels <= n_levels, DV_ERR_ARG, "path needs more levels than supplied");
        if (cfg->n_level_iterations > 0) {
            DV_REQUIRE(cfg->level_iterations != nullptr, DV_ERR_ARG, "null level_iterations");
            g->level_iter.assign(cfg->level_iterations, cfg->level_iterations + cfg->n_level_iterations);
        } else {
            g->level_iter.assign(1, 4);
        }
        for (int32_t v : g->level_iter) DV_REQUIRE(v >= 0, DV_ERR_ARG, "negative level iterations");
        const int32_t TL = g->total_levels;
        g->lv.resize(TL - 1);
        cudaStream_t s = ctx->stream;
        std::vector<std::vector<double>> dinv(TL - 1);
        for (int32_t l = 0; l < TL - 1; ++l) {
            GLevel &L = g->lv[l];
            DV_REQUIRE(A[l].n_rows == A[l].n_cols, DV_ERR_ARG, "level operator not square");
            DV_REQUIRE(R[l].n_cols == A[l].n_rows && R[l].n_rows == A[l + 1].n_rows, DV_ERR_ARG, "restriction shape");
            DV_REQUIRE(P[l].n_rows == A[l].n_rows && P[l].n_cols == A[l + 1].n_rows, DV_ERR_ARG, "interpolation shape");
            L.n = A[l].n_rows;
            L.A.reset(dv_matrix_build(ctx, A[l], cfg->format, DV_F64, 0, 1e-10));
            L.R.reset(dv_matrix_build(ctx, R[l], cfg->format, DV_F64, 0, 1e-10));
            L.P.reset(dv_matrix_build(ctx, P[l], cfg->format, DV_F64, 0, 1e-10));
            dinv[l].resize(L.n);
            for (int32_t i = 0; i < L.n; ++i) {
                DV_REQUIRE(L.A->host_diag[i] != 0.0, DV_ERR_SINGULAR, "zero diagonal entry");
                dinv[l][i] = 1 / L.A->host_diag[i];   // JacobiPreconditioner (GeometricMultigridSolver.cs:128-134)
            }
            const size_t nb = 8 * (size_t)L.n;
            L.b.alloc(nb); L.x.alloc(nb); L.t.alloc(nb); L.r.alloc(nb); L.D.alloc(nb);
            if (cfg->smoother != DV_SMOOTHER_JACOBI) gs_build_order(A[l], cfg->smoother == DV_SMOOTHER_GS_LEX, s, L.gs);
        }
        // relaxation (GeometricMultigridSolver.cs:209-214 / :109-121 / OpenCLCsrGeometricMultigridSolver.cs:164-171)
        if (cfg->coarse_relaxation) {
            double l = dv_row_ratio_bound(A[TL - 1]);
            for (auto &L : g->lv) L.omega = 2 / l;
        } else {
            for (int32_t l = 0; l < TL - 1; ++l) g->lv[l].omega = 2 / (1.2 * dv_power_bound_ref(A[l], dinv[l]));
        }
        for (int32_t l = 0; l < TL - 1; ++l) {
            GLevel &L = g->lv[l];
            for (double &v : dinv[l]) v *= L.omega;
            DV_CUDA(cudaMemcpyAsync(L.D.p, dinv[l].data(), 8 * dinv[l].size(), cudaMemcpyHostToDevice, s));
            DV_CUDA(cudaStreamSynchronize(s));
        }
        // coarsest level: dense inverse from LDL^T (SkylineMatrix.FactorLdl(true, 1e-15), :255)
        const dv_csr_host &Ac = A[TL - 1];
        g->nc = Ac.n_rows;
        DV_REQUIRE(g->nc <= 16384, DV_ERR_UNSUPPORTED, "coarsest level above 16384 dofs (dense inverse)");
        std::vector<double> dense((size_t)g->nc * g->nc, 0.0);
        for (int32_t r = 0; r < g->nc; ++r)
            for (int32_t k = Ac.rowptr[r]; k < Ac.rowptr[r + 1]; ++k) dense[(size_t)r * g->nc + Ac.col[k]] = Ac.val[k];
        DV_REQUIRE(dv_dense_inverse(g->nc, dense, 1e-15), DV_ERR_SINGULAR, "coarse matrix is singular");
        g->ainv.alloc(8 * dense.size());
        DV_CUDA(cudaMemcpyAsync(g->ainv.p, dense.data(), 8 * dense.size(), cudaMemcpyHostToDevice, s));
        g->bc.alloc(8 * (size_t)g->nc);
        g->xc.alloc(8 * (size_t)g->nc);
        DV_CUDA(cudaStreamSynchronize(s));
        *out = g.release();
    });
}

extern "C" DV_API int dv_gmg_solve(dv_gmg *g, const double *b, const double *x0, double *x, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(g != nullptr, DV_ERR_NOT_INITIALIZED, "You must call Initialize(model) first");
        DV_REQUIRE(b && x, DV_ERR_ARG, "null argument");
        dv_context *ctx = g->ctx;
        dv_ctx_check(ctx);
        cudaStream_t s = ctx->stream;
        GLevel &L0 = g->lv[0];
        const size_t nb = 8 * (size_t)L0.n;
        DV_CUDA(cudaMemcpyAsync(L0.b.p, b, nb, cudaMemcpyHostToDevice, s));
        if (x0) DV_CUDA(cudaMemcpyAsync(L0.x.p, x0, nb, cudaMemcpyHostToDevice, s));
        else DV_CUDA(cudaMemsetAsync(L0.x.p, 0, nb, s));
        cudaEvent_t e0, e1;
        DV_CUDA(cudaEventCreate(&e0));
        DV_CUDA(cudaEventCreate(&e1));
        DV_CUDA(cudaEventRecord(e0, s));
        SolverWs &ws = *g->ws;
        SolverScalars &h = *ws.host_scal;
        std::memset(&h, 0, sizeof(h));
        h.max_it = g->max_cycles;
        ws.push();
        LaunchEnv e = ws.env(true);
        auto body = [&] {
            for (int k = 0; k < g->cycles_per_sync; ++k) cycle(g, e);
        };
        for (;;) {
            ws.run_chunk(body, true, 0);
            ws.pull();
            if (h.done) break;
        }
        DV_CUDA(cudaEventRecord(e1, s));
        DV_CUDA(cudaMemcpyAsync(x, L0.x.p, nb, cudaMemcpyDeviceToHost, s));
        // relative residual of the returned x, recomputed in FP64: r = b - A x, ||r||^2 and ||b||^2
        {
            LaunchEnv ec = ws.env(false);
            OpResid<double> op{{}, L0.b.as<double>(), L0.r.as<double>()};
            launch_rows<double>(ec, L0.A.get(), GatherVec<double, double>{L0.x.as<double>()}, op);
            k_gmg_norm2<<<grid_n(ctx, L0.n), kThreads, 0, s>>>(L0.r.as<double>(), L0.n, ws.sc(), 1, ec.partials,
                                                              ec.ticket);
            DV_CUDA(cudaGetLastError());
            k_gmg_norm2<<<grid_n(ctx, L0.n), kThreads, 0, s>>>(L0.b.as<double>(), L0.n, ws.sc(), 0, ec.partials,
                                                              ec.ticket);
            DV_CUDA(cudaGetLastError());
            ctx->count(2);
        }
        ws.pull();
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (stats) {
            stats->iterations = h.cycle;
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

extern "C" DV_API int dv_gmg_omega(const dv_gmg *g, int32_t level, double *omega) {
    return dv_guard([&] {
        DV_REQUIRE(g && omega, DV_ERR_ARG, "null argument");
        DV_REQUIRE(level >= 0 && level < (int32_t)g->lv.size(), DV_ERR_ARG, "level out of range");
        *omega = g->lv[level].omega;
    });
}

extern "C" DV_API int dv_gmg_destroy(dv_gmg *g) {
    return dv_guard([&] {
        if (!g) return;
        cudaSetDevice(g->ctx->device);
        cudaStreamSynchronize(g->ctx->stream);
        delete g;
    });
}
