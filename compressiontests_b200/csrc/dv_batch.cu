// Batched multigrid-preconditioned flexible CG over many independent meshes.
//
// The meshes (each with its own hierarchy, of its own depth) are solved
// together: per level, the operators of all meshes that smooth on that level
// are concatenated into one block-diagonal matrix, so each smoothing sweep,
// residual, restriction, prolongation and outer product is ONE launch over all
// meshes, and the whole chunk of iterations is captured in one CUDA graph.
//
// Level layout.  Meshes are ordered by depth (deepest first).  The level-l
// vector holds every mesh with at least l+1 levels; the meshes that continue
// to level l+1 form its prefix (smoothed, restricted, prolonged), the meshes
// whose coarsest level is l form its suffix and get their dense coarse solve
// there (block-diagonal inverse, warp per row).  The level-(l+1) vector then
// covers exactly the prefix meshes, so restriction and prolongation are
// plain block-diagonal products.
//
// Outer loop.  FCG(1) in FP64 on the block-diagonal fine operator with
// per-mesh scalars (alpha, beta, ||r||/||b|| stop test): reductions run over
// chunks of at most 512 rows that never cross a mesh, and the last block sums
// every mesh's chunks in order (deterministic).  A converged mesh is frozen
// (alpha = 0) while the others continue; the FP64 true residual of every mesh
// is verified at exit.  The reference solves one model per solver object
// (GeometricMultigridSolver.Initialize / Solve, GeometricMultigridSolver.cs:57-181).
#include "dv_mgpcg.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>

namespace {

constexpr int kChunkRows = 512;
constexpr int kMaxRefinements = 4;
constexpr int32_t kMaxCoarseDofs = 16384;

struct MeshScalars {
    double zr, zq, pq, alpha, beta, rr, bb;
    int converged, restart, conv_it, pad;
};

struct SegPlan {
    const int32_t *chunk_seg, *chunk_begin, *chunk_end, *seg_chunk;   // seg_chunk: first chunk of each mesh (+ end)
    int32_t nseg;
};

// Per-mesh reduction of NQ sums: block = one chunk (one mesh), the last block
// adds each mesh's chunk partials in chunk order and calls fin(mesh, totals).
template <int NQ, class Fin>
__device__ __forceinline__ void seg_reduce(double (&v)[NQ], const SegPlan &sp, double *partials, unsigned *ticket,
                                           Fin fin) {
    dvk::block_reduce<NQ, 0>(v);
    __shared__ int is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[(size_t)blockIdx.x * NQ + q] = v[q];
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    for (int s = threadIdx.x; s < sp.nseg; s += blockDim.x) {
        double t[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) t[q] = 0.0;
        for (int32_t c = sp.seg_chunk[s]; c < sp.seg_chunk[s + 1]; ++c)
#pragma unroll
            for (int q = 0; q < NQ; ++q) t[q] += __ldcg(partials + (size_t)c * NQ + q);
        fin(s, t);
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0;
}

struct FinRed {
    MeshScalars *ms;
    __device__ void operator()(int s, const double *t) const {
        ms[s].zq = t[0];
        ms[s].zr = t[1];
        ms[s].beta = (ms[s].restart || ms[s].converged) ? 0.0 : -t[0] / ms[s].pq;
        ms[s].restart = 0;
    }
};
// per mesh: z.q and z.r; beta = -(z.q)/(p.q) (FCG(1))
template <class ZT>
__global__ void __launch_bounds__(256) k_seg_fcg_red(const ZT *__restrict__ z, const double *__restrict__ q,
                                                     const double *__restrict__ r, SegPlan sp, MeshScalars *ms,
                                                     const int *__restrict__ done, double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    const int32_t rb = sp.chunk_begin[blockIdx.x], re = sp.chunk_end[blockIdx.x];
    double v[2] = {0.0, 0.0};
    for (int32_t i = rb + threadIdx.x; i < re; i += blockDim.x) {
        const double zi = (double)z[i];
        v[0] += zi * q[i];
        v[1] += zi * r[i];
    }
    seg_reduce<2>(v, sp, partials, ticket, FinRed{ms});
}

// outer product epilogue: q = A z + beta_m q, p = z + beta_m p (m = mesh of the row)
template <class ZT>
struct OpFcgSeg : dvk::NoRed {
    const ZT *__restrict__ z;
    double *__restrict__ p;
    double *__restrict__ q;
    const int32_t *__restrict__ seg_of;
    const MeshScalars *ms;
    __device__ __forceinline__ double init(int32_t) const { return 0.0; }
    __device__ __forceinline__ void row(int32_t i, double s, double *) const {
        const double bt = ms[seg_of[i]].beta;
        q[i] = s + bt * q[i];
        p[i] = (double)z[i] + bt * p[i];
    }
};

struct FinPq {
    MeshScalars *ms;
    __device__ void operator()(int s, const double *t) const {
        ms[s].pq = t[0];
        ms[s].alpha = ms[s].converged ? 0.0 : ms[s].zr / t[0];
    }
};
__global__ void __launch_bounds__(256) k_seg_pq(const double *__restrict__ p, const double *__restrict__ q, SegPlan sp,
                                                MeshScalars *ms, const int *__restrict__ done, double *partials,
                                                unsigned *ticket) {
    if (*(volatile const int *)done) return;
    const int32_t rb = sp.chunk_begin[blockIdx.x], re = sp.chunk_end[blockIdx.x];
    double v[1] = {0.0};
    for (int32_t i = rb + threadIdx.x; i < re; i += blockDim.x) v[0] += p[i] * q[i];
    seg_reduce<1>(v, sp, partials, ticket, FinPq{ms});
}

struct FinUpdate {
    MeshScalars *ms;
    double tol2;
    const dvk::SolverScalars *sc;
    __device__ void operator()(int s, const double *t) const {
        ms[s].rr = t[0];
        if (!ms[s].converged && t[0] <= tol2 * ms[s].bb) {
            ms[s].converged = 1;
            ms[s].conv_it = sc->it + 1;
        }
    }
};
// x += alpha_m p; r -= alpha_m q; rlow = r; ||r||^2 per mesh
template <class RT>
__global__ void __launch_bounds__(256) k_seg_update(double *__restrict__ x, double *__restrict__ r, RT *__restrict__ rlow,
                                                    const double *__restrict__ p, const double *__restrict__ q,
                                                    SegPlan sp, MeshScalars *ms, double tol2, const dvk::SolverScalars *sc,
                                                    const int *__restrict__ done, double *partials, unsigned *ticket) {
    if (*(volatile const int *)done) return;
    const int32_t rb = sp.chunk_begin[blockIdx.x], re = sp.chunk_end[blockIdx.x];
    const double a = ms[sp.chunk_seg[blockIdx.x]].alpha;
    double v[1] = {0.0};
    for (int32_t i = rb + threadIdx.x; i < re; i += blockDim.x) {
        x[i] = x[i] + a * p[i];
        const double ri = r[i] - a * q[i];
        r[i] = ri;
        if (rlow) rlow[i] = (RT)ri;
        v[0] += ri * ri;
    }
    seg_reduce<1>(v, sp, partials, ticket, FinUpdate{ms, tol2, sc});
}

__global__ void k_seg_stop(const MeshScalars *ms, int nseg, dvk::SolverScalars *sc) {
    if (sc->done) return;
    int all = 1, bad = 0;
    for (int s = 0; s < nseg; ++s) {
        all &= ms[s].converged;
        bad |= isnan(ms[s].rr) ? 1 : 0;
    }
    sc->it += 1;
    if (all || bad || sc->it >= sc->max_it) {
        sc->done = 1;
        sc->converged = all && !bad;
        sc->failed = bad;
    }
}

struct FinNorm {
    MeshScalars *ms;
    int slot;
    __device__ void operator()(int s, const double *t) const {
        if (slot == 0) {
            ms[s].bb = t[0];
            if (t[0] == 0.0) {   // zero load: x = 0 is exact
                ms[s].converged = 1;
                ms[s].conv_it = 0;
            }
        } else {
            ms[s].rr = t[0];
        }
    }
};
__global__ void __launch_bounds__(256) k_seg_norm(const double *__restrict__ v, SegPlan sp, MeshScalars *ms, int slot,
                                                  double *partials, unsigned *ticket) {
    const int32_t rb = sp.chunk_begin[blockIdx.x], re = sp.chunk_end[blockIdx.x];
    double a[1] = {0.0};
    for (int32_t i = rb + threadIdx.x; i < re; i += blockDim.x) a[0] += v[i] * v[i];
    seg_reduce<1>(a, sp, partials, ticket, FinNorm{ms, slot});
}

// Block-diagonal dense coarse solve y = Ainv_m b_m for the meshes of a level
// suffix: one warp per row, lanes over the row of the mesh's inverse.
template <class T>
__global__ void __launch_bounds__(256) k_block_coarse(const T *__restrict__ ainv, const int64_t *__restrict__ aoff,
                                                      const int32_t *__restrict__ bstart,
                                                      const int32_t *__restrict__ bsize, const T *__restrict__ b,
                                                      T *__restrict__ y, int32_t nrows, const int *__restrict__ done) {
    if (done && *(volatile const int *)done) return;
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrows; row += nw) {
        const T *a = ainv + aoff[row];
        const T *bb = b + bstart[row];
        const int32_t n = bsize[row];
        T s = 0;
        for (int32_t c = lane; c < n; c += 32) s += a[c] * bb[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[row] = s;
    }
}

// ---------------------------------------------------------------------------
// batched V-cycle
// ---------------------------------------------------------------------------
template <class T>
struct BLevel {
    int32_t t = 0, s = 0;   // rows of the level vector, rows of its smoothing prefix
    std::unique_ptr<dv_matrix> A, R, P;   // prefix operators (null when s == 0)
    DevMem w, b, x, tt, r;                // level vectors (length t)
    DevMem ainv, aoff, bstart, bsize;     // dense inverses of the suffix meshes
};

template <class T>
struct BCycle {
    dv_context *ctx = nullptr;
    int nu = 2;
    std::vector<BLevel<T>> lv;

    T *level(const LaunchEnv &e, size_t l, const T *b) {
        cudaStream_t st = e.stream;
        BLevel<T> &L = lv[l];
        T *x = L.x.template as<T>(), *t = L.tt.template as<T>();
        if (L.s > 0) {
            const T *w = L.w.template as<T>();
            if (nu == 1) {
                k_scale<T><<<grid_for(ctx, L.s), kThreads, 0, st>>>(w, b, x, L.s, e.done);
                DV_CUDA(cudaGetLastError());
                ctx->count();
            } else {
                OpJacobiFromZero<T> op{{}, w, b, x};
                launch_rows<T>(e, L.A.get(), GatherWB<T>{w, b}, op);
                for (int k = 2; k < nu; ++k) {
                    OpJacobi<T> oj{{}, x, w, b, t};
                    launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, oj);
                    std::swap(x, t);
                }
            }
            OpResid<T> orr{{}, b, L.r.template as<T>()};
            launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, orr);
            T *bn = lv[l + 1].b.template as<T>();
            OpSpmv<T, T> orst;
            orst.y = bn;
            orst.clear = 1;
            launch_rows<T>(e, L.R.get(), GatherVec<T, T>{L.r.template as<T>()}, orst);
            T *xn = level(e, l + 1, bn);
            OpSpmv<T, T> opro;
            opro.y = x;
            opro.clear = 0;
            launch_rows<T>(e, L.P.get(), GatherVec<T, T>{xn}, opro);
            for (int k = 0; k < nu; ++k) {
                OpJacobi<T> oj{{}, x, w, b, t};
                launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, oj);
                std::swap(x, t);
            }
        }
        if (L.t > L.s) {
            const int32_t nr = L.t - L.s;
            const int grid = std::max(1, std::min((nr * 32 + 255) / 256, ctx->num_sms * 16));
            k_block_coarse<T><<<grid, 256, 0, st>>>(L.ainv.template as<T>(), L.aoff.template as<int64_t>(),
                                                    L.bstart.template as<int32_t>(), L.bsize.template as<int32_t>(),
                                                    b + L.s, x + L.s, nr, e.done);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
        return x;
    }
};

struct HostCsr {
    std::vector<int32_t> rp, ci;
    std::vector<double> va;
    int32_t nr = 0, nc = 0;
    dv_csr_host view() const { return dv_csr_host{nr, nc, rp.data(), ci.data(), va.data()}; }
};

HostCsr blockdiag(const std::vector<const dv_csr_host *> &blocks) {
    HostCsr h;
    int64_t nnz = 0;
    for (auto *b : blocks) nnz += b->rowptr[b->n_rows];
    DV_REQUIRE(nnz < INT32_MAX, DV_ERR_ARG, "batch level exceeds int32 offsets");
    h.rp.reserve(1);
    h.rp.push_back(0);
    h.ci.reserve(nnz);
    h.va.reserve(nnz);
    for (auto *b : blocks) {
        for (int32_t r = 0; r < b->n_rows; ++r) {
            for (int32_t k = b->rowptr[r]; k < b->rowptr[r + 1]; ++k) {
                h.ci.push_back(b->col[k] + h.nc);
                h.va.push_back(b->val[k]);
            }
            h.rp.push_back((int32_t)h.ci.size());
        }
        h.nr += b->n_rows;
        h.nc += b->n_cols;
    }
    return h;
}

}  // namespace

struct dv_batch {
    dv_context *ctx = nullptr;
    dv_mgpcg_config cfg{};
    int32_t nmesh = 0;
    std::vector<int32_t> order;               // internal position -> user mesh
    std::vector<int64_t> user_off, int_off;   // fine-level row offsets: user order, internal order
    std::vector<int32_t> nfine;               // fine rows per user mesh
    int32_t n = 0;                            // fine rows in all
    std::unique_ptr<BCycle<float>> c32;
    std::unique_ptr<BCycle<double>> c64;
    std::unique_ptr<dv_matrix> Aout;
    std::unique_ptr<SolverWs> ws;
    DevMem b, x, r, r32, p, q, seg_of, ms, red;
    DevMem chunk_seg, chunk_begin, chunk_end, seg_chunk;
    int32_t nchunks = 0;
    std::vector<double> omega_eff;
    SegPlan plan() const {
        return SegPlan{chunk_seg.as<int32_t>(), chunk_begin.as<int32_t>(), chunk_end.as<int32_t>(),
                       seg_chunk.as<int32_t>(), nmesh};
    }
};

namespace {

template <class T>
std::unique_ptr<BCycle<T>> build_bcycle(dv_batch *B, const int32_t *nlev, const dv_csr_host *const *A,
                                        const dv_csr_host *const *P) {
    dv_context *ctx = B->ctx;
    auto c = std::make_unique<BCycle<T>>();
    c->ctx = ctx;
    c->nu = B->cfg.nu;
    const int prec = sizeof(T) == 8 ? DV_F64 : DV_F32;
    cudaStream_t st = ctx->stream;
    const int32_t lmax = nlev[B->order[0]];
    c->lv.resize(lmax);
    for (int32_t l = 0; l < lmax; ++l) {
        BLevel<T> &L = c->lv[l];
        std::vector<const dv_csr_host *> sA, sP;
        std::vector<int32_t> coarse;
        for (int32_t m : B->order) {
            if (nlev[m] >= l + 2) {
                sA.push_back(&A[m][l]);
                sP.push_back(&P[m][l]);
                L.s += A[m][l].n_rows;
            } else if (nlev[m] == l + 1) {
                coarse.push_back(m);
            }
        }
        L.t = L.s;
        for (int32_t m : coarse) L.t += A[m][l].n_rows;
        if (L.s > 0) {
            HostCsr ha = blockdiag(sA), hp = blockdiag(sP);
            dv_csr_host av = ha.view(), pv = hp.view();
            L.A.reset(dv_matrix_build(ctx, av, B->cfg.format, prec, 0, 1e-10));
            L.P.reset(dv_matrix_build(ctx, pv, B->cfg.format, prec, 0, 1e-10));
            HostCsr hr;
            dv_csr_transpose(pv, hr.rp, hr.ci, hr.va);
            hr.nr = pv.n_cols;
            hr.nc = pv.n_rows;
            dv_csr_host rv = hr.view();
            L.R.reset(dv_matrix_build(ctx, rv, B->cfg.format, prec, 0, 1e-10));
            for (double d : L.A->host_diag) DV_REQUIRE(d != 0.0, DV_ERR_SINGULAR, "zero diagonal entry");
            double om = B->cfg.omega;
            if (B->cfg.omega_mode == DV_OMEGA_SPECTRAL) {
                const double lam = dv_power_estimate(ctx, *B->ws, L.A.get(), 40);
                om = B->cfg.omega * 2.0 / (1.1 * lam);
            }
            B->omega_eff.push_back(om);
            L.w.alloc(sizeof(T) * (size_t)L.s);
            std::vector<T> w(L.s);
            for (int32_t i = 0; i < L.s; ++i) w[i] = (T)(om / L.A->host_diag[i]);
            DV_CUDA(cudaMemcpyAsync(L.w.p, w.data(), sizeof(T) * w.size(), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaStreamSynchronize(st));
        }
        const size_t vb = sizeof(T) * (size_t)L.t;
        L.b.alloc(vb);
        L.x.alloc(vb);
        L.tt.alloc(vb);
        L.r.alloc(vb);
        if (!coarse.empty()) {
            std::vector<T> inv;
            std::vector<int64_t> aoff;
            std::vector<int32_t> bstart, bsize;
            int32_t start = 0;
            for (int32_t m : coarse) {
                const dv_csr_host &a = A[m][l];
                const int32_t nc = a.n_rows;
                DV_REQUIRE(nc <= kMaxCoarseDofs, DV_ERR_UNSUPPORTED, "coarsest level above 16384 dofs (dense inverse)");
                std::vector<double> dense((size_t)nc * nc, 0.0);
                for (int32_t r = 0; r < nc; ++r)
                    for (int32_t k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) dense[(size_t)r * nc + a.col[k]] = a.val[k];
                DV_REQUIRE(dv_dense_inverse(nc, dense, 1e-300), DV_ERR_SINGULAR, "coarse matrix is singular");
                const int64_t base = (int64_t)inv.size();
                for (double v : dense) inv.push_back((T)v);
                for (int32_t r = 0; r < nc; ++r) {
                    aoff.push_back(base + (int64_t)r * nc);
                    bstart.push_back(start);
                    bsize.push_back(nc);
                }
                start += nc;
            }
            L.ainv.alloc(sizeof(T) * inv.size());
            L.aoff.alloc(8 * aoff.size());
            L.bstart.alloc(4 * bstart.size());
            L.bsize.alloc(4 * bsize.size());
            DV_CUDA(cudaMemcpyAsync(L.ainv.p, inv.data(), sizeof(T) * inv.size(), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaMemcpyAsync(L.aoff.p, aoff.data(), 8 * aoff.size(), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaMemcpyAsync(L.bstart.p, bstart.data(), 4 * bstart.size(), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaMemcpyAsync(L.bsize.p, bsize.data(), 4 * bsize.size(), cudaMemcpyHostToDevice, st));
            DV_CUDA(cudaStreamSynchronize(st));
        }
    }
    return c;
}

template <class T>
void batch_solve_impl(dv_batch *B, BCycle<T> &vc, int32_t *conv_per_mesh, int32_t *its_per_mesh, dv_stats *stats) {
    dv_context *ctx = B->ctx;
    cudaStream_t st = ctx->stream;
    const int32_t n = B->n;
    const size_t nb = 8 * (size_t)n;
    constexpr bool kMixed = std::is_same<T, float>::value;
    SolverWs &ws = *B->ws;
    dvk::SolverScalars &h = *ws.host_scal;
    std::memset(&h, 0, sizeof(h));
    h.max_it = B->cfg.max_iterations;
    h.tol2 = B->cfg.tol * B->cfg.tol;
    ws.push();
    LaunchEnv e0 = ws.env(false);
    e0.ticket = B->red.as<unsigned>();
    e0.partials = reinterpret_cast<double *>(B->red.as<char>() + 64);
    LaunchEnv ed = e0;
    ed.done = &ws.sc()->done;
    const SegPlan sp = B->plan();
    MeshScalars *ms = B->ms.as<MeshScalars>();
    std::vector<MeshScalars> hm(B->nmesh);
    for (auto &m : hm) {
        std::memset(&m, 0, sizeof(m));
        m.restart = 1;
        m.pq = 1.0;
        m.conv_it = -1;
    }
    DV_CUDA(cudaMemcpyAsync(ms, hm.data(), sizeof(MeshScalars) * hm.size(), cudaMemcpyHostToDevice, st));
    auto norms = [&](const double *v, int slot) {
        k_seg_norm<<<B->nchunks, 256, 0, st>>>(v, sp, ms, slot, e0.partials, e0.ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
    };
    norms(B->b.as<double>(), 0);
    DV_CUDA(cudaMemsetAsync(B->x.p, 0, nb, st));
    DV_CUDA(cudaMemcpyAsync(B->r.p, B->b.p, nb, cudaMemcpyDeviceToDevice, st));
    DV_CUDA(cudaMemsetAsync(B->p.p, 0, nb, st));
    DV_CUDA(cudaMemsetAsync(B->q.p, 0, nb, st));
    T *rin = kMixed ? reinterpret_cast<T *>(B->r32.p) : reinterpret_cast<T *>(B->r.p);
    auto to_low = [&] {
        if (kMixed) {
            dvk::k_convert<double, float><<<grid_for(ctx, n), kThreads, 0, st>>>(B->r.as<double>(), B->r32.as<float>(), n);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        }
    };
    to_low();
    const T *z = vc.level(ed, 0, rin);
    const int per = B->cfg.iterations_per_sync > 0 ? B->cfg.iterations_per_sync : 4;
    const double tol2 = h.tol2;
    double *Xd = B->x.as<double>(), *Rd = B->r.as<double>(), *Pd = B->p.as<double>(), *Qd = B->q.as<double>();
    const T *zfinal = z;
    auto body = [&] {
        const T *zz = z;
        for (int it = 0; it < per; ++it) {
            k_seg_fcg_red<T><<<B->nchunks, 256, 0, st>>>(zz, Qd, Rd, sp, ms, ed.done, ed.partials, ed.ticket);
            DV_CUDA(cudaGetLastError());
            ctx->count();
            OpFcgSeg<T> op{{}, zz, Pd, Qd, B->seg_of.as<int32_t>(), ms};
            launch_rows<double>(ed, B->Aout.get(), GatherVec<T, double>{zz}, op);
            k_seg_pq<<<B->nchunks, 256, 0, st>>>(Pd, Qd, sp, ms, ed.done, ed.partials, ed.ticket);
            DV_CUDA(cudaGetLastError());
            T *rl = kMixed ? reinterpret_cast<T *>(B->r32.p) : nullptr;
            k_seg_update<T><<<B->nchunks, 256, 0, st>>>(Xd, Rd, rl, Pd, Qd, sp, ms, tol2, ws.sc(), ed.done,
                                                        ed.partials, ed.ticket);
            DV_CUDA(cudaGetLastError());
            k_seg_stop<<<1, 1, 0, st>>>(ms, B->nmesh, ws.sc());
            DV_CUDA(cudaGetLastError());
            ctx->count(3);
            zz = vc.level(ed, 0, rin);
        }
        zfinal = zz;
    };
    auto true_residual = [&] {   // into Pd, per-mesh ||r||^2 into rr
        OpResid<double> orr{{}, B->b.as<double>(), Pd};
        launch_rows<double>(e0, B->Aout.get(), GatherVec<double, double>{Xd}, orr);
        norms(Pd, 1);
        DV_CUDA(cudaMemcpyAsync(hm.data(), ms, sizeof(MeshScalars) * hm.size(), cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    };
    int refinements = 0;
    bool verified = false;   // the last true_residual() was taken on the final iterate
    for (;;) {
        ws.run_chunk(body, B->cfg.use_graphs != 0, 0);
        DV_REQUIRE(zfinal == z, DV_ERR_ARG, "batched V-cycle output buffer is not stable across iterations");
        ws.pull();
        if (!h.done) continue;
        if (!h.converged) break;
        true_residual();
        int bad = 0;
        for (auto &m : hm)
            if (!(m.rr <= tol2 * m.bb)) {
                m.converged = 0;
                ++bad;
            }
        if (bad == 0 || refinements >= kMaxRefinements || h.it >= h.max_it) {
            verified = true;
            break;
        }
        ++refinements;
        for (auto &m : hm) m.restart = 1;
        DV_CUDA(cudaMemcpyAsync(ms, hm.data(), sizeof(MeshScalars) * hm.size(), cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaMemcpyAsync(Rd, Pd, nb, cudaMemcpyDeviceToDevice, st));
        to_low();
        h.done = 0;
        h.converged = 0;
        ws.push();
        z = vc.level(ed, 0, rin);
    }
    if (!verified) true_residual();
    double worst = 0.0, worst_abs = 0.0;
    int all = 1;
    for (int32_t pos = 0; pos < B->nmesh; ++pos) {
        const MeshScalars &m = hm[pos];
        const int32_t user = B->order[pos];
        const int ok = m.rr <= tol2 * m.bb;
        all &= ok;
        if (conv_per_mesh) conv_per_mesh[user] = ok;
        if (its_per_mesh) its_per_mesh[user] = m.conv_it >= 0 ? m.conv_it : h.it;
        worst = std::max(worst, m.bb > 0 ? std::sqrt(m.rr / m.bb) : std::sqrt(m.rr));
        worst_abs = std::max(worst_abs, std::sqrt(m.rr));
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

void run(dv_batch *B, int32_t *conv, int32_t *its, dv_stats *stats) {
    cudaStream_t st = B->ctx->stream;
    cudaEvent_t e0, e1;
    DV_CUDA(cudaEventCreate(&e0));
    DV_CUDA(cudaEventCreate(&e1));
    DV_CUDA(cudaEventRecord(e0, st));
    if (B->c32) batch_solve_impl<float>(B, *B->c32, conv, its, stats);
    else batch_solve_impl<double>(B, *B->c64, conv, its, stats);
    DV_CUDA(cudaEventRecord(e1, st));
    DV_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) stats->solve_ms = ms;
}

// user-order <-> internal-order copies of the fine-level vectors
void permute(dv_batch *B, const double *src, double *dst, bool to_internal, cudaMemcpyKind kind) {
    for (int32_t pos = 0; pos < B->nmesh; ++pos) {
        const int32_t m = B->order[pos];
        const size_t bytes = 8 * (size_t)B->nfine[m];
        const double *s = src + (to_internal ? B->user_off[m] : B->int_off[pos]);
        double *d = dst + (to_internal ? B->int_off[pos] : B->user_off[m]);
        DV_CUDA(cudaMemcpyAsync(d, s, bytes, kind, B->ctx->stream));
    }
}

}  // namespace

extern "C" DV_API int dv_batch_create(dv_context *ctx, int32_t n_meshes, const int32_t *n_levels,
                                      const dv_csr_host *const *A, const dv_csr_host *const *P,
                                      const dv_mgpcg_config *cfg, dv_batch **out) {
    return dv_guard([&] {
        DV_REQUIRE(ctx && n_levels && A && P && cfg && out && n_meshes >= 1, DV_ERR_ARG, "null argument");
        DV_REQUIRE(cfg->precision == DV_F64 || cfg->precision == DV_MIXED, DV_ERR_ARG, "precision must be DV_F64 or DV_MIXED");
        DV_REQUIRE(cfg->nu >= 1 && cfg->max_iterations >= 1 && cfg->tol > 0, DV_ERR_ARG, "bad smoothing or stop parameters");
        DV_REQUIRE(cfg->smoother == DV_SMOOTHER_JACOBI, DV_ERR_UNSUPPORTED, "batched meshes smooth with weighted Jacobi only");
        dv_ctx_check(ctx);
        for (int32_t m = 0; m < n_meshes; ++m) {
            DV_REQUIRE(n_levels[m] >= 1 && A[m] && (n_levels[m] == 1 || P[m]), DV_ERR_ARG, "mesh without levels");
            for (int32_t l = 0; l < n_levels[m]; ++l)
                DV_REQUIRE(A[m][l].n_rows == A[m][l].n_cols && A[m][l].n_rows >= 1, DV_ERR_ARG, "level operators must be square");
            for (int32_t l = 0; l + 1 < n_levels[m]; ++l)
                DV_REQUIRE(P[m][l].n_rows == A[m][l].n_rows && P[m][l].n_cols == A[m][l + 1].n_rows, DV_ERR_ARG,
                           "prolongation shape does not match the levels");
        }
        auto B = std::make_unique<dv_batch>();
        B->ctx = ctx;
        B->cfg = *cfg;
        B->nmesh = n_meshes;
        B->order.resize(n_meshes);
        std::iota(B->order.begin(), B->order.end(), 0);
        std::stable_sort(B->order.begin(), B->order.end(), [&](int32_t a, int32_t b) { return n_levels[a] > n_levels[b]; });
        B->nfine.resize(n_meshes);
        B->user_off.assign(n_meshes + 1, 0);
        for (int32_t m = 0; m < n_meshes; ++m) {
            B->nfine[m] = A[m][0].n_rows;
            B->user_off[m + 1] = B->user_off[m] + B->nfine[m];
        }
        DV_REQUIRE(B->user_off[n_meshes] < INT32_MAX, DV_ERR_ARG, "batch exceeds int32 rows");
        B->n = (int32_t)B->user_off[n_meshes];
        B->int_off.assign(n_meshes + 1, 0);
        for (int32_t pos = 0; pos < n_meshes; ++pos) B->int_off[pos + 1] = B->int_off[pos] + B->nfine[B->order[pos]];
        B->ws = std::make_unique<SolverWs>(ctx);
        // outer FP64 operator over all meshes
        {
            std::vector<const dv_csr_host *> a0;
            for (int32_t m : B->order) a0.push_back(&A[m][0]);
            HostCsr h = blockdiag(a0);
            dv_csr_host v = h.view();
            B->Aout.reset(dv_matrix_build(ctx, v, cfg->outer_format, DV_F64, 0, 1e-10));
        }
        if (cfg->precision == DV_MIXED) B->c32 = build_bcycle<float>(B.get(), n_levels, A, P);
        else B->c64 = build_bcycle<double>(B.get(), n_levels, A, P);
        // reduction chunks: <= kChunkRows rows, never across a mesh
        std::vector<int32_t> cseg, cbeg, cend, segc(1, 0), segof(B->n);
        for (int32_t pos = 0; pos < n_meshes; ++pos) {
            const int32_t r0 = (int32_t)B->int_off[pos], r1 = (int32_t)B->int_off[pos + 1];
            for (int32_t r = r0; r < r1; r += kChunkRows) {
                cseg.push_back(pos);
                cbeg.push_back(r);
                cend.push_back(std::min(r1, r + kChunkRows));
            }
            segc.push_back((int32_t)cseg.size());
            std::fill(segof.begin() + r0, segof.begin() + r1, pos);
        }
        B->nchunks = (int32_t)cseg.size();
        cudaStream_t st = ctx->stream;
        auto up = [&](DevMem &d, const std::vector<int32_t> &v) {
            d.alloc(4 * v.size());
            DV_CUDA(cudaMemcpyAsync(d.p, v.data(), 4 * v.size(), cudaMemcpyHostToDevice, st));
        };
        up(B->chunk_seg, cseg);
        up(B->chunk_begin, cbeg);
        up(B->chunk_end, cend);
        up(B->seg_chunk, segc);
        up(B->seg_of, segof);
        DV_CUDA(cudaStreamSynchronize(st));
        const size_t nb = 8 * (size_t)B->n;
        B->b.alloc(nb);
        B->x.alloc(nb);
        B->r.alloc(nb);
        B->p.alloc(nb);
        B->q.alloc(nb);
        if (cfg->precision == DV_MIXED) B->r32.alloc(4 * (size_t)B->n);
        B->ms.alloc(sizeof(MeshScalars) * (size_t)n_meshes);
        B->red.alloc(64 + sizeof(double) * 2 * (size_t)B->nchunks);
        *out = B.release();
    });
}

extern "C" DV_API int dv_batch_create_hex(dv_context *ctx, int32_t n_meshes, const int32_t *ne, double E, double nu,
                                          int32_t max_coarse_dofs, const dv_mgpcg_config *cfg, dv_batch **out) {
    return dv_guard([&] {
        DV_REQUIRE(ctx && ne && cfg && out && n_meshes >= 1 && max_coarse_dofs >= 1, DV_ERR_ARG, "null argument");
        // per mesh: the stiffness and its Galerkin hierarchy (vertex factor-2 coarsening, trilinear P)
        std::vector<std::vector<HostCsr>> A(n_meshes), P(n_meshes);
        for (int32_t m = 0; m < n_meshes; ++m) {
            int32_t cur[3] = {ne[3 * m], ne[3 * m + 1], ne[3 * m + 2]};
            HostCsr a;
            int64_t nnz;
            int st = dv_hex_csr_size(cur, &a.nr, &nnz);
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            a.nc = a.nr;
            a.rp.resize((size_t)a.nr + 1);
            a.ci.resize(nnz);
            a.va.resize(nnz);
            st = dv_hex_assemble(cur, nullptr, 1.0, E, nu, a.rp.data(), a.ci.data(), a.va.data());
            DV_REQUIRE(st == DV_OK, st, dv_last_error());
            A[m].push_back(std::move(a));
            while (A[m].back().nr > max_coarse_dofs && std::max(cur[0], std::max(cur[1], cur[2])) > 1) {
                HostCsr p, g;
                int64_t pn;
                st = dv_hex_trilinear_size(cur, &p.nr, &p.nc, &pn);
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                p.rp.resize((size_t)p.nr + 1);
                p.ci.resize(pn);
                p.va.resize(pn);
                st = dv_hex_trilinear(cur, p.rp.data(), p.ci.data(), p.va.data());
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                const dv_csr_host av = A[m].back().view(), pv = p.view();
                int64_t gn;
                st = dv_galerkin_size(&av, &pv, &g.nr, &gn);
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                g.nc = g.nr;
                g.rp.resize((size_t)g.nr + 1);
                g.ci.resize(gn);
                g.va.resize(gn);
                st = dv_galerkin(&av, &pv, g.rp.data(), g.ci.data(), g.va.data());
                DV_REQUIRE(st == DV_OK, st, dv_last_error());
                P[m].push_back(std::move(p));
                A[m].push_back(std::move(g));
                for (auto &c : cur) c = (c + 1) / 2;
            }
        }
        std::vector<std::vector<dv_csr_host>> av(n_meshes), pv(n_meshes);
        std::vector<const dv_csr_host *> ap(n_meshes), pp(n_meshes);
        std::vector<int32_t> nlev(n_meshes);
        for (int32_t m = 0; m < n_meshes; ++m) {
            for (auto &a : A[m]) av[m].push_back(a.view());
            for (auto &p : P[m]) pv[m].push_back(p.view());
            if (pv[m].empty()) pv[m].push_back(dv_csr_host{});
            ap[m] = av[m].data();
            pp[m] = pv[m].data();
            nlev[m] = (int32_t)A[m].size();
        }
        dv_batch *B = nullptr;
        int st = dv_batch_create(ctx, n_meshes, nlev.data(), ap.data(), pp.data(), cfg, &B);
        DV_REQUIRE(st == DV_OK, st, dv_last_error());
        std::unique_ptr<dv_batch, int (*)(dv_batch *)> guard(B, dv_batch_destroy);
        // the finest operators applied matrix-free: the outer FP64 one over every mesh, the V-cycle's level 0
        // over the meshes that smooth there (internal order, the block-diagonal layout of the batch)
        const char *mf = getenv("DV_MATRIX_FREE");
        if (!(mf && mf[0] == '0')) {
            std::vector<int32_t> all, smoothed;
            for (int32_t m : B->order) {
                all.insert(all.end(), ne + 3 * m, ne + 3 * m + 3);
                if (nlev[m] >= 2) smoothed.insert(smoothed.end(), ne + 3 * m, ne + 3 * m + 3);
            }
            B->Aout.reset(dv_hex_operator_build(ctx, n_meshes, all.data(), nullptr, 1.0, E, nu, DV_F64));
            if (!smoothed.empty()) {
                const int32_t ns = (int32_t)smoothed.size() / 3;
                if (B->c32) B->c32->lv[0].A.reset(dv_hex_operator_build(ctx, ns, smoothed.data(), nullptr, 1.0, E, nu, DV_F32));
                else B->c64->lv[0].A.reset(dv_hex_operator_build(ctx, ns, smoothed.data(), nullptr, 1.0, E, nu, DV_F64));
            }
        }
        *out = guard.release();
    });
}

extern "C" DV_API int dv_batch_info(const dv_batch *B, int32_t *n_rows, int32_t *n_levels_max, int32_t *n_launches_per_cycle) {
    return dv_guard([&] {
        DV_REQUIRE(B != nullptr, DV_ERR_NOT_INITIALIZED, "batch not created");
        if (n_rows) *n_rows = B->n;
        if (n_levels_max) *n_levels_max = B->c32 ? (int32_t)B->c32->lv.size() : (int32_t)B->c64->lv.size();
        if (n_launches_per_cycle) *n_launches_per_cycle = (int32_t)B->ws->graph_launches;
    });
}

extern "C" DV_API int dv_batch_omega(const dv_batch *B, int32_t level, double *omega) {
    return dv_guard([&] {
        DV_REQUIRE(B && omega, DV_ERR_ARG, "null argument");
        DV_REQUIRE(level >= 0 && level < (int32_t)B->omega_eff.size(), DV_ERR_ARG, "level out of range");
        *omega = B->omega_eff[level];
    });
}

extern "C" DV_API int dv_batch_solve_device(dv_batch *B, const double *d_b, double *d_x, int32_t *converged_per_mesh,
                                            int32_t *iterations_per_mesh, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(B != nullptr, DV_ERR_NOT_INITIALIZED, "batch not created");
        DV_REQUIRE(d_b && d_x, DV_ERR_ARG, "null argument");
        dv_ctx_check(B->ctx);
        permute(B, d_b, B->b.as<double>(), true, cudaMemcpyDeviceToDevice);
        run(B, converged_per_mesh, iterations_per_mesh, stats);
        permute(B, B->x.as<double>(), d_x, false, cudaMemcpyDeviceToDevice);
        DV_CUDA(cudaStreamSynchronize(B->ctx->stream));
    });
}

extern "C" DV_API int dv_batch_solve(dv_batch *B, const double *b, double *x, int32_t *converged_per_mesh,
                                     int32_t *iterations_per_mesh, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(B != nullptr, DV_ERR_NOT_INITIALIZED, "batch not created");
        DV_REQUIRE(b && x, DV_ERR_ARG, "null argument");
        dv_ctx_check(B->ctx);
        permute(B, b, B->b.as<double>(), true, cudaMemcpyHostToDevice);
        run(B, converged_per_mesh, iterations_per_mesh, stats);
        permute(B, B->x.as<double>(), x, false, cudaMemcpyDeviceToHost);
        DV_CUDA(cudaStreamSynchronize(B->ctx->stream));
    });
}

extern "C" DV_API int dv_batch_destroy(dv_batch *B) {
    return dv_guard([&] {
        if (!B) return;
        cudaSetDevice(B->ctx->device);
        cudaStreamSynchronize(B->ctx->stream);
        delete B;
    });
}
