// Multigrid-preconditioned flexible CG: the V-cycle hierarchy and the solver
// object, shared by the single- and multi-right-hand-side drivers.
#pragma once

#include "dv_gs.cuh"
#include "dv_kernels.cuh"
#include "dv_solvers.cuh"

#include <algorithm>
#include <memory>
#include <vector>

inline int grid_for(dv_context *ctx, int64_t n) {
    int64_t b = (n + dvk::kThreads - 1) / dvk::kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, ctx->num_sms * 8));
}

struct MultiHolder;
void dv_mgpcg_multi_release(MultiHolder *m);

using namespace dvk;   // internal header: the V-cycle code below is written against dvk

template <class T>
struct VLevel {
    std::unique_ptr<dv_matrix> A, R, P;
    DevMem w, b, x, t, r;
    DevMem wb;    // w .* b, written by the restriction from the level above (Jacobi, nu > 1)
    int32_t n = 0;
    GsOrder gs;   // Gauss-Seidel row groups (smoother != Jacobi)
};

template <class T>
struct VCycle {
    dv_context *ctx = nullptr;
    std::vector<VLevel<T>> lv;   // all but the coarsest
    int32_t nc = 0;
    DevMem ainv, bc, xc;
    int nu = 2;
    int smoother = DV_SMOOTHER_JACOBI;

    // x_0 = V(b_0); returns the buffer that holds the result (level-0 x or t).
    // Flexible-CG reduction fused into the finest level's last sweep (Jacobi only): set
    // by the driver, consumed by level 0.
    const double *fuse_q = nullptr, *fuse_r = nullptr;
    // w .* b of level 0 when the caller already formed it (the flexible CG's update writes it next to
    // the FP32 residual): the first sweep then gathers one staged array instead of two
    const T *wb0 = nullptr;
    SolverScalars *fuse_sc = nullptr;
    bool fused_red() const { return fuse_sc != nullptr && smoother == DV_SMOOTHER_JACOBI; }

    T *run(const LaunchEnv &e, const T *b0) { return level(e, 0, b0, wb0); }

    // wb: w .* b of this level when the caller formed it (else the first sweep forms it)
    T *level(const LaunchEnv &e, size_t l, const T *b, const T *wb = nullptr) {
        cudaStream_t s = e.stream;
        if (l == lv.size()) {
            k_dense_gemv_rows<T><<<std::max(1, std::min(nc, ctx->num_sms * 16)), 128, 0, s>>>(
                ainv.template as<T>(), b, xc.template as<T>(), nc, e.done);
            DV_CUDA(cudaGetLastError());
            ctx->count();
            return xc.template as<T>();
        }
        VLevel<T> &L = lv[l];
        if (smoother != DV_SMOOTHER_JACOBI) return level_gs(e, l, b);
        T *x = L.x.template as<T>(), *t = L.t.template as<T>();
        const T *w = L.w.template as<T>();
        if (nu == 1) {
            k_scale<T><<<grid_for(ctx, L.n), kThreads, 0, s>>>(w, b, x, L.n, e.done);
            DV_CUDA(cudaGetLastError());
            ctx->count();
        } else {
            OpJacobiFromZero<T> op{{}, w, b, x};
            if (wb) launch_rows<T>(e, L.A.get(), GatherVec<T, T>{wb}, op);
            else launch_rows<T>(e, L.A.get(), GatherWB<T>{w, b}, op);
            for (int k = 2; k < nu; ++k) {
                OpJacobi<T> oj{{}, x, w, b, t};
                launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, oj);
                std::swap(x, t);
            }
        }
        OpResid<T> orr{{}, b, L.r.template as<T>()};
        launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, orr);
        T *bn = l + 1 < lv.size() ? lv[l + 1].b.template as<T>() : bc.template as<T>();
        T *wbn = nullptr;
        if (l + 1 < lv.size() && nu > 1) {   // the next level's first sweep gathers w .* b
            wbn = lv[l + 1].wb.template as<T>();
            OpRestrictWB<T> orst{{}, bn, wbn, lv[l + 1].w.template as<T>()};
            launch_rows<T>(e, L.R.get(), GatherVec<T, T>{L.r.template as<T>()}, orst);
        } else {
            OpSpmv<T, T> orst;
            orst.y = bn;
            orst.clear = 1;
            launch_rows<T>(e, L.R.get(), GatherVec<T, T>{L.r.template as<T>()}, orst);
        }
        T *xn = level(e, l + 1, bn, wbn);
        OpSpmv<T, T> opro;
        opro.y = x;
        opro.clear = 0;
        launch_rows<T>(e, L.P.get(), GatherVec<T, T>{xn}, opro);
        for (int k = 0; k < nu; ++k) {
            if (l == 0 && k == nu - 1 && fused_red()) {
                OpJacobiFcgRed<T> oj{x, w, b, t, fuse_q, fuse_r, fuse_sc};
                launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, oj);
            } else {
                OpJacobi<T> oj{{}, x, w, b, t};
                launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, oj);
            }
            std::swap(x, t);
        }
        return x;
    }

    // Gauss-Seidel variant: x = 0, nu forward sweeps, coarse correction, nu forward sweeps.
    T *level_gs(const LaunchEnv &e, size_t l, const T *b) {
        cudaStream_t s = e.stream;
        VLevel<T> &L = lv[l];
        T *x = L.x.template as<T>();
        k_fill<T><<<grid_for(ctx, L.n), kThreads, 0, s>>>(x, T(0), L.n, e.done);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        for (int k = 0; k < nu; ++k) gs_sweep<T>(e, L.A.get(), L.gs, b, x);
        OpResid<T> orr{{}, b, L.r.template as<T>()};
        launch_rows<T>(e, L.A.get(), GatherVec<T, T>{x}, orr);
        T *bn = l + 1 < lv.size() ? lv[l + 1].b.template as<T>() : bc.template as<T>();
        OpSpmv<T, T> orst;
        orst.y = bn;
        orst.clear = 1;
        launch_rows<T>(e, L.R.get(), GatherVec<T, T>{L.r.template as<T>()}, orst);
        T *xn = level(e, l + 1, bn);
        OpSpmv<T, T> opro;
        opro.y = x;
        opro.clear = 0;
        launch_rows<T>(e, L.P.get(), GatherVec<T, T>{xn}, opro);
        for (int k = 0; k < nu; ++k) gs_sweep<T>(e, L.A.get(), L.gs, b, x);
        return x;
    }
};

struct dv_mgpcg {
    dv_context *ctx = nullptr;
    dv_mgpcg_config cfg{};
    std::unique_ptr<dv_matrix> Aout;   // FP64 operator of the outer loop
    std::unique_ptr<VCycle<float>> v32;
    std::unique_ptr<VCycle<double>> v64;
    std::unique_ptr<SolverWs> ws;
    int32_t n = 0;
    DevMem b, x, r, r32, wb32, p, q;
    std::vector<double> omega_eff;
    int64_t launches_last = 0;
    MultiHolder *multi = nullptr;   // block (multi-right-hand-side) work buffers, created on first use
    ~dv_mgpcg() { dv_mgpcg_multi_release(multi); }
};

