// Shared solver workspace of libduvigpu.so.
#pragma once

#include "dv_kernels.cuh"

#include <functional>

// Reduction partials, device scalars (with a pinned host mirror) and the
// CUDA graph of one chunk of solver iterations.
struct SolverWs {
    dv_context *ctx;
    DevMem red, scal;
    dvk::SolverScalars *host_scal = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int64_t graph_launches = 0;
    bool warmed = false;
    explicit SolverWs(dv_context *c);
    ~SolverWs();
    dvk::SolverScalars *sc() const { return scal.as<dvk::SolverScalars>(); }
    dvk::LaunchEnv env(bool with_done) const;
    void pull();   // device scalars -> host mirror (synchronises the stream)
    void push();   // host mirror -> device scalars (stream ordered)
    void run_chunk(const std::function<void()> &body, bool use_graph, int64_t launches_per_chunk);
    void reset_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
};

double dv_power_estimate(dv_context *ctx, SolverWs &ws, dv_matrix *A, int iters);
