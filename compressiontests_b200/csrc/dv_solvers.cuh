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
    struct Chunk {
        int key;
        cudaGraphExec_t exec;
        int64_t launches;
    };
    std::vector<Chunk> chunks;   // captured graphs, one per chunk key (e.g. iterations per chunk)
    int64_t graph_launches = 0;  // launches of the graph run last
    bool warmed = false;
    explicit SolverWs(dv_context *c);
    ~SolverWs();
    dvk::SolverScalars *sc() const { return scal.as<dvk::SolverScalars>(); }
    dvk::LaunchEnv env(bool with_done) const;
    void pull();   // device scalars -> host mirror (synchronises the stream)
    void push();   // host mirror -> device scalars (stream ordered)
    // Runs `body` (the same launches for the same key every time) eagerly on first use,
    // afterwards through the graph captured for `key`.
    void run_chunk(const std::function<void()> &body, bool use_graph, int key);
    void reset_graph() {
        for (auto &c : chunks) cudaGraphExecDestroy(c.exec);
        chunks.clear();
    }
};

double dv_power_estimate(dv_context *ctx, SolverWs &ws, dv_matrix *A, int iters);
