// Jacobi PCG without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// solve: host applications that reserve all their device memory once at
// start-up (a pool owned by another allocator) and forbid allocations
// afterwards, and time-critical loops that cannot afford cudaFree, which
// synchronises the whole device.  dv_pcg_solve_noalloc serves them: it runs the same kernels as dv_pcg_solve,
// but its work vectors (r, z, p, Ap), reduction partials and scalars live in
// one file-scope device array of fixed size, so the call itself allocates
// nothing.  The caller passes the matrix (already uploaded) and device
// pointers for b and x.
//
// Limits and sharing:
//  - at most kNoAllocMaxRows rows (the array holds four FP64 work vectors of
//    that length); larger systems are rejected with DV_ERR_ARG;
//  - the array exists once per device in every process that loads the library
//    and lives until exit; every call on that device uses the same array, so
//    calls whose work overlaps on the GPU (other threads, other streams)
//    race and must be serialised by the caller;
//  - the array keeps the previous call's contents; the call clears what must
//    start from zero (the reduction ticket) and initialises the rest;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress); make that first call before any stream capture;
//  - the array, like the kernels' code, is device memory that CUDA allocates
//    when it loads this part of the library.  Under CUDA's default lazy module
//    loading that happens at the first call on each device (and a kernel's code
//    at its first launch), not when the context is created.  A caller that
//    reserves all free device memory should either make one call with each
//    matrix format it will use before reserving it, or run with
//    CUDA_MODULE_LOADING=EAGER, which loads everything when CUDA initialises.
#include "dv_kernels.cuh"

#include <chrono>
#include <cmath>
#include <mutex>

using namespace dvk;

namespace {

constexpr int32_t kNoAllocMaxRows = 131072;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kHeaderBytes = 256;                                   // ticket + scalars
constexpr size_t kPartialBytes = sizeof(double) * kMaxRed * kNoAllocMaxBlocks;
constexpr size_t kVectorBytes = sizeof(double) * (size_t)kNoAllocMaxRows;
constexpr size_t kScratchBytes = kHeaderBytes + kPartialBytes + 4 * kVectorBytes;   // 4,325,632 bytes
static_assert(sizeof(SolverScalars) + 16 <= kHeaderBytes, "scalars do not fit the header");

// The scratch array.  Host code must not take its address directly (that is a
// host-side stand-in); it uses the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mutex;
void *g_addr[64] = {};   // device address of the array, per device ordinal

void *scratch_address(int device) {
    DV_REQUIRE(device >= 0 && device < 64, DV_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_addr_mutex);
    if (!g_addr[device]) {
        void *p = nullptr;
        DV_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));   // the device is current (dv_ctx_check)
        DV_REQUIRE(p != nullptr, DV_ERR_CUDA, "no device address for the scratch array");
        g_addr[device] = p;
    }
    return g_addr[device];
}

__global__ void k_na_init(SolverScalars *sc, int32_t max_it) {
    SolverScalars z{};
    z.max_it = max_it;
    *sc = z;
}

// p = z = M r with M = 1/diag (JacobiPreconditioner), r.z
__global__ void k_na_pcg_init(const double *__restrict__ diag, const double *__restrict__ r, double *__restrict__ z,
                              double *__restrict__ p, int32_t n, SolverScalars *sc, double *partials, unsigned *ticket) {
    double red[1] = {0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = 1 / diag[i];
        double zi = m * r[i];
        z[i] = zi;
        p[i] = zi;
        red[0] += r[i] * zi;
    }
    double tot[1];
    if (grid_reduce<1, 0>(red, partials, ticket, tot)) sc->rz = tot[0];
}

__global__ void k_na_update(const double *__restrict__ diag, const double *__restrict__ ap, const double *__restrict__ p,
                            double *__restrict__ x, double *__restrict__ r, double *__restrict__ z, int32_t n,
                            double tol, SolverScalars *sc, double *partials, unsigned *ticket) {
    if (*(volatile const int *)&sc->done) return;
    const double a = sc->alpha;
    double red[4] = {0.0, 0.0, 0.0, 0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = x[i] + a * p[i];
        double ri = r[i] - a * ap[i];
        r[i] = ri;
        double zi = (1 / diag[i]) * ri;
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
        bool converged = !failed && t[0] <= tol;
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

__global__ void k_na_p(const double *__restrict__ z, double *__restrict__ p, int32_t n, const SolverScalars *sc) {
    if (*(volatile const int *)&sc->done) return;
    const double b = sc->beta;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = z[i] + b * p[i];
}

// ||b||^2 and ||r||^2 of the exit check (r = b - A x recomputed in FP64).
__global__ void k_na_norms(const double *__restrict__ b, const double *__restrict__ r, int32_t n, SolverScalars *sc,
                           double *partials, unsigned *ticket) {
    double red[2] = {0.0, 0.0};
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        red[0] += b[i] * b[i];
        red[1] += r[i] * r[i];
    }
    double t[2];
    if (grid_reduce<2, 0>(red, partials, ticket, t)) {
        sc->bb = t[0];
        sc->rr = t[1];
    }
}

}  // namespace

extern "C" DV_API int dv_pcg_solve_noalloc(dv_matrix *A, const double *d_b, double *d_x, int32_t use_x0,
                                           int32_t max_iterations, double tol, dv_stats *stats) {
    return dv_guard([&] {
        DV_REQUIRE(A && d_b && d_x, DV_ERR_ARG, "null argument");
        DV_REQUIRE(A->n_rows == A->n_cols, DV_ERR_ARG, "matrix must be square");
        DV_REQUIRE(A->precision == DV_F64, DV_ERR_ARG, "the allocation-free PCG needs an FP64 matrix");
        DV_REQUIRE(A->n_rows <= kNoAllocMaxRows, DV_ERR_ARG,
                   "system larger than the allocation-free limit of 131072 rows; use dv_pcg_solve");
        DV_REQUIRE(max_iterations >= 0 && tol >= 0, DV_ERR_ARG, "bad iteration limit or tolerance");
        DV_REQUIRE(!A->zero_diag, DV_ERR_SINGULAR, "zero diagonal entry");
        dv_context *ctx = A->ctx;
        dv_ctx_check(ctx);
        const auto t0 = std::chrono::steady_clock::now();
        cudaStream_t st = ctx->stream;
        const int32_t n = A->n_rows;
        unsigned char *base = static_cast<unsigned char *>(scratch_address(ctx->device));
        unsigned *ticket = reinterpret_cast<unsigned *>(base);
        SolverScalars *sc = reinterpret_cast<SolverScalars *>(base + 16);
        double *partials = reinterpret_cast<double *>(base + kHeaderBytes);
        double *r = reinterpret_cast<double *>(base + kHeaderBytes + kPartialBytes);
        double *z = r + kNoAllocMaxRows, *p = z + kNoAllocMaxRows, *ap = p + kNoAllocMaxRows;
        // The ticket must start at zero; the scalars are written by k_na_init.
        DV_CUDA(cudaMemsetAsync(ticket, 0, 16, st));
        k_na_init<<<1, 1, 0, st>>>(sc, max_iterations);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        LaunchEnv e;
        e.ctx = ctx;
        e.stream = st;
        e.done = nullptr;
        e.partials = partials;
        e.ticket = ticket;
        e.max_blocks = std::min(kNoAllocMaxBlocks, ctx->num_sms * 16);
        // r = b - A x0, or r = b with x = 0
        if (use_x0) {
            OpResid<double> op{{}, d_b, r};
            launch_rows<double>(e, A, GatherVec<double, double>{d_x}, op);
        } else {
            DV_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, st));
            DV_CUDA(cudaMemcpyAsync(r, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, e.max_blocks));
        // M = 1/diag is formed on the fly from the diagonal the matrix already holds on the device.
        k_na_pcg_init<<<grid, kThreads, 0, st>>>(A->diag.as<double>(), r, z, p, n, sc, partials, ticket);
        DV_CUDA(cudaGetLastError());
        ctx->count();
        LaunchEnv ed = e;
        ed.done = &sc->done;
        SolverScalars h{};
        for (;;) {
            for (int k = 0; k < 8; ++k) {
                OpPcgAp op{p, ap, sc};
                launch_rows<double>(ed, A, GatherVec<double, double>{p}, op);
                k_na_update<<<grid, kThreads, 0, st>>>(A->diag.as<double>(), ap, p, d_x, r, z, n, tol, sc, partials,
                                                       ticket);
                DV_CUDA(cudaGetLastError());
                k_na_p<<<grid, kThreads, 0, st>>>(z, p, n, sc);
                DV_CUDA(cudaGetLastError());
                ctx->count(2);
            }
            DV_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
            DV_CUDA(cudaStreamSynchronize(st));
            if (h.done) break;
        }
        // relative residual of the returned x in FP64: z = b - A x (z is free now), ||b||, ||z||
        {
            OpResid<double> op{{}, d_b, z};
            launch_rows<double>(e, A, GatherVec<double, double>{d_x}, op);
            k_na_norms<<<grid, kThreads, 0, st>>>(d_b, z, n, sc, partials, ticket);
            DV_CUDA(cudaGetLastError());
            ctx->count();
            DV_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
            DV_CUDA(cudaStreamSynchronize(st));
        }
        if (stats) {
            stats->iterations = h.it;
            stats->converged = h.converged;
            stats->failed = h.failed;
            stats->reserved = 0;
            stats->residual_max = h.res_max;
            stats->residual_norm2 = h.res_norm2;
            stats->relative_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : (h.rr > 0 ? INFINITY : 0.0);
            stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}
