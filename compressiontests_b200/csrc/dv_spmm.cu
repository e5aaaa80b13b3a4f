// Multi-vector product Y = A X for k right-hand sides (row-interleaved n x k),
// reading the matrix once per call.  One warp per row: the row's entries are
// decoded once (warp-uniform loads) and lanes own right-hand-side columns, so
// each gather of X(col, :) is a contiguous, coalesced k-vector.
#include "dv_kernels.cuh"

using namespace dvk;

dvk::LaunchEnv dv_default_env(dv_context *ctx);

template <class T>
__global__ void __launch_bounds__(kThreads) k_spmm_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                                       const T *__restrict__ va, int32_t n, int32_t k,
                                                       const T *__restrict__ X, T *__restrict__ Y, int clear) {
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += nw) {
        const int32_t s0 = __ldg(rp + row), s1 = __ldg(rp + row + 1);
        for (int32_t j0 = 0; j0 < k; j0 += 128) {
            T acc[4] = {0, 0, 0, 0};
            for (int32_t e = s0; e < s1; ++e) {
                const T a = __ldg(va + e);
                const T *xr = X + (size_t)__ldg(ci + e) * k;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    int32_t j = j0 + lane + 32 * u;
                    if (j < k) acc[u] += a * __ldg(xr + j);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int32_t j = j0 + lane + 32 * u;
                if (j < k) {
                    T *yp = Y + (size_t)row * k + j;
                    *yp = clear ? acc[u] : *yp + acc[u];
                }
            }
        }
    }
}

template <class VI, class T>
__global__ void __launch_bounds__(kThreads) k_spmm_duvi(DuviArgs A, int32_t n, int32_t k, const T *__restrict__ X,
                                                        T *__restrict__ Y, int clear) {
    const int lane = threadIdx.x & 31;
    const int32_t nw = (gridDim.x * blockDim.x) >> 5;
    const T *tab = static_cast<const T *>(A.values);
    const VI *vi = static_cast<const VI *>(A.vidx);
    for (int32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += nw) {
        const uint32_t b0 = __ldg(A.row_to_col + row), b1 = __ldg(A.row_to_col + row + 1);
        const uint32_t d0 = __ldg(A.row_to_dist + row);
        for (int32_t j0 = 0; j0 < k; j0 += 128) {
            T acc[4] = {0, 0, 0, 0};
            uint32_t di = d0;
            for (uint32_t b = b0; b < b1; ++b) {
                uint32_t c = __ldg(A.col_idx + b);
                const int cnt = __ldg(A.dist + di);
                for (int q = 0;; ++q) {
                    const T a = __ldg(tab + __ldg(vi + di));
                    const T *xr = X + (size_t)c * k;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        int32_t j = j0 + lane + 32 * u;
                        if (j < k) acc[u] += a * __ldg(xr + j);
                    }
                    ++di;
                    if (q == cnt) break;
                    c += __ldg(A.dist + di) + 1u;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int32_t j = j0 + lane + 32 * u;
                if (j < k) {
                    T *yp = Y + (size_t)row * k + j;
                    *yp = clear ? acc[u] : *yp + acc[u];
                }
            }
        }
    }
}

template <class T>
static void spmm(dv_matrix *m, int32_t k, const T *X, T *Y, int clear) {
    dv_context *ctx = m->ctx;
    int64_t warps = m->n_rows;
    int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((warps * 32 + kThreads - 1) / kThreads, ctx->num_sms * 16));
    if (m->format == DV_FORMAT_CSR) {
        k_spmm_csr<T><<<blocks, kThreads, 0, ctx->stream>>>(m->rowptr.as<int32_t>(), m->col.as<int32_t>(),
                                                             static_cast<const T *>(m->val.p), m->n_rows, k, X, Y, clear);
    } else {
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
        if (m->vi_bits == 8) k_spmm_duvi<uint8_t, T><<<blocks, kThreads, 0, ctx->stream>>>(a, m->n_rows, k, X, Y, clear);
        else if (m->vi_bits == 16) k_spmm_duvi<uint16_t, T><<<blocks, kThreads, 0, ctx->stream>>>(a, m->n_rows, k, X, Y, clear);
        else k_spmm_duvi<uint32_t, T><<<blocks, kThreads, 0, ctx->stream>>>(a, m->n_rows, k, X, Y, clear);
    }
    DV_CUDA(cudaGetLastError());
    ctx->count();
}

extern "C" DV_API int dv_spmm_device(dv_matrix *m, int32_t k, const void *X, void *Y, int32_t vprec, int32_t clear) {
    return dv_guard([&] {
        DV_REQUIRE(m && X && Y && k >= 1, DV_ERR_ARG, "null argument or k < 1");
        dv_ctx_check(m->ctx);
        if (m->precision == DV_F64) {
            DV_REQUIRE(vprec == DV_F64, DV_ERR_ARG, "FP64 matrix needs FP64 vectors");
            spmm<double>(m, k, static_cast<const double *>(X), static_cast<double *>(Y), clear);
        } else {
            DV_REQUIRE(vprec == DV_F32, DV_ERR_ARG, "FP32 matrix needs FP32 vectors");
            spmm<float>(m, k, static_cast<const float *>(X), static_cast<float *>(Y), clear);
        }
    });
}
