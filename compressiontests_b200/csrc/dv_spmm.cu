// Multi-vector product Y = A X for k right-hand sides (row-interleaved n x k),
// reading the matrix once per 128 columns.  The kernels are the block products
// of dv_block.cuh (one warp per node group, lanes over right-hand sides).
#include "dv_block.cuh"

template <class T>
static void spmm(dv_matrix *m, int32_t k, const T *X, T *Y, int clear) {
    dvk::LaunchEnv e = dv_default_env(m->ctx);
    for (int32_t j0 = 0; j0 < k; j0 += dvb::kMaxCols) {
        const int kc = std::min<int32_t>(dvb::kMaxCols, k - j0);
        dvb::launch_bprod<T>(e, m, kc, dvb::BGatherVec<T, T>{X + j0, k}, dvb::BEpiSpmm<T>{Y + j0, k, clear, {}});
    }
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
