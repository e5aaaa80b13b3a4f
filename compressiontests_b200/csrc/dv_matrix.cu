// Context, matrix upload and the SpMV/SpMM entry points of libduvigpu.so.
#include "dv_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

static thread_local std::string g_last_error;
void dv_set_last_error(const std::string &m) { g_last_error = m; }

extern "C" DV_API const char *dv_last_error(void) { return g_last_error.c_str(); }
extern "C" DV_API int dv_version(void) { return 10000; }
extern "C" DV_API const char *dv_status_string(int s) {
    switch (s) {
        case DV_OK: return "ok";
        case DV_ERR_ARG: return "invalid argument";
        case DV_ERR_CUDA: return "CUDA error";
        case DV_ERR_NOT_INITIALIZED: return "not initialized";
        case DV_ERR_UNSUPPORTED: return "unsupported";
        case DV_ERR_NOMEM: return "out of memory";
        case DV_ERR_FORMAT: return "format error";
        case DV_ERR_NO_DEVICE: return "no CUDA device";
        case DV_ERR_SINGULAR: return "singular matrix";
        default: return "unknown status";
    }
}

void dv_ctx_check(dv_context *ctx) {
    DV_REQUIRE(ctx != nullptr, DV_ERR_NOT_INITIALIZED, "null context");
    DV_CUDA(cudaSetDevice(ctx->device));
}

extern "C" DV_API int dv_context_create(int device, dv_context **out) {
    return dv_guard([&] {
        DV_REQUIRE(out != nullptr, DV_ERR_ARG, "null output");
        *out = nullptr;
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        DV_REQUIRE(e == cudaSuccess && n > 0, DV_ERR_NO_DEVICE,
                   std::string("no usable CUDA device: ") + cudaGetErrorString(e));
        DV_REQUIRE(device >= 0 && device < n, DV_ERR_ARG, "device ordinal out of range");
        DV_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        DV_CUDA(cudaGetDeviceProperties(&prop, device));
        DV_REQUIRE(prop.major >= 10, DV_ERR_UNSUPPORTED, "this library is built for sm_100a (B200)");
        auto ctx = std::make_unique<dv_context>();
        ctx->device = device;
        ctx->num_sms = prop.multiProcessorCount;
        ctx->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
        DV_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->red.alloc(sizeof(double) * dvk::kMaxRed * ctx->num_sms * 16 + 64);
        *out = ctx.release();
    });
}

extern "C" DV_API int dv_context_destroy(dv_context *ctx) {
    return dv_guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ctx->red.release();
        cudaStreamDestroy(ctx->stream);
        delete ctx;
    });
}
extern "C" DV_API int dv_context_synchronize(dv_context *ctx) {
    return dv_guard([&] {
        dv_ctx_check(ctx);
        DV_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}
extern "C" DV_API void *dv_context_stream(dv_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
extern "C" DV_API int64_t dv_context_launch_count(const dv_context *ctx) { return ctx ? ctx->launches : -1; }

// ---------------------------------------------------------------------------
// matrix build
// ---------------------------------------------------------------------------
static void upload(DevMem &d, const void *h, size_t bytes, cudaStream_t s) {
    d.alloc(bytes);
    if (bytes) DV_CUDA(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, s));
}


static int pick_tpr(double mean_nnz) {
    if (mean_nnz < 6) return 4;
    if (mean_nnz < 20) return 8;
    if (mean_nnz < 48) return 16;
    return 32;
}

// Uploads the SoA arrays of encoding h and derives the device layouts; h is only read
// here (export reads the device arrays back), so callers keep it only while building.
void dv_upload_patterns(dv_matrix *m, const DuviPatternHost &P, const std::vector<double> &values, cudaStream_t s) {
    const int rec_bytes = m->precision == DV_F64 ? 32 : 16;
    const size_t ne = P.off.size();
    std::vector<unsigned char> recs(ne * rec_bytes, 0);
    for (size_t k = 0; k < ne; ++k) {
        unsigned char *r = recs.data() + k * rec_bytes;
        std::memcpy(r, &P.off[k], 4);
        for (int d = 0; d < P.group; ++d) {
            const double v = values[P.vi[k * P.group + d]];
            if (m->precision == DV_F64) std::memcpy(r + 8 + 8 * d, &v, 8);
            else { const float f = (float)v; std::memcpy(r + 4 + 4 * d, &f, 4); }
        }
    }
    upload(m->pat_start, P.start.data(), 4 * P.start.size(), s);
    upload(m->pat_rec, recs.data(), recs.size(), s);
    if (P.based) upload(m->pat_base, P.base.data(), 4 * P.base.size(), s);
    DV_CUDA(cudaStreamSynchronize(s));
    m->pat_ok = 1;
    m->pat_based = P.based;
    m->pat_shift = P.shift;
    m->pat_count = (int32_t)P.start.size() - 1;
    m->pat_entries = (int32_t)ne;
}

bool dv_set_grid(dv_matrix *m, const DuviGridHost &Gd, const std::vector<double> &values) {
    m->grid_lx = Gd.lx;
    m->grid_ly = Gd.ly;
    m->grid_lz = Gd.lz;
    m->grid_hot = Gd.hot;
    m->grid_all_hot = Gd.all_hot;
    m->grid_coef.resize(Gd.vi.size());
    for (size_t i = 0; i < Gd.vi.size(); ++i) m->grid_coef[i] = values[Gd.vi[i]];
    // the hex stencil's structure: equal values within each class, zeros where expected
    bool hex = true, seen[dvk::kHexClasses] = {};
    for (int i = 0; i < 243 && hex; ++i) {
        const int c = dvk::hex_class(i);
        const double v = m->grid_coef[i];
        if (c < 0) hex = v == 0.0 && !std::signbit(v);
        else if (!seen[c]) { seen[c] = true; m->grid_cls[c] = v; }
        else hex = v == m->grid_cls[c] && std::signbit(v) == std::signbit(m->grid_cls[c]);
    }
    m->grid_hex = hex ? 1 : 0;
    // FP64 runs the stencil with the hex structure only (the general FP64 stencil would hold 243
    // coefficients in registers); otherwise the node patterns stay
    m->grid_ok = m->grid_hex || m->precision == DV_F32;
    return m->grid_ok;
}

static void finish_duvi_upload(dv_matrix *m, const DuviHost &h, cudaStream_t s) {
    m->vi_bits = h.vi_bits;
    m->nblocks = (int64_t)h.col_idx.size();
    m->nuniq = (int64_t)h.values.size();
    upload(m->row_to_col, h.row_to_col.data(), 4 * h.row_to_col.size(), s);
    upload(m->row_to_dist, h.row_to_dist.data(), 4 * h.row_to_dist.size(), s);
    upload(m->col_idx, h.col_idx.data(), 4 * h.col_idx.size(), s);
    upload(m->dist, h.dist.data(), h.dist.size(), s);
    // value indices at their storage width
    size_t nnz = h.vidx.size();
    if (m->vi_bits == 8) {
        std::vector<uint8_t> v(nnz);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)nnz; ++i) v[i] = (uint8_t)h.vidx[i];
        upload(m->vidx, v.data(), nnz, s);
        DV_CUDA(cudaStreamSynchronize(s));
    } else if (m->vi_bits == 16) {
        std::vector<uint16_t> v(nnz);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)nnz; ++i) v[i] = (uint16_t)h.vidx[i];
        upload(m->vidx, v.data(), 2 * nnz, s);
        DV_CUDA(cudaStreamSynchronize(s));
    } else {
        upload(m->vidx, h.vidx.data(), 4 * nnz, s);
    }
    if (m->precision == DV_F64) {
        upload(m->values, h.values.data(), 8 * h.values.size(), s);
    } else {
        std::vector<float> f(h.values.size());
        for (size_t i = 0; i < f.size(); ++i) f[i] = (float)h.values[i];
        upload(m->values, f.data(), 4 * f.size(), s);
        DV_CUDA(cudaStreamSynchronize(s));
    }
    // most frequent block length picks the batch width of the decode loop
    {
        std::vector<int64_t> hist(257, 0);
        for (size_t r = 0; r + 1 < h.row_to_col.size(); ++r) {
            uint32_t di = h.row_to_dist[r];
            for (uint32_t bl = h.row_to_col[r]; bl < h.row_to_col[r + 1]; ++bl) {
                hist[h.dist[di] + 1]++;
                di += h.dist[di] + 1u;
            }
        }
        int mode = (int)(std::max_element(hist.begin(), hist.end()) - hist.begin());
        m->duvi_batch = (mode >= 9 && mode % 9 == 0) ? 9 : 4;
    }
    {   // lane-interleaved derived layout
        DuviLanesHost L;
        dv_build_duvi_lanes(h, m->n_rows, m->n_cols, m->precision == DV_F64 ? 8 : 4, L);
        m->lanes_group = L.group;
        m->lanes_scaled = L.scaled;
        m->lanes_shift = L.shift;
        m->lanes_tuples = L.tuples;
        m->lanes_stencil = L.stencil;
        if (L.stencil) {
            m->lanes_noff = (int32_t)L.offsets.size();
            upload(m->lanes_off, L.offsets.data(), 4 * L.offsets.size(), s);
            DV_CUDA(cudaStreamSynchronize(s));
        }
        if (L.tuples) {   // 4 values (zero-padded) per tuple, in the matrix precision
            const size_t ntup = L.tuple_vi.size() / L.group;
            if (m->precision == DV_F64) {
                std::vector<double> tv(4 * ntup, 0.0);
                for (size_t t = 0; t < ntup; ++t)
                    for (int d = 0; d < L.group; ++d) tv[4 * t + d] = h.values[L.tuple_vi[t * L.group + d]];
                upload(m->lanes_tup, tv.data(), 8 * tv.size(), s);
                DV_CUDA(cudaStreamSynchronize(s));
            } else {
                std::vector<float> tv(4 * ntup, 0.0f);
                for (size_t t = 0; t < ntup; ++t)
                    for (int d = 0; d < L.group; ++d) tv[4 * t + d] = (float)h.values[L.tuple_vi[t * L.group + d]];
                upload(m->lanes_tup, tv.data(), 4 * tv.size(), s);
                DV_CUDA(cudaStreamSynchronize(s));
            }
            m->lanes_ntup = (int32_t)ntup;
        }
        m->row_group = L.shift ? 1 : L.group;   // block products need identical columns
        m->lanes_groups = L.ngroups;
        m->lanes_bundles = L.nbundles;
        upload(m->lanes_meta, L.meta.data(), 4 * L.meta.size(), s);
        upload(m->lanes_dist, L.dist.data(), 4 * L.dist.size(), s);
        upload(m->lanes_vi, L.vi.data(), L.vi.size(), s);
        upload(m->lanes_cols, L.cols.data(), 4 * L.cols.size(), s);
        upload(m->lanes_nent, L.nent.data(), 4 * L.nent.size(), s);
        DV_CUDA(cudaStreamSynchronize(s));
        const size_t vs = m->precision == DV_F64 ? 8 : 4;
        m->lanes_bytes = (int64_t)(4 * L.meta.size() + 4 * L.dist.size() + L.vi.size() + 4 * L.cols.size() +
                                   4 * L.nent.size() + 4 * L.offsets.size() +
                                   vs * (L.tuples ? 4 * (size_t)m->lanes_ntup : h.values.size()));
        // the lane kernel is the default when rows come in node groups
        m->lanes_ok = 1;
        m->duvi_variant = L.group > 1 ? 1 : 0;
        const char *pe = getenv("DV_PATTERNS");   // DV_PATTERNS=0 keeps the lane layout (A/B comparisons)
        if (!(pe && pe[0] == '0')) {   // node patterns: records {offset, 3 values} in shared memory
            const int rec_bytes = m->precision == DV_F64 ? 32 : 16;
            DuviPatternHost P;
            dv_build_duvi_patterns(h, m->n_rows, m->n_cols, L.group, L.shift, 1024, (96 * 1024) / rec_bytes, P);
            if (P.ok) {
                upload(m->pat_id, P.id.data(), 2 * P.id.size(), s);
                dv_upload_patterns(m, P, h.values, s);
                m->duvi_variant = 2;
                const char *ge = getenv("DV_GRID");   // DV_GRID=0 keeps the node-pattern kernel (A/B comparisons)
                DuviGridHost Gd;
                if (!(ge && ge[0] == '0')) dv_build_duvi_grid(P, Gd);
                if (Gd.ok && dv_set_grid(m, Gd, h.values)) {
                    m->grid_nb = (int64_t)Gd.boundary.size();
                    upload(m->grid_bnode, Gd.boundary.data(), 4 * Gd.boundary.size(), s);
                    DV_CUDA(cudaStreamSynchronize(s));
                    m->duvi_variant = 3;
                }
            }
        }
    }
    std::vector<int32_t> b;
    dv_make_bundles(h, m->n_rows, m->vi_bits, b);
    m->nbundles = (int32_t)b.size() - 1;
    upload(m->bundles, b.data(), 4 * b.size(), s);
    DV_CUDA(cudaStreamSynchronize(s));
    const size_t vs = m->precision == DV_F64 ? 8 : 4;
    m->device_bytes = (int64_t)(m->nnz * (1 + m->vi_bits / 8) + 4 * m->nblocks + 8 * ((int64_t)m->n_rows + 1) +
                                vs * m->nuniq);
}

static dvk::LaunchEnv env_for(dv_context *ctx, const int *done = nullptr) {
    dvk::LaunchEnv e;
    e.ctx = ctx;
    e.stream = ctx->stream;
    e.done = done;
    e.ticket = reinterpret_cast<unsigned *>(ctx->red.as<char>());
    e.partials = reinterpret_cast<double *>(ctx->red.as<char>() + 64);
    e.max_blocks = ctx->num_sms * 16;
    return e;
}

// Project autotuner: time every launch shape of the SpMV on this matrix with
// CUDA events (FP32 or FP64 vectors as stored) and keep the fastest.  Runs once
// per matrix at upload; small matrices keep the heuristic choice.
static void autotune(dv_matrix *m) {
    const char *env = getenv("DV_AUTOTUNE");
    if (env && env[0] == '0') return;
    if (m->n_rows < 100000 || m->n_rows != m->n_cols) return;
    dv_context *ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    CountScope tuning(ctx, dv_context::kCountTuning);   // trial launches are not part of any solve
    const size_t vs = m->precision == DV_F64 ? 8 : 4;
    DevMem x(vs * (size_t)m->n_cols), y(vs * (size_t)m->n_rows);
    {   // a representative x: values of one sign and magnitude ~1 (1 + i/n)
        const int32_t nc = m->n_cols;
        if (m->precision == DV_F64) {
            std::vector<double> h(nc);
            for (int32_t i = 0; i < nc; ++i) h[i] = 1.0 + (double)i / nc;
            upload(x, h.data(), 8 * (size_t)nc, s);
        } else {
            std::vector<float> h(nc);
            for (int32_t i = 0; i < nc; ++i) h[i] = 1.0f + (float)i / nc;
            upload(x, h.data(), 4 * (size_t)nc, s);
        }
        DV_CUDA(cudaStreamSynchronize(s));
    }
    auto e = env_for(ctx);
    auto run = [&] {
        if (m->precision == DV_F64) {
            dvk::OpSpmv<double, double> op;
            op.y = y.as<double>();
            op.clear = 1;
            dvk::launch_rows<double>(e, m, dvk::GatherVec<double, double>{x.as<double>()}, op);
        } else {
            dvk::OpSpmv<float, float> op;
            op.y = y.as<float>();
            op.clear = 1;
            dvk::launch_rows<float>(e, m, dvk::GatherVec<float, float>{x.as<float>()}, op);
        }
    };
    // CSR: threads per row; DuVi: 4 / 9 = staged kernel with that batch width, 100 = lane kernel
    std::vector<int> cand = m->format == DV_FORMAT_CSR ? std::vector<int>{8, 16, 32} : std::vector<int>{4, 9};
    if (m->format == DV_FORMAT_DUVI && m->lanes_ok) cand.push_back(100);
    if (m->format == DV_FORMAT_DUVI && m->pat_ok) cand.push_back(200);
    if (m->format == DV_FORMAT_DUVI && m->grid_ok) cand.push_back(300);
    cudaEvent_t e0, e1;
    DV_CUDA(cudaEventCreate(&e0));
    DV_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    auto current = [&] {
        return m->format == DV_FORMAT_CSR ? m->csr_tpr
                                          : (m->duvi_variant == 3 ? 300 : m->duvi_variant == 2 ? 200
                                             : m->duvi_variant == 1 ? 100 : m->duvi_batch);
    };
    auto apply = [&](int v) {
        if (m->format == DV_FORMAT_CSR) m->csr_tpr = v;
        else if (v == 300) m->duvi_variant = 3;
        else if (v == 200) m->duvi_variant = 2;
        else if (v == 100) m->duvi_variant = 1;
        else { m->duvi_variant = 0; m->duvi_batch = v; }
    };
    int best_v = current();
    for (int v : cand) {
        apply(v);
        run();
        DV_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < 3; ++k) run();
        DV_CUDA(cudaEventRecord(e1, s));
        DV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const char *vb = getenv("DV_AUTOTUNE_VERBOSE");
        if (vb && vb[0] == '1')
            fprintf(stderr, "autotune %s n=%d variant=%d: %.4f ms\n", m->format == DV_FORMAT_CSR ? "csr" : "duvi",
                    m->n_rows, v, ms / 3);
        if (ms < best) { best = ms; best_v = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(best_v);
}

void dv_autotune(dv_matrix *m) { autotune(m); }

dv_matrix *dv_matrix_build(dv_context *ctx, const dv_csr_host &a, int format, int precision, int vi_bits, double tol,
                           const DuviHost *encoded) {
    dv_ctx_check(ctx);
    dv_check_csr(a);
    DV_REQUIRE(format == DV_FORMAT_CSR || format == DV_FORMAT_DUVI, DV_ERR_ARG, "unknown format");
    DV_REQUIRE(precision == DV_F64 || precision == DV_F32, DV_ERR_ARG, "precision must be DV_F64 or DV_F32");
    auto m = std::make_unique<dv_matrix>();
    m->ctx = ctx;
    m->n_rows = a.n_rows;
    m->n_cols = a.n_cols;
    m->nnz = a.rowptr[a.n_rows];
    m->format = format;
    m->precision = precision;
    cudaStream_t s = ctx->stream;
    if (format == DV_FORMAT_CSR) {
        upload(m->rowptr, a.rowptr, 4 * ((size_t)a.n_rows + 1), s);
        upload(m->col, a.col, 4 * (size_t)m->nnz, s);
        if (precision == DV_F64) {
            upload(m->val, a.val, 8 * (size_t)m->nnz, s);
            DV_CUDA(cudaStreamSynchronize(s));
        } else {
            std::vector<float> f(m->nnz);
            for (int64_t i = 0; i < m->nnz; ++i) f[i] = (float)a.val[i];
            upload(m->val, f.data(), 4 * (size_t)m->nnz, s);
            DV_CUDA(cudaStreamSynchronize(s));
        }
        m->csr_tpr = pick_tpr(a.n_rows ? (double)m->nnz / a.n_rows : 1.0);
        m->row_group = dv_csr_row_group(a);
        m->device_bytes = m->nnz * (4 + (precision == DV_F64 ? 8 : 4)) + 4 * ((int64_t)a.n_rows + 1);
    } else {
        if (encoded) {
            finish_duvi_upload(m.get(), *encoded, s);
        } else {
            DuviHost h;
            dv_encode_duvi(a, tol, vi_bits, h);
            finish_duvi_upload(m.get(), h, s);
        }
    }
    if (a.n_rows == a.n_cols) {
        dv_extract_diag(a, m->host_diag);
        m->zero_diag = std::any_of(m->host_diag.begin(), m->host_diag.end(), [](double d) { return d == 0.0; });
        upload(m->diag, m->host_diag.data(), 8 * m->host_diag.size(), s);
        DV_CUDA(cudaStreamSynchronize(s));
    }
    autotune(m.get());
    return m.release();
}

namespace {
// rowptr monotone within [0, nnz], columns strictly increasing and in range; bad[0] = 1 otherwise
__global__ void k_check_csr(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int32_t n, int32_t n_cols,
                            int *__restrict__ bad) {
    const int32_t nnz = rp[n];
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        bool ok = rp[i] >= 0 && rp[i + 1] >= rp[i] && rp[i + 1] <= nnz;
        for (int32_t k = rp[i]; ok && k < rp[i + 1]; ++k)
            ok = col[k] >= 0 && col[k] < n_cols && (k == rp[i] || col[k] > col[k - 1]);
        if (!ok) atomicOr(bad, 1);
    }
}
}  // namespace

extern "C" DV_API int dv_matrix_create_duvi_device(dv_context *ctx, int32_t n_rows, int32_t n_cols,
                                                   const int32_t *d_rowptr, const int32_t *d_col, const double *d_val,
                                                   int32_t precision, int32_t value_index_bits, double dedup_tol,
                                                   dv_matrix **out) {
    return dv_guard([&] {
        DV_REQUIRE(out && d_rowptr, DV_ERR_ARG, "null argument");
        DV_REQUIRE(n_rows > 0 && n_cols > 0, DV_ERR_ARG, "empty matrix");
        DV_REQUIRE(precision == DV_F64 || precision == DV_F32, DV_ERR_ARG, "precision must be DV_F64 or DV_F32");
        dv_ctx_check(ctx);
        cudaStream_t s = ctx->stream;
        int32_t nnz = 0;
        DV_CUDA(cudaMemcpyAsync(&nnz, d_rowptr + n_rows, 4, cudaMemcpyDeviceToHost, s));
        DV_CUDA(cudaStreamSynchronize(s));
        DV_REQUIRE(nnz >= 0 && (nnz == 0 || (d_col && d_val)), DV_ERR_FORMAT, "bad row offsets or null col/val");
        {
            DevMem bad(16);
            DV_CUDA(cudaMemsetAsync(bad.p, 0, 16, s));
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_rows + 255) / 256, (int64_t)ctx->num_sms * 16));
            k_check_csr<<<grid, 256, 0, s>>>(d_rowptr, d_col, n_rows, n_cols, bad.as<int>());
            DV_CUDA(cudaGetLastError());
            int hb = 0;
            DV_CUDA(cudaMemcpyAsync(&hb, bad.p, 4, cudaMemcpyDeviceToHost, s));
            DV_CUDA(cudaStreamSynchronize(s));
            DV_REQUIRE(!hb, DV_ERR_FORMAT, "not a CSR matrix with strictly increasing columns in range");
        }
        auto m = std::make_unique<dv_matrix>();
        m->ctx = ctx;
        m->n_rows = n_rows;
        m->n_cols = n_cols;
        m->nnz = nnz;
        m->format = DV_FORMAT_DUVI;
        m->precision = precision;
        dv_duvi_from_device_csr(m.get(), d_rowptr, d_col, d_val, value_index_bits, dedup_tol);
        autotune(m.get());
        *out = m.release();
    });
}

extern "C" DV_API int dv_matrix_create_csr(dv_context *ctx, const dv_csr_host *a, int32_t precision, dv_matrix **out) {
    return dv_guard([&] {
        DV_REQUIRE(a && out, DV_ERR_ARG, "null argument");
        *out = dv_matrix_build(ctx, *a, DV_FORMAT_CSR, precision, 0, 0.0);
    });
}

extern "C" DV_API int dv_matrix_create_duvi(dv_context *ctx, const dv_csr_host *a, int32_t precision,
                                            int32_t value_index_bits, double dedup_tol, dv_matrix **out) {
    return dv_guard([&] {
        DV_REQUIRE(a && out, DV_ERR_ARG, "null argument");
        *out = dv_matrix_build(ctx, *a, DV_FORMAT_DUVI, precision, value_index_bits, dedup_tol);
    });
}

extern "C" DV_API int dv_matrix_create_duvi_soa(dv_context *ctx, int32_t n_rows, int32_t n_cols, const uint32_t *rc,
                                                const uint32_t *rd, const uint32_t *ci, int64_t nblocks,
                                                const uint8_t *dist, int64_t nnz, const void *vidx, int32_t bits,
                                                const double *values, int64_t nuniq, int32_t precision,
                                                dv_matrix **out) {
    return dv_guard([&] {
        dv_ctx_check(ctx);
        DV_REQUIRE(out && rc && rd && (nblocks == 0 || ci) && (nnz == 0 || (dist && vidx)) && (nuniq == 0 || values),
                   DV_ERR_ARG, "null argument");
        DV_REQUIRE(bits == 8 || bits == 16 || bits == 32, DV_ERR_ARG, "value_index_bits must be 8, 16 or 32");
        DV_REQUIRE(precision == DV_F64 || precision == DV_F32, DV_ERR_ARG, "bad precision");
        DV_REQUIRE(n_rows >= 0 && n_cols >= 0 && rc[0] == 0 && rd[0] == 0 && rc[n_rows] == (uint64_t)nblocks &&
                       rd[n_rows] == (uint64_t)nnz, DV_ERR_FORMAT, "inconsistent DuVi offsets");
        auto m = std::make_unique<dv_matrix>();
        m->ctx = ctx;
        m->n_rows = n_rows;
        m->n_cols = n_cols;
        m->nnz = nnz;
        m->format = DV_FORMAT_DUVI;
        m->precision = precision;
        DuviHost h;
        h.row_to_col.assign(rc, rc + n_rows + 1);
        h.row_to_dist.assign(rd, rd + n_rows + 1);
        h.col_idx.assign(ci, ci + nblocks);
        h.dist.assign(dist, dist + nnz);
        h.vidx.resize(nnz);
        for (int64_t i = 0; i < nnz; ++i)
            h.vidx[i] = bits == 8 ? ((const uint8_t *)vidx)[i] : bits == 16 ? ((const uint16_t *)vidx)[i] : ((const uint32_t *)vidx)[i];
        h.values.assign(values, values + nuniq);
        h.vi_bits = bits;
        // validate the walk of every row (no read outside the arrays on the device)
        for (int32_t r = 0; r < n_rows; ++r) {
            DV_REQUIRE(rc[r + 1] >= rc[r] && rd[r + 1] >= rd[r], DV_ERR_FORMAT, "offsets not monotone");
            uint64_t di = rd[r];
            for (uint32_t b = rc[r]; b < rc[r + 1]; ++b) {
                DV_REQUIRE(di < rd[r + 1], DV_ERR_FORMAT, "block runs past its row");
                uint64_t c = ci[b];
                uint64_t end = di + dist[di] + 1;
                DV_REQUIRE(end <= rd[r + 1], DV_ERR_FORMAT, "block runs past its row");
                DV_REQUIRE(c < (uint64_t)n_cols, DV_ERR_FORMAT, "column out of range");
                for (uint64_t k = di + 1; k < end; ++k) {
                    c += dist[k] + 1u;
                    DV_REQUIRE(c < (uint64_t)n_cols, DV_ERR_FORMAT, "column out of range");
                }
                di = end;
            }
            DV_REQUIRE(di == rd[r + 1], DV_ERR_FORMAT, "row entries not covered by its blocks");
        }
        for (int64_t i = 0; i < nnz; ++i) DV_REQUIRE(h.vidx[i] < (uint64_t)nuniq, DV_ERR_FORMAT, "value index out of range");
        m->nuniq = nuniq;
        finish_duvi_upload(m.get(), h, ctx->stream);
        *out = m.release();
    });
}

extern "C" DV_API int dv_matrix_get_info(const dv_matrix *m, dv_matrix_info *info) {
    return dv_guard([&] {
        DV_REQUIRE(m && info, DV_ERR_ARG, "null argument");
        info->n_rows = m->n_rows;
        info->n_cols = m->n_cols;
        info->nnz = m->nnz;
        info->nblocks = m->format == DV_FORMAT_DUVI ? m->nblocks : 0;
        info->nuniq = m->format == DV_FORMAT_DUVI ? m->nuniq : 0;
        info->format = m->format;
        info->precision = m->precision;
        info->value_index_bits = m->format == DV_FORMAT_DUVI ? m->vi_bits : 0;
        info->kernel_variant = m->format == DV_FORMAT_HEX ? 400 : m->format == DV_FORMAT_TRILINEAR ? 500
                               : m->format == DV_FORMAT_CSR ? m->csr_tpr
                               : (m->duvi_variant == 3 ? 300 + m->lanes_group
                                  : m->duvi_variant == 2 ? 200 + m->lanes_group
                                  : m->duvi_variant == 1 ? 100 + m->lanes_group : m->duvi_batch);
        info->device_bytes = m->device_bytes;
        info->row_group = m->row_group;
        info->reserved = 0;
    });
}

extern "C" DV_API int dv_matrix_export_duvi(const dv_matrix *m, uint32_t *rc, uint32_t *rd, uint32_t *ci, uint8_t *dist,
                                            uint32_t *vidx, double *values) {
    return dv_guard([&] {
        DV_REQUIRE(m != nullptr, DV_ERR_ARG, "null matrix");
        DV_REQUIRE(m->format == DV_FORMAT_DUVI, DV_ERR_UNSUPPORTED, "not a DuVi matrix");
        // Read back what the device holds (not the host copy), widening the indices.
        dv_ctx_check(m->ctx);
        cudaStream_t s = m->ctx->stream;
        if (rc) DV_CUDA(cudaMemcpyAsync(rc, m->row_to_col.p, 4 * ((size_t)m->n_rows + 1), cudaMemcpyDeviceToHost, s));
        if (rd) DV_CUDA(cudaMemcpyAsync(rd, m->row_to_dist.p, 4 * ((size_t)m->n_rows + 1), cudaMemcpyDeviceToHost, s));
        if (ci) DV_CUDA(cudaMemcpyAsync(ci, m->col_idx.p, 4 * (size_t)m->nblocks, cudaMemcpyDeviceToHost, s));
        if (dist) DV_CUDA(cudaMemcpyAsync(dist, m->dist.p, (size_t)m->nnz, cudaMemcpyDeviceToHost, s));
        std::vector<unsigned char> raw;
        if (vidx) {
            raw.resize((size_t)m->nnz * (m->vi_bits / 8));
            DV_CUDA(cudaMemcpyAsync(raw.data(), m->vidx.p, raw.size(), cudaMemcpyDeviceToHost, s));
        }
        std::vector<unsigned char> tab((size_t)m->nuniq * (m->precision == DV_F64 ? 8 : 4));
        if (values && !tab.empty()) DV_CUDA(cudaMemcpyAsync(tab.data(), m->values.p, tab.size(), cudaMemcpyDeviceToHost, s));
        DV_CUDA(cudaStreamSynchronize(s));
        if (vidx)
            for (int64_t i = 0; i < m->nnz; ++i)
                vidx[i] = m->vi_bits == 8 ? raw[i] : m->vi_bits == 16 ? ((uint16_t *)raw.data())[i] : ((uint32_t *)raw.data())[i];
        if (values)
            for (int64_t i = 0; i < m->nuniq; ++i)
                values[i] = m->precision == DV_F64 ? ((double *)tab.data())[i] : (double)((float *)tab.data())[i];
    });
}

extern "C" DV_API int dv_matrix_destroy(dv_matrix *m) {
    return dv_guard([&] {
        if (!m) return;
        cudaSetDevice(m->ctx->device);
        cudaStreamSynchronize(m->ctx->stream);
        delete m;
    });
}

// ---------------------------------------------------------------------------
// products
// ---------------------------------------------------------------------------
dvk::LaunchEnv dv_default_env(dv_context *ctx) { return env_for(ctx); }

static void spmv_device(dv_matrix *m, const void *x, void *y, int vprec, int clear) {
    auto e = env_for(m->ctx);
    if (m->precision == DV_F64) {
        DV_REQUIRE(vprec == DV_F64, DV_ERR_ARG, "FP64 matrix needs FP64 vectors");
        dvk::OpSpmv<double, double> op;
        op.y = static_cast<double *>(y);
        op.clear = clear;
        dvk::launch_rows<double>(e, m, dvk::GatherVec<double, double>{static_cast<const double *>(x)}, op);
    } else {
        DV_REQUIRE(vprec == DV_F32, DV_ERR_ARG, "FP32 matrix needs FP32 vectors");
        dvk::OpSpmv<float, float> op;
        op.y = static_cast<float *>(y);
        op.clear = clear;
        dvk::launch_rows<float>(e, m, dvk::GatherVec<float, float>{static_cast<const float *>(x)}, op);
    }
}

extern "C" DV_API int dv_spmv_device(dv_matrix *m, const void *x, void *y, int32_t vprec, int32_t clear) {
    return dv_guard([&] {
        DV_REQUIRE(m && x && y, DV_ERR_ARG, "null argument");
        dv_ctx_check(m->ctx);
        spmv_device(m, x, y, vprec, clear);
    });
}

extern "C" DV_API int dv_residual_device(dv_matrix *m, const void *b, const void *x, void *r, int32_t vprec) {
    return dv_guard([&] {
        DV_REQUIRE(m && b && x && r, DV_ERR_ARG, "null argument");
        dv_ctx_check(m->ctx);
        auto e = env_for(m->ctx);
        if (m->precision == DV_F64) {
            DV_REQUIRE(vprec == DV_F64, DV_ERR_ARG, "FP64 matrix needs FP64 vectors");
            dvk::OpResid<double> op{{}, static_cast<const double *>(b), static_cast<double *>(r)};
            dvk::launch_rows<double>(e, m, dvk::GatherVec<double, double>{static_cast<const double *>(x)}, op);
        } else {
            DV_REQUIRE(vprec == DV_F32, DV_ERR_ARG, "FP32 matrix needs FP32 vectors");
            dvk::OpResid<float> op{{}, static_cast<const float *>(b), static_cast<float *>(r)};
            dvk::launch_rows<float>(e, m, dvk::GatherVec<float, float>{static_cast<const float *>(x)}, op);
        }
    });
}

extern "C" DV_API int dv_spmv(dv_matrix *m, const double *x, double *y, int32_t clear) {
    return dv_guard([&] {
        DV_REQUIRE(m && x && y, DV_ERR_ARG, "null argument");
        dv_ctx_check(m->ctx);
        cudaStream_t s = m->ctx->stream;
        const size_t vs = m->precision == DV_F64 ? 8 : 4;
        DevMem dx(vs * (size_t)m->n_cols), dy(vs * (size_t)m->n_rows);
        if (m->precision == DV_F64) {
            DV_CUDA(cudaMemcpyAsync(dx.p, x, 8 * (size_t)m->n_cols, cudaMemcpyHostToDevice, s));
            if (!clear) DV_CUDA(cudaMemcpyAsync(dy.p, y, 8 * (size_t)m->n_rows, cudaMemcpyHostToDevice, s));
            spmv_device(m, dx.p, dy.p, DV_F64, clear);
            DV_CUDA(cudaMemcpyAsync(y, dy.p, 8 * (size_t)m->n_rows, cudaMemcpyDeviceToHost, s));
        } else {
            std::vector<float> hx(x, x + m->n_cols), hy(m->n_rows);
            if (!clear) for (int32_t i = 0; i < m->n_rows; ++i) hy[i] = (float)y[i];
            DV_CUDA(cudaMemcpyAsync(dx.p, hx.data(), 4 * hx.size(), cudaMemcpyHostToDevice, s));
            DV_CUDA(cudaMemcpyAsync(dy.p, hy.data(), 4 * hy.size(), cudaMemcpyHostToDevice, s));
            spmv_device(m, dx.p, dy.p, DV_F32, clear);
            DV_CUDA(cudaMemcpyAsync(hy.data(), dy.p, 4 * hy.size(), cudaMemcpyDeviceToHost, s));
            DV_CUDA(cudaStreamSynchronize(s));
            for (int32_t i = 0; i < m->n_rows; ++i) y[i] = hy[i];
        }
        DV_CUDA(cudaStreamSynchronize(s));
    });
}
