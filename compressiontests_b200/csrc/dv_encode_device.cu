// DuVi encoding of a device-resident CSR matrix, on the device.
//
// The arrays equal the host encoder's (dv_encode_duvi, the reference's FromDokRowMajor,
// OpenCLDuViGeometricMultigridSolver.cs:753-851) bit for bit:
//  - blocks ("DU"): one thread per row walks its columns with the reference's block rule
//    (a block ends when the gap - 1 reaches 256 or it holds 255 following entries,
//    :779-789); a first pass counts the blocks of every row, a scan places them;
//  - value indices ("VI"): the values are numbered in CSR order by the reference's
//    dictionary (ToleranceComparer, DuViCompressedSparseMatrix.cs:168-174).  A radix sort of
//    (bit pattern, position) finds every distinct bit pattern and its first position; the
//    distinct patterns, in order of first occurrence, pass through the dictionary on the host
//    (that order inserts the keys exactly where the sequential walk does) and every entry
//    takes its pattern's key.  When the dictionary says a lookup could depend on insertion
//    time, all values are numbered on the host instead.
// The node-pattern layout (groups of 3 rows with one column list) and the grid-stencil layout
// derived from it are built on the device as well: a signature per group (the host builder's
// hash of its column offsets and value indices), first-occurrence numbering by sort, and an
// entry-by-entry check of every group against its pattern's first group.  Nothing of the
// matrix passes through host memory except the distinct values and the pattern tables.
#include "dv_kernels.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

using namespace dvk;

namespace {

constexpr int kT = 256;
inline int blocks_for(int64_t n, dv_context *ctx) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, (int64_t)ctx->num_sms * 32));
}

// ---- blocks ----------------------------------------------------------------
__global__ void k_du_count(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int32_t n,
                           uint32_t *__restrict__ nb) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t from = rp[i], to = rp[i + 1];
        uint32_t b = 0;
        for (int32_t j = from; j < to; ++j) {
            ++b;
            int cnt = 0;
            for (; j + 1 < to && cnt < 255; ++j) {
                if (col[j + 1] - col[j] - 1 < 256) ++cnt;
                else break;
            }
        }
        nb[i] = b;
    }
}

__global__ void k_du_fill(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int32_t n,
                          const uint32_t *__restrict__ row_to_col, uint32_t *__restrict__ row_to_dist,
                          uint32_t *__restrict__ col_idx, uint8_t *__restrict__ dist) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t from = rp[i], to = rp[i + 1];
        row_to_dist[i] = (uint32_t)from;
        if (i == n - 1) row_to_dist[n] = (uint32_t)to;
        uint32_t b = row_to_col[i];
        for (int32_t j = from; j < to; ++j) {
            const int32_t begin = j;
            int cnt = 0;
            col_idx[b++] = (uint32_t)col[j];
            for (; j + 1 < to && cnt < 255; ++j) {
                const int32_t diff = col[j + 1] - col[j] - 1;
                if (diff < 256) {
                    ++cnt;
                    dist[j + 1] = (uint8_t)diff;
                } else {
                    break;
                }
            }
            dist[begin] = (uint8_t)cnt;
        }
    }
}

// ---- value numbering ---------------------------------------------------------
__global__ void k_bits(const double *__restrict__ val, int64_t n, unsigned long long *__restrict__ key,
                       uint32_t *__restrict__ pos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        key[i] = (unsigned long long)__double_as_longlong(val[i]);
        pos[i] = (uint32_t)i;
    }
}
// 1 where a run of equal keys starts (sorted keys)
template <class K>
__global__ void k_heads(const K *__restrict__ key, int64_t n, uint32_t *__restrict__ head) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}
// at each run start: the run's first (smallest) position and its key; seg1 = run number + 1
template <class K>
__global__ void k_run_first(const K *__restrict__ key, const uint32_t *__restrict__ pos, const uint32_t *__restrict__ head,
                            const uint32_t *__restrict__ seg1, int64_t n, uint32_t *__restrict__ first,
                            K *__restrict__ run_key) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (head[i]) {
            first[seg1[i] - 1] = pos[i];
            run_key[seg1[i] - 1] = key[i];
        }
}
// rank of each run in order of first occurrence
__global__ void k_rank(const uint32_t *__restrict__ run_of_rank, int64_t nr, uint32_t *__restrict__ rank) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nr; r += (int64_t)gridDim.x * blockDim.x)
        rank[run_of_rank[r]] = (uint32_t)r;
}
template <class K>
__global__ void k_gather_runs(const uint32_t *__restrict__ run_of_rank, const K *__restrict__ run_key, int64_t nr,
                              K *__restrict__ out) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nr; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = run_key[run_of_rank[r]];
}
// out[pos[i]] = value_of_rank[rank[run of i]]
__global__ void k_scatter_runs(const uint32_t *__restrict__ pos, const uint32_t *__restrict__ seg1,
                               const uint32_t *__restrict__ rank, const uint32_t *__restrict__ value_of_rank, int64_t n,
                               uint32_t *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[pos[i]] = value_of_rank[rank[seg1[i] - 1]];
}
template <class T>
__global__ void k_narrow(const uint32_t *__restrict__ v, int64_t n, T *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (T)v[i];
}
__global__ void k_diag(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, const double *__restrict__ val,
                       int32_t n, double *__restrict__ d) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (col[k] == i) v = val[k];
        d[i] = v;
    }
}

// ---- node patterns -------------------------------------------------------------
// groups of 3 rows with one column list; bad[0] set otherwise
// groups of 3 rows with one column list: row d's columns equal row 0's plus shift * d
// (shift 1: the trilinear transfers, component d coupling to component d); bad[0] set otherwise
__global__ void k_group_check(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int64_t ng, int shift,
                              int *__restrict__ bad) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r0 = (int32_t)(3 * g);
        const int32_t len = rp[r0 + 1] - rp[r0];
        bool ok = rp[r0 + 2] - rp[r0 + 1] == len && rp[r0 + 3] - rp[r0 + 2] == len;
        for (int32_t e = 0; ok && e < len; ++e)
            ok = col[rp[r0 + 1] + e] == col[rp[r0] + e] + shift && col[rp[r0 + 2] + e] == col[rp[r0] + e] + 2 * shift;
        if (!ok) atomicOr(bad, 1);
    }
}
// the column the offsets of group g count from: its first row (square, unshifted operators) or
// its first column (0 for an empty group), as in the host builder
__device__ __forceinline__ int64_t group_origin(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int64_t g,
                                                bool based) {
    const int32_t r0 = (int32_t)(3 * g);
    if (!based) return r0;
    return rp[r0 + 1] > rp[r0] ? col[rp[r0]] : 0;
}
__global__ void k_group_base(const int32_t *__restrict__ rp, const int32_t *__restrict__ col, int64_t ng,
                             uint32_t *__restrict__ base) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x)
        base[g] = (uint32_t)group_origin(rp, col, g, true);
}
// signature of a group: the host builder's FNV-1a hash of its entry count and, per entry, the
// column offset from the group's origin and the 3 value indices
__global__ void k_group_sig(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                            const uint32_t *__restrict__ vidx, int64_t ng, int based,
                            unsigned long long *__restrict__ sig, uint32_t *__restrict__ gid) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r0 = (int32_t)(3 * g);
        const int64_t b0 = group_origin(rp, col, g, based);
        const int32_t len = rp[r0 + 1] - rp[r0];
        unsigned long long x = 1469598103934665603ull ^ (unsigned long long)(4 * (int64_t)len);
        for (int32_t e = 0; e < len; ++e) {
            x = (x ^ (unsigned long long)((int64_t)col[rp[r0] + e] - b0)) * 1099511628211ull;
            for (int d = 0; d < 3; ++d) x = (x ^ (unsigned long long)vidx[rp[r0 + d] + e]) * 1099511628211ull;
        }
        sig[g] = x;
        gid[g] = (uint32_t)g;
    }
}
// every group equal to its pattern's first group, entry by entry; bad[0] set otherwise
__global__ void k_group_verify(const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                               const uint32_t *__restrict__ vidx, const uint16_t *__restrict__ pid,
                               const uint32_t *__restrict__ rep, int64_t ng, int based, int *__restrict__ bad) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = rep[pid[g]];
        const int32_t r0 = (int32_t)(3 * g), q0 = (int32_t)(3 * q);
        const int64_t b0 = group_origin(rp, col, g, based), c0 = group_origin(rp, col, q, based);
        const int32_t len = rp[r0 + 1] - rp[r0];
        bool ok = rp[q0 + 1] - rp[q0] == len;
        for (int32_t e = 0; ok && e < len; ++e) {
            ok = (int64_t)col[rp[r0] + e] - b0 == (int64_t)col[rp[q0] + e] - c0;
            for (int d = 0; d < 3 && ok; ++d) ok = vidx[rp[r0 + d] + e] == vidx[rp[q0 + d] + e];
        }
        if (!ok) atomicOr(bad, 1);
    }
}
__global__ void k_pattern_ids(const uint32_t *__restrict__ gid, const uint32_t *__restrict__ seg1,
                              const uint32_t *__restrict__ rank, int64_t ng, uint16_t *__restrict__ pid,
                              unsigned *__restrict__ count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ng; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = rank[seg1[i] - 1];
        pid[gid[i]] = (uint16_t)p;
        atomicAdd(count + p, 1u);
    }
}
// groups that the grid stencil leaves to their pattern records (flag 1)
__global__ void k_grid_flags(const uint16_t *__restrict__ pid, int64_t ng, int32_t lx, int32_t ly, int32_t lz, int hot,
                             uint32_t *__restrict__ flag, unsigned *__restrict__ inner_other) {
    const int64_t lxy = (int64_t)lx * ly;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ix = g % lx, iy = (g / lx) % ly, iz = g / lxy;
        const bool inner = ix >= 1 && ix <= lx - 2 && iy >= 1 && iy <= ly - 2 && iz >= 1 && iz <= lz - 2;
        const bool stencil = inner && pid[g] == hot;
        flag[g] = stencil ? 0u : 1u;
        if (inner && !stencil) atomicAdd(inner_other, 1u);
    }
}

template <class Kt, class Vt>
void sort_pairs(cudaStream_t s, const Kt *kin, Kt *kout, const Vt *vin, Vt *vout, int64_t n, int end_bit) {
    size_t bytes = 0;
    DV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, (int)n, 0, end_bit, s));
    DevMem tmp(bytes);
    DV_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, kin, kout, vin, vout, (int)n, 0, end_bit, s));
    DV_CUDA(cudaStreamSynchronize(s));   // tmp is released on return
}
void inclusive_sum(cudaStream_t s, const uint32_t *in, uint32_t *out, int64_t n) {
    size_t bytes = 0;
    DV_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, (int)n, s));
    DevMem tmp(bytes);
    DV_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, bytes, in, out, (int)n, s));
    DV_CUDA(cudaStreamSynchronize(s));
}
template <class T>
void to_host(std::vector<T> &h, const void *d, size_t n, cudaStream_t s) {
    h.resize(n);
    if (n) DV_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
}
template <class T>
void to_device(DevMem &d, const std::vector<T> &h, cudaStream_t s) {
    d.alloc(sizeof(T) * h.size());
    if (!h.empty()) DV_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    DV_CUDA(cudaStreamSynchronize(s));
}

// Runs of equal keys of a sorted (key, position) sequence, numbered by first position:
// rank[run] and, per rank, the run's key and first position.
struct Runs {
    DevMem seg1, rank, run_of_rank, first_sorted;
    int64_t nr = 0;
};
template <class K>
void number_runs(dv_context *ctx, const K *key, const uint32_t *pos, int64_t n, Runs &R, DevMem &key_by_rank) {
    cudaStream_t s = ctx->stream;
    DevMem head(4 * (size_t)n);
    R.seg1.alloc(4 * (size_t)n);
    k_heads<K><<<blocks_for(n, ctx), kT, 0, s>>>(key, n, head.as<uint32_t>());
    DV_CUDA(cudaGetLastError());
    inclusive_sum(s, head.as<uint32_t>(), R.seg1.as<uint32_t>(), n);
    uint32_t nr = 0;
    DV_CUDA(cudaMemcpyAsync(&nr, R.seg1.as<uint32_t>() + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
    R.nr = nr;
    DevMem first(4 * (size_t)nr), run_key(sizeof(K) * (size_t)nr), runs(4 * (size_t)nr);
    k_run_first<K><<<blocks_for(n, ctx), kT, 0, s>>>(key, pos, head.as<uint32_t>(), R.seg1.as<uint32_t>(), n,
                                                     first.as<uint32_t>(), run_key.as<K>());
    DV_CUDA(cudaGetLastError());
    {   // runs in order of first position
        std::vector<uint32_t> iota(nr);
        for (uint32_t r = 0; r < nr; ++r) iota[r] = r;
        DevMem runs_in;
        to_device(runs_in, iota, s);
        R.first_sorted.alloc(4 * (size_t)nr);
        R.run_of_rank.alloc(4 * (size_t)nr);
        sort_pairs<uint32_t, uint32_t>(s, first.as<uint32_t>(), R.first_sorted.as<uint32_t>(), runs_in.as<uint32_t>(),
                                       R.run_of_rank.as<uint32_t>(), nr, 32);
    }
    R.rank.alloc(4 * (size_t)nr);
    k_rank<<<blocks_for(nr, ctx), kT, 0, s>>>(R.run_of_rank.as<uint32_t>(), nr, R.rank.as<uint32_t>());
    DV_CUDA(cudaGetLastError());
    key_by_rank.alloc(sizeof(K) * (size_t)nr);
    k_gather_runs<K><<<blocks_for(nr, ctx), kT, 0, s>>>(R.run_of_rank.as<uint32_t>(), run_key.as<K>(), nr,
                                                       key_by_rank.as<K>());
    DV_CUDA(cudaGetLastError());
    DV_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

// Builds the DuVi SoA, value table, diagonal and derived layouts of m from device CSR.
void dv_duvi_from_device_csr(dv_matrix *m, const int32_t *rp, const int32_t *col, const double *val, int force_bits,
                             double tol) {
    dv_context *ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    const int32_t n = m->n_rows;
    const int64_t nnz = m->nnz;
    DV_REQUIRE(nnz < (int64_t)INT32_MAX, DV_ERR_FORMAT, "the device encoder takes fewer than 2^31 entries");
    // blocks
    DevMem nb(4 * ((size_t)n + 1));
    k_du_count<<<blocks_for(n, ctx), kT, 0, s>>>(rp, col, n, nb.as<uint32_t>() + 1);
    DV_CUDA(cudaGetLastError());
    DV_CUDA(cudaMemsetAsync(nb.p, 0, 4, s));
    m->row_to_col.alloc(4 * ((size_t)n + 1));
    inclusive_sum(s, nb.as<uint32_t>(), m->row_to_col.as<uint32_t>(), (int64_t)n + 1);
    uint32_t nblocks = 0;
    DV_CUDA(cudaMemcpyAsync(&nblocks, m->row_to_col.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
    m->nblocks = nblocks;
    m->row_to_dist.alloc(4 * ((size_t)n + 1));
    m->col_idx.alloc(4 * (size_t)nblocks);
    m->dist.alloc((size_t)nnz);
    k_du_fill<<<blocks_for(n, ctx), kT, 0, s>>>(rp, col, n, m->row_to_col.as<uint32_t>(), m->row_to_dist.as<uint32_t>(),
                                                 m->col_idx.as<uint32_t>(), m->dist.as<uint8_t>());
    DV_CUDA(cudaGetLastError());
    // value numbering
    DevMem vidx32(4 * (size_t)nnz);
    std::vector<double> keys;
    {
        DevMem kin(8 * (size_t)nnz), kout(8 * (size_t)nnz), pin(4 * (size_t)nnz), pout(4 * (size_t)nnz);
        using K = unsigned long long;
        k_bits<<<blocks_for(nnz, ctx), kT, 0, s>>>(val, nnz, kin.as<K>(), pin.as<uint32_t>());
        DV_CUDA(cudaGetLastError());
        sort_pairs<K, uint32_t>(s, kin.as<K>(), kout.as<K>(), pin.as<uint32_t>(), pout.as<uint32_t>(), nnz, 64);
        kin.release();
        pin.release();
        Runs R;
        DevMem bits_by_rank;
        number_runs<K>(ctx, kout.as<K>(), pout.as<uint32_t>(), nnz, R, bits_by_rank);
        std::vector<double> distinct;
        to_host(distinct, bits_by_rank.p, (size_t)R.nr, s);
        std::vector<uint32_t> key_of(R.nr);
        if (dv_number_distinct(distinct.data(), R.nr, tol, key_of.data(), keys)) {
            DevMem dkey;
            to_device(dkey, key_of, s);
            k_scatter_runs<<<blocks_for(nnz, ctx), kT, 0, s>>>(pout.as<uint32_t>(), R.seg1.as<uint32_t>(),
                                                                 R.rank.as<uint32_t>(), dkey.as<uint32_t>(), nnz,
                                                                 vidx32.as<uint32_t>());
            DV_CUDA(cudaGetLastError());
            DV_CUDA(cudaStreamSynchronize(s));
        } else {   // a lookup could depend on insertion time: number every value on the host
            std::vector<double> hv;
            to_host(hv, val, (size_t)nnz, s);
            std::vector<uint32_t> hi(nnz);
            keys = dv_number_values(hv.data(), nnz, tol, hi.data());
            DV_CUDA(cudaMemcpyAsync(vidx32.p, hi.data(), 4 * (size_t)nnz, cudaMemcpyHostToDevice, s));
            DV_CUDA(cudaStreamSynchronize(s));
        }
    }
    const int64_t nu = (int64_t)keys.size();
    int bits = nu <= 256 ? 8 : (nu <= 65536 ? 16 : 32);
    if (force_bits != 0) {
        DV_REQUIRE(force_bits == 8 || force_bits == 16 || force_bits == 32, DV_ERR_ARG,
                   "value_index_bits must be 0, 8, 16 or 32");
        DV_REQUIRE(force_bits >= bits, DV_ERR_FORMAT, "too many distinct values for the requested index width");
        bits = force_bits;
    }
    m->vi_bits = bits;
    m->nuniq = nu;
    if (bits == 32) {
        m->vidx.alloc(4 * (size_t)nnz);
        DV_CUDA(cudaMemcpyAsync(m->vidx.p, vidx32.p, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, s));
    } else if (bits == 16) {
        m->vidx.alloc(2 * (size_t)nnz);
        k_narrow<uint16_t><<<blocks_for(nnz, ctx), kT, 0, s>>>(vidx32.as<uint32_t>(), nnz, m->vidx.as<uint16_t>());
    } else {
        m->vidx.alloc((size_t)nnz);
        k_narrow<uint8_t><<<blocks_for(nnz, ctx), kT, 0, s>>>(vidx32.as<uint32_t>(), nnz, m->vidx.as<uint8_t>());
    }
    DV_CUDA(cudaGetLastError());
    if (m->precision == DV_F64) {
        to_device(m->values, keys, s);
    } else {
        std::vector<float> f(keys.begin(), keys.end());
        to_device(m->values, f, s);
    }
    // bundles of the staged kernel (from the row offsets of both streams)
    {
        DuviHost hb;
        to_host(hb.row_to_col, m->row_to_col.p, (size_t)n + 1, s);
        to_host(hb.row_to_dist, m->row_to_dist.p, (size_t)n + 1, s);
        std::vector<int32_t> b;
        dv_make_bundles(hb, n, bits, b);
        m->nbundles = (int32_t)b.size() - 1;
        to_device(m->bundles, b, s);
    }
    m->duvi_batch = 4;
    m->duvi_variant = 0;
    m->lanes_group = 1;
    m->row_group = 1;
    // diagonal
    if (n == m->n_cols) {
        m->diag.alloc(8 * (size_t)n);
        k_diag<<<blocks_for(n, ctx), kT, 0, s>>>(rp, col, val, n, m->diag.as<double>());
        DV_CUDA(cudaGetLastError());
        to_host(m->host_diag, m->diag.p, (size_t)n, s);
        m->zero_diag = std::any_of(m->host_diag.begin(), m->host_diag.end(), [](double d) { return d == 0.0; });
    }
    const size_t vs = m->precision == DV_F64 ? 8 : 4;
    m->device_bytes = (int64_t)(nnz * (1 + bits / 8) + 4 * (int64_t)nblocks + 8 * ((int64_t)n + 1) + vs * nu);
    // node patterns: groups of 3 rows with one column list (shifted by the row's index in the
    // group for the transfers), at most 1024 patterns; offsets from the group's first row on square
    // unshifted operators, else from its first column
    const char *pe = getenv("DV_PATTERNS");
    if ((pe && pe[0] == '0') || n % 3 != 0 || n == 0) return;
    const int64_t ng = n / 3;
    DevMem bad(16);
    int hbad = 0, shift = -1;
    for (int sh : {0, 1}) {
        DV_CUDA(cudaMemsetAsync(bad.p, 0, 16, s));
        k_group_check<<<blocks_for(ng, ctx), kT, 0, s>>>(rp, col, ng, sh, bad.as<int>());
        DV_CUDA(cudaGetLastError());
        DV_CUDA(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, s));
        DV_CUDA(cudaStreamSynchronize(s));
        if (!hbad) { shift = sh; break; }
    }
    if (shift < 0) return;
    const int based = shift || n != m->n_cols;
    DV_CUDA(cudaMemsetAsync(bad.p, 0, 16, s));
    using K = unsigned long long;
    DevMem sig(8 * (size_t)ng), gid(4 * (size_t)ng), sig_s(8 * (size_t)ng), gid_s(4 * (size_t)ng);
    k_group_sig<<<blocks_for(ng, ctx), kT, 0, s>>>(rp, col, vidx32.as<uint32_t>(), ng, based, sig.as<K>(),
                                                   gid.as<uint32_t>());
    DV_CUDA(cudaGetLastError());
    sort_pairs<K, uint32_t>(s, sig.as<K>(), sig_s.as<K>(), gid.as<uint32_t>(), gid_s.as<uint32_t>(), ng, 64);
    Runs R;
    DevMem sig_by_rank;
    number_runs<K>(ctx, sig_s.as<K>(), gid_s.as<uint32_t>(), ng, R, sig_by_rank);
    const int64_t npat = R.nr;
    if (npat > 1024) return;
    DevMem pid(2 * (size_t)ng), count(4 * (size_t)npat);
    DV_CUDA(cudaMemsetAsync(count.p, 0, 4 * (size_t)npat, s));
    k_pattern_ids<<<blocks_for(ng, ctx), kT, 0, s>>>(gid_s.as<uint32_t>(), R.seg1.as<uint32_t>(), R.rank.as<uint32_t>(),
                                                     ng, pid.as<uint16_t>(), count.as<unsigned>());
    DV_CUDA(cudaGetLastError());
    // R.first_sorted[p] = the first group of pattern p
    k_group_verify<<<blocks_for(ng, ctx), kT, 0, s>>>(rp, col, vidx32.as<uint32_t>(), pid.as<uint16_t>(),
                                                      R.first_sorted.as<uint32_t>(), ng, based, bad.as<int>());
    DV_CUDA(cudaGetLastError());
    DV_CUDA(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
    if (hbad) return;
    // pattern table from each pattern's first group
    std::vector<uint32_t> rep;
    to_host(rep, R.first_sorted.p, (size_t)npat, s);
    std::vector<int32_t> hrp(4);
    DuviPatternHost P;
    P.group = 3;
    P.ngroups = ng;
    P.start.assign(1, 0);
    for (int64_t p = 0; p < npat; ++p) {
        const int32_t r0 = (int32_t)(3 * (int64_t)rep[p]);
        int64_t b0 = r0;
        DV_CUDA(cudaMemcpyAsync(hrp.data(), rp + r0, 16, cudaMemcpyDeviceToHost, s));
        DV_CUDA(cudaStreamSynchronize(s));
        const int32_t len = hrp[1] - hrp[0];
        std::vector<int32_t> c(len);
        std::vector<uint32_t> v(3 * (size_t)len);
        if (len) {
            DV_CUDA(cudaMemcpyAsync(c.data(), col + hrp[0], 4 * (size_t)len, cudaMemcpyDeviceToHost, s));
            for (int d = 0; d < 3; ++d)
                DV_CUDA(cudaMemcpyAsync(v.data() + (size_t)d * len, vidx32.as<uint32_t>() + hrp[d], 4 * (size_t)len,
                                        cudaMemcpyDeviceToHost, s));
            DV_CUDA(cudaStreamSynchronize(s));
        }
        if (based) b0 = len ? c[0] : 0;
        for (int32_t e = 0; e < len; ++e) {
            P.off.push_back((int32_t)(c[e] - b0));
            for (int d = 0; d < 3; ++d) P.vi.push_back(v[(size_t)d * len + e]);
        }
        P.start.push_back((uint32_t)P.off.size());
    }
    const int rec_bytes = m->precision == DV_F64 ? 32 : 16;
    if ((int64_t)P.off.size() > (96 * 1024) / rec_bytes) return;
    P.ok = 1;
    P.shift = shift;
    P.based = based;   // the per-group origins stay on the device (k_group_base)
    dv_upload_patterns(m, P, keys, s);
    if (based) {
        m->pat_base.alloc(4 * (size_t)ng);
        k_group_base<<<blocks_for(ng, ctx), kT, 0, s>>>(rp, col, ng, m->pat_base.as<uint32_t>());
        DV_CUDA(cudaGetLastError());
    }
    m->pat_id = std::move(pid);
    m->lanes_group = 3;
    m->row_group = 3;
    m->duvi_variant = 2;
    // grid stencil: the most frequent pattern, its geometry, the groups left to their records
    std::vector<unsigned> cnt;
    to_host(cnt, count.p, (size_t)npat, s);
    const int hot = (int)(std::max_element(cnt.begin(), cnt.end()) - cnt.begin());
    int32_t lx, ly, lz;
    const char *ge = getenv("DV_GRID");
    if ((ge && ge[0] == '0') || !dv_grid_geometry(P, hot, ng, lx, ly, lz)) return;
    DevMem flag(4 * (size_t)ng), other(16), bsel(4 * (size_t)ng), nsel(16);
    DV_CUDA(cudaMemsetAsync(other.p, 0, 16, s));
    k_grid_flags<<<blocks_for(ng, ctx), kT, 0, s>>>(m->pat_id.as<uint16_t>(), ng, lx, ly, lz, hot, flag.as<uint32_t>(),
                                                    other.as<unsigned>());
    DV_CUDA(cudaGetLastError());
    {
        cub::CountingInputIterator<uint32_t> it(0);
        size_t bytes = 0;
        DV_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, it, flag.as<uint32_t>(), bsel.as<uint32_t>(),
                                           nsel.as<int>(), (int)ng, s));
        DevMem tmp(bytes);
        DV_CUDA(cub::DeviceSelect::Flagged(tmp.p, bytes, it, flag.as<uint32_t>(), bsel.as<uint32_t>(), nsel.as<int>(),
                                           (int)ng, s));
        DV_CUDA(cudaStreamSynchronize(s));
    }
    int nb_sel = 0;
    unsigned inner_other = 0;
    DV_CUDA(cudaMemcpyAsync(&nb_sel, nsel.p, 4, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaMemcpyAsync(&inner_other, other.p, 4, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
    DuviGridHost Gd;
    Gd.ok = 1;
    Gd.lx = lx;
    Gd.ly = ly;
    Gd.lz = lz;
    Gd.hot = hot;
    Gd.all_hot = inner_other == 0;
    const uint32_t s0 = P.start[hot];
    Gd.vi.assign(P.vi.begin() + 3 * (size_t)s0, P.vi.begin() + 3 * (size_t)(s0 + 81));
    if (dv_set_grid(m, Gd, keys)) {
        m->grid_nb = nb_sel;
        m->grid_bnode.alloc(4 * (size_t)std::max(nb_sel, 1));
        if (nb_sel) DV_CUDA(cudaMemcpyAsync(m->grid_bnode.p, bsel.p, 4 * (size_t)nb_sel, cudaMemcpyDeviceToDevice, s));
        DV_CUDA(cudaStreamSynchronize(s));
        m->duvi_variant = 3;
    }
}
