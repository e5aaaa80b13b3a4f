// Host-side setup of libduvigpu.so: DuVi encoding, row bundles, Jacobi and
// coarse-solve preparation, Gauss-Seidel orderings, structured hex workload
// generator.  None of this runs inside a solve.
#include "dv_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>

#ifdef _OPENMP
#include <omp.h>
#endif

// ---------------------------------------------------------------------------
// .NET Dictionary<double,int> semantics used by the DuVi value dedup
// ---------------------------------------------------------------------------
// double.GetHashCode (.NET 8): zeros and NaNs normalised, then the two 32-bit
// halves xor-ed.
static inline int32_t net_double_hash(double x) {
    uint64_t bits;
    std::memcpy(&bits, &x, 8);
    const uint64_t sign = 0x8000000000000000ull, pinf = 0x7FF0000000000000ull;
    if (((bits - 1) & ~sign) >= pinf) bits &= pinf;
    return (int32_t)(uint32_t)bits ^ (int32_t)(uint32_t)(bits >> 32);
}

namespace {
// Chained hash table with the bucket-chain discipline of System.Collections.
// Generic.Dictionary: new entries go to the head of their chain, lookups walk
// newest-first and accept the first entry whose 32-bit hash code matches and
// whose comparer says Equals (DuViCompressedSparseMatrix.cs:168-174).
struct NetDoubleDict {
    double tol;
    std::vector<double> keys;
    std::vector<int32_t> codes, next;
    std::vector<int32_t> buckets;   // head entry + 1, 0 = empty
    uint32_t mask = 0;
    explicit NetDoubleDict(double t) : tol(t) { rehash(1024); }
    int32_t code(double x) const {
        return tol > 0 ? net_double_hash(std::nearbyint(x / (2 * tol))) : net_double_hash(x);
    }
    bool eq(double s, double k) const {
        return tol > 0 ? std::fabs(s - k) < tol : (s == k || (std::isnan(s) && std::isnan(k)));
    }
    void rehash(size_t nb) {
        buckets.assign(nb, 0);
        mask = (uint32_t)nb - 1;
        for (size_t i = 0; i < keys.size(); ++i) {
            uint32_t b = (uint32_t)codes[i] & mask;
            next[i] = buckets[b] - 1;
            buckets[b] = (int32_t)i + 1;
        }
    }
    int32_t find_or_insert(double v) {
        int32_t c = code(v);
        uint32_t b = (uint32_t)c & mask;
        for (int32_t i = buckets[b] - 1; i >= 0; i = next[i])
            if (codes[i] == c && eq(keys[i], v)) return i;
        int32_t id = (int32_t)keys.size();
        keys.push_back(v);
        codes.push_back(c);
        next.push_back(buckets[b] - 1);
        buckets[b] = id + 1;
        if (keys.size() > buckets.size()) rehash(buckets.size() * 2);
        return id;
    }
};
}  // namespace

namespace {
// Exact-bit-pattern numbering of one chunk's values in first-occurrence order
// (open addressing, grows at half load).
struct BitsTable {
    std::vector<uint64_t> key;
    std::vector<int32_t> id;
    uint64_t mask = 0;
    uint64_t last_bits = 0;
    int32_t last_id = -1;
    BitsTable() { resize(256); }
    void resize(size_t cap) {
        std::vector<uint64_t> k(cap, 0);
        std::vector<int32_t> d(cap, -1);
        const uint64_t m = cap - 1;
        for (size_t i = 0; i < key.size(); ++i)
            if (id[i] >= 0) {
                uint64_t j = slot(key[i], m);
                while (d[j] >= 0) j = (j + 1) & m;
                k[j] = key[i];
                d[j] = id[i];
            }
        key.swap(k);
        id.swap(d);
        mask = m;
    }
    static uint64_t slot(uint64_t b, uint64_t m) { return ((b ^ (b >> 31)) * 0x9E3779B97F4A7C15ull >> 17) & m; }
    uint32_t number(double v, std::vector<double> &distinct) {
        uint64_t b;
        std::memcpy(&b, &v, 8);
        if (b == last_bits && last_id >= 0) return (uint32_t)last_id;
        uint64_t j = slot(b, mask);
        while (id[j] >= 0 && key[j] != b) j = (j + 1) & mask;
        int32_t r = id[j];
        if (r < 0) {
            r = (int32_t)distinct.size();
            key[j] = b;
            id[j] = r;
            distinct.push_back(v);
            if (2 * distinct.size() > key.size()) resize(2 * key.size());
        }
        last_bits = b;
        last_id = r;
        return (uint32_t)r;
    }
};

// Value numbering of FromDokRowMajor: find_or_insert of every entry, in CSR
// order, into the Dictionary above; returns the keys (the values table).
// In parallel: each chunk of consecutive entries numbers its distinct bit
// patterns locally; the chunks' distinct values then pass through the
// dictionary in chunk order, which inserts every key at the same entry as the
// sequential walk; each entry finally takes its value's key.  That equals the
// sequential walk when no distinct value is within the tolerance of two keys
// of its hash code: a value's key is then the one matching key of its code,
// whenever it is looked up.  Otherwise a lookup can depend on the keys
// inserted before it, and the sequential walk runs instead; so it does for
// non-finite values under a tolerance (they equal nothing, not even
// themselves, so every occurrence becomes a key).
}  // namespace

// True when none of the values could match two keys of its hash code, so that a lookup
// returns the same key whenever it happens (the parallel numberings rely on it).
static bool unambiguous(const NetDoubleDict &map, const double *vals, int64_t n) {
    std::vector<std::pair<int32_t, int32_t>> ck(map.keys.size());   // (code, key) for codes held by 2+ keys
    for (size_t k = 0; k < ck.size(); ++k) ck[k] = {map.codes[k], (int32_t)k};
    std::sort(ck.begin(), ck.end());
    std::vector<std::pair<int32_t, std::vector<int32_t>>> shared;
    for (size_t k = 0; k < ck.size();) {
        size_t e = k + 1;
        while (e < ck.size() && ck[e].first == ck[k].first) ++e;
        if (e - k > 1) {
            shared.push_back({ck[k].first, {}});
            for (size_t q = k; q < e; ++q) shared.back().second.push_back(ck[q].second);
        }
        k = e;
    }
    if (shared.empty()) return true;
    for (int64_t i = 0; i < n; ++i) {
        const double v = vals[i];
        const int32_t c = map.code(v);
        auto it = std::lower_bound(shared.begin(), shared.end(), c,
                                   [](const std::pair<int32_t, std::vector<int32_t>> &x, int32_t y) { return x.first < y; });
        if (it == shared.end() || it->first != c) continue;
        int hits = 0;
        for (int32_t k : it->second) hits += map.eq(v, map.keys[k]) ? 1 : 0;
        if (hits > 1) return false;
    }
    return true;
}

std::vector<double> dv_number_values(const double *val, int64_t nnz, double tol, uint32_t *vidx) {
    auto sequential = [&] {
        NetDoubleDict map(tol);
        for (int64_t i = 0; i < nnz; ++i) vidx[i] = (uint32_t)map.find_or_insert(val[i]);
        return map.keys;
    };
#ifdef _OPENMP
    const int T = omp_get_max_threads();
#else
    const int T = 1;
#endif
    if (T <= 1 || nnz < (int64_t)1 << 16) return sequential();
    std::vector<std::vector<double>> distinct(T);
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        BitsTable tab;
        const int64_t b = nnz * t / T, e = nnz * (t + 1) / T;
        for (int64_t i = b; i < e; ++i) vidx[i] = tab.number(val[i], distinct[t]);
    }
    bool nonfinite = false;
    for (int t = 0; t < T; ++t)
        for (double v : distinct[t]) nonfinite = nonfinite || !std::isfinite(v);
    if (nonfinite && tol > 0) return sequential();
    NetDoubleDict map(tol);
    std::vector<std::vector<uint32_t>> key(T);
    for (int t = 0; t < T; ++t) {
        key[t].reserve(distinct[t].size());
        for (double v : distinct[t]) key[t].push_back((uint32_t)map.find_or_insert(v));
    }
    for (int t = 0; t < T; ++t)
        if (!unambiguous(map, distinct[t].data(), (int64_t)distinct[t].size())) return sequential();
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        const int64_t b = nnz * t / T, e = nnz * (t + 1) / T;
        const uint32_t *kt = key[t].data();
        for (int64_t i = b; i < e; ++i) vidx[i] = kt[vidx[i]];
    }
    return map.keys;
}

bool dv_number_distinct(const double *distinct, int64_t nd, double tol, uint32_t *key_of, std::vector<double> &keys) {
    for (int64_t i = 0; i < nd; ++i)
        if (tol > 0 && !std::isfinite(distinct[i])) return false;
    NetDoubleDict map(tol);
    for (int64_t i = 0; i < nd; ++i) key_of[i] = (uint32_t)map.find_or_insert(distinct[i]);
    if (!unambiguous(map, distinct, nd)) return false;
    keys = std::move(map.keys);
    return true;
}

// FromDokRowMajor (OpenCLDuViGeometricMultigridSolver.cs:753-851).  The block
// ("DU") part is independent per row and built in parallel; the value ("VI")
// part is sequential in CSR order because first occurrence defines the index.
void dv_encode_duvi(const dv_csr_host &a, double tol, int force_bits, DuviHost &h) {
    const int32_t n = a.n_rows;
    const int64_t nnz = a.rowptr[n];
    DV_REQUIRE(nnz <= 0xFFFFFFFFll, DV_ERR_FORMAT, "DuVi offsets are 32-bit");
    std::vector<int64_t> row_blocks(n + 1, 0);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        int32_t from = a.rowptr[i], to = a.rowptr[i + 1];
        int64_t nb = 0;
        for (int32_t j = from; j < to; ++j) {
            ++nb;
            int cnt = 0;
            for (; j + 1 < to && cnt < 255; ++j) {
                if (a.col[j + 1] - a.col[j] - 1 < 256) ++cnt;
                else break;
            }
        }
        row_blocks[i + 1] = nb;
    }
    for (int32_t i = 0; i < n; ++i) row_blocks[i + 1] += row_blocks[i];
    h.row_to_col.resize(n + 1);
    h.row_to_dist.resize(n + 1);
    h.col_idx.resize(row_blocks[n]);
    h.dist.assign(nnz, 0);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i <= n; ++i) {
        h.row_to_col[i] = (uint32_t)row_blocks[i];
        h.row_to_dist[i] = (uint32_t)(i < n ? a.rowptr[i] : nnz);
        if (i == n) continue;
        int32_t from = a.rowptr[i], to = a.rowptr[i + 1];
        int64_t b = row_blocks[i];
        for (int32_t j = from; j < to; ++j) {
            int64_t begin = j;
            int cnt = 0;
            h.col_idx[b++] = (uint32_t)a.col[j];
            for (; j + 1 < to && cnt < 255; ++j) {
                int32_t diff = a.col[j + 1] - a.col[j] - 1;
                if (diff < 256) { ++cnt; h.dist[j + 1] = (uint8_t)diff; }
                else break;
            }
            h.dist[begin] = (uint8_t)cnt;
        }
    }
    h.vidx.resize(nnz);
    h.values = dv_number_values(a.val, nnz, tol, h.vidx.data());
    int64_t nu = (int64_t)h.values.size();
    int bits = nu <= 256 ? 8 : (nu <= 65536 ? 16 : 32);
    if (force_bits != 0) {
        DV_REQUIRE(force_bits == 8 || force_bits == 16 || force_bits == 32, DV_ERR_ARG,
                   "value_index_bits must be 0, 8, 16 or 32");
        DV_REQUIRE(force_bits >= bits, DV_ERR_FORMAT, "too many distinct values for the requested index width");
        bits = force_bits;
    }
    h.vi_bits = bits;
}

void dv_check_csr(const dv_csr_host &a) {
    DV_REQUIRE(a.n_rows >= 0 && a.n_cols >= 0, DV_ERR_ARG, "negative dimensions");
    DV_REQUIRE(a.rowptr != nullptr, DV_ERR_ARG, "null rowptr");
    DV_REQUIRE(a.rowptr[0] == 0, DV_ERR_FORMAT, "rowptr[0] must be 0");
    const int64_t nnz = a.rowptr[a.n_rows];
    DV_REQUIRE(nnz == 0 || (a.col && a.val), DV_ERR_ARG, "null col/val");
    // rows checked in parallel; the first bad row (lowest index) names the error
    int32_t bad_row = INT32_MAX;
    int bad_kind = 0;
#pragma omp parallel for schedule(static) reduction(min : bad_row)
    for (int32_t i = 0; i < a.n_rows; ++i) {
        bool ok = a.rowptr[i + 1] >= a.rowptr[i] && a.rowptr[i + 1] <= nnz;   // past nnz: not monotone later
        for (int32_t k = a.rowptr[i]; ok && k < a.rowptr[i + 1]; ++k)
            ok = a.col[k] >= 0 && a.col[k] < a.n_cols && (k == a.rowptr[i] || a.col[k] > a.col[k - 1]);
        if (!ok) bad_row = std::min(bad_row, i);
    }
    if (bad_row != INT32_MAX) {
        const int32_t i = bad_row;
        if (a.rowptr[i + 1] < a.rowptr[i] || a.rowptr[i + 1] > nnz) bad_kind = 1;
        else
            for (int32_t k = a.rowptr[i]; k < a.rowptr[i + 1] && !bad_kind; ++k)
                bad_kind = (a.col[k] < 0 || a.col[k] >= a.n_cols) ? 2 : (k > a.rowptr[i] && a.col[k] <= a.col[k - 1]) ? 3 : 0;
        DV_REQUIRE(bad_kind != 1, DV_ERR_FORMAT, "rowptr not monotone");
        DV_REQUIRE(bad_kind != 2, DV_ERR_FORMAT, "column index out of range");
        DV_REQUIRE(false, DV_ERR_FORMAT, "columns must be strictly increasing within a row");
    }
}

void dv_make_bundles(const DuviHost &h, int32_t n_rows, int vi_bits, std::vector<int32_t> &bundles) {
    (void)vi_bits;
    bundles.clear();
    int32_t r = 0;
    while (r < n_rows) {
        bundles.push_back(r);
        int32_t r1 = r + 1;
        while (r1 < n_rows && r1 - r < kBundleRows) {
            uint32_t bytes = h.row_to_dist[r1 + 1] - h.row_to_dist[r];
            uint32_t blocks = h.row_to_col[r1 + 1] - h.row_to_col[r];
            if (bytes > (uint32_t)kBundleBytes || blocks > (uint32_t)kBundleBlocks) break;
            ++r1;
        }
        r = r1;
    }
    bundles.push_back(n_rows);
}

// Group size: g consecutive rows with the same block structure (same block
// count, same gap bytes) whose block columns are either identical (the dofs of
// one node in a stiffness matrix) or shifted by the row's index in the group
// (shift = 1: component d of a node couples to component d of its neighbours,
// as in the trilinear transfers).  Returns g (1 if none) and sets shift.
static int detect_group(const DuviHost &h, int32_t n, int &shift) {
    for (int sh : {0, 1})
        for (int g : {3, 2}) {
            if (n % g != 0 || n == 0) continue;
            int ok = 1;
#pragma omp parallel for schedule(static) reduction(min : ok)
            for (int32_t gi = 0; gi < n / g; ++gi) {
                const int32_t r0 = gi * g;
                const uint32_t nb = h.row_to_col[r0 + 1] - h.row_to_col[r0], ne = h.row_to_dist[r0 + 1] - h.row_to_dist[r0];
                for (int d = 1; d < g && ok; ++d) {
                    const int32_t r = r0 + d;
                    if (h.row_to_col[r + 1] - h.row_to_col[r] != nb || h.row_to_dist[r + 1] - h.row_to_dist[r] != ne) {
                        ok = 0;
                        break;
                    }
                    if (std::memcmp(&h.dist[h.row_to_dist[r]], &h.dist[h.row_to_dist[r0]], ne) != 0) ok = 0;
                    for (uint32_t b = 0; b < nb && ok; ++b)
                        if (h.col_idx[h.row_to_col[r] + b] != h.col_idx[h.row_to_col[r0] + b] + (uint32_t)(sh * d)) ok = 0;
                }
            }
            if (ok) {
                shift = sh;
                return g;
            }
        }
    shift = 0;
    return 1;
}

int dv_csr_row_group(const dv_csr_host &a) {
    const int32_t n = a.n_rows;
    for (int g : {3, 2}) {
        if (n % g != 0 || n == 0) continue;
        int ok = 1;
#pragma omp parallel for schedule(static) reduction(min : ok)
        for (int32_t gi = 0; gi < n / g; ++gi) {
            const int32_t r0 = gi * g;
            const int32_t len = a.rowptr[r0 + 1] - a.rowptr[r0];
            for (int d = 1; d < g && ok; ++d) {
                const int32_t r = r0 + d;
                if (a.rowptr[r + 1] - a.rowptr[r] != len ||
                    std::memcmp(a.col + a.rowptr[r], a.col + a.rowptr[r0], 4 * (size_t)len) != 0)
                    ok = 0;
            }
        }
        if (ok) return g;
    }
    return 1;
}

// Entry bytes of the lane layout: 255 marks a lane-block start (its column comes
// from the lane's column list), any other value is gap - 1.  Lane blocks are the
// SoA blocks, further split before every entry whose gap is exactly 256 (gap - 1 =
// 255 is legal inside an SoA block), so the marker is never ambiguous.  With at
// most 256 / value_bytes distinct values, 8-bit value indices are stored
// pre-multiplied by the value size, as byte offsets into the table.
namespace {
// Walks the leader row r0 of a group: calls f(entry, column, starts_lane_block).
template <class F>
void walk_lane_blocks(const DuviHost &h, int32_t r0, F f) {
    const uint32_t d0 = h.row_to_dist[r0], ne = h.row_to_dist[r0 + 1] - d0;
    uint32_t bl = h.row_to_col[r0], next_start = 0, c = 0;
    for (uint32_t e = 0; e < ne; ++e) {
        const uint32_t byte = h.dist[d0 + e];
        bool start = false;
        if (e == next_start) {   // SoA block start: byte = entries that follow in the block
            next_start = e + byte + 1;
            c = h.col_idx[bl++];
            start = true;
        } else {
            c += byte + 1;
            start = byte == 255u;
        }
        f(e, c, start, byte);
    }
}
}  // namespace

void dv_build_duvi_lanes(const DuviHost &h, int32_t n, int32_t n_cols, int value_bytes, DuviLanesHost &L) {
    int shift = 0;
    const int g = detect_group(h, n, shift);
    const int vib = h.vi_bits / 8;            // bytes per value index
    const size_t chunk = 4 * (size_t)vib;     // bytes per chunk of 4 indices
    L.group = g;
    L.shift = shift;
    L.scaled = (vib == 1 && (int64_t)h.values.size() * value_bytes <= 256) ? 1 : 0;
    L.ngroups = n / g;
    // Node tuples: with 8-bit indices and groups of 2-3 rows, the g value indices of a
    // node-entry often take few distinct combinations (165 for the hex operators at any
    // size); up to 256 of them, each node-entry stores one tuple index instead of g
    // value indices.  Tuples are numbered in first-occurrence order.
    L.tuples = 0;
    L.tuple_vi.clear();
    if (g >= 2 && vib == 1) {
        // each chunk of groups lists its tuples in first-occurrence order; merged in
        // chunk order they give the numbering of one walk over all groups
#ifdef _OPENMP
        const int T = omp_get_max_threads();
#else
        const int T = 1;
#endif
        const size_t nkeys = (size_t)1 << (8 * g);
        std::vector<std::vector<uint32_t>> first(T);
#pragma omp parallel for schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            std::vector<uint8_t> seen(nkeys / 8 + 1, 0);
            const int64_t gb = L.ngroups * t / T, ge = L.ngroups * (t + 1) / T;
            for (int64_t gi = gb; gi < ge && first[t].size() <= 256; ++gi) {
                const int32_t r0 = (int32_t)(gi * g);
                const uint32_t ne = h.row_to_dist[r0 + 1] - h.row_to_dist[r0];
                for (uint32_t e = 0; e < ne && first[t].size() <= 256; ++e) {
                    uint32_t key = 0;
                    for (int d = 0; d < g; ++d) key |= h.vidx[h.row_to_dist[r0 + d] + e] << (8 * d);
                    if (!(seen[key >> 3] & (1u << (key & 7)))) {
                        seen[key >> 3] |= (uint8_t)(1u << (key & 7));
                        first[t].push_back(key);
                    }
                }
            }
        }
        std::vector<int16_t> id(nkeys, -1);
        int ntup = 0;
        bool ok = true;
        for (int t = 0; t < T; ++t) ok = ok && first[t].size() <= 256;   // more in one chunk: more in all
        for (int t = 0; t < T && ok; ++t)
            for (uint32_t key : first[t]) {
                if (id[key] >= 0) continue;
                if (ntup == 256) { ok = false; break; }
                id[key] = (int16_t)ntup++;
                for (int d = 0; d < g; ++d) L.tuple_vi.push_back((key >> (8 * d)) & 0xFFu);
            }
        if (ok) {
            L.tuples = 1;
            L.tuple_id.swap(id);
        } else {
            L.tuple_vi.clear();
        }
    }
    const int nv = L.tuples ? 1 : g;   // index chunks per word
    // Stencil mode (square operators with node tuples, identical columns in a group):
    // on a structured mesh the column offset of a node-entry from the group's first
    // row takes few values (81 for the hex operators: 27 neighbours x 3 dofs); up to
    // 256 of them, the entry byte is an index into an offset table and the column
    // list, block starts and gaps are not stored at all.
    L.stencil = 0;
    L.offsets.clear();
    if (L.tuples && !shift && n_cols == n) {
        bool ok = true;
#pragma omp parallel
        {
            OffsetSet local;
#pragma omp for schedule(static)
            for (int64_t gi = 0; gi < L.ngroups; ++gi) {
                if (!ok) continue;
                const int32_t r0 = (int32_t)(gi * g);
                walk_lane_blocks(h, r0, [&](uint32_t, uint32_t c, bool, uint32_t) {
                    if (!local.insert((int64_t)c - r0)) ok = false;
                });
            }
#pragma omp critical
            {
                for (int64_t k : local.keys)
                    if (ok && !L.offset_set.insert(k)) ok = false;
            }
        }
        if (ok) {   // ids in ascending offset order (independent of the thread schedule)
            std::vector<int64_t> ks = L.offset_set.keys;
            std::sort(ks.begin(), ks.end());
            L.offset_set = OffsetSet();
            for (int64_t k : ks) {
                L.offset_set.insert(k);
                L.offsets.push_back((int32_t)k);
            }
            L.stencil = 1;
        }
    }
    L.nbundles = (L.ngroups + 31) / 32;
    L.meta.assign(5 * L.nbundles, 0);
    L.nent.assign(L.ngroups, 0);
    // sizes per bundle
    std::vector<uint64_t> dwords(L.nbundles + 1, 0), vchunks(L.nbundles + 1, 0), cwords(L.nbundles + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t bi = 0; bi < L.nbundles; ++bi) {
        uint32_t le = 0, lb = 0;
        for (int t = 0; t < 32; ++t) {
            int64_t gi = bi * 32 + t;
            if (gi >= L.ngroups) break;
            int32_t r0 = (int32_t)(gi * g);
            uint32_t ne = h.row_to_dist[r0 + 1] - h.row_to_dist[r0], nb = 0;
            walk_lane_blocks(h, r0, [&](uint32_t, uint32_t, bool start, uint32_t) { nb += start; });
            L.nent[gi] = ne;
            le = std::max(le, ne);
            lb = std::max(lb, nb);
        }
        const uint32_t words = (le + 3) / 4;
        dwords[bi + 1] = (uint64_t)words * 32;
        vchunks[bi + 1] = (uint64_t)words * nv * 32;
        cwords[bi + 1] = L.stencil ? 0 : (uint64_t)lb * 32;
        L.meta[5 * bi + 3] = words;
        L.meta[5 * bi + 4] = lb;
    }
    for (int64_t bi = 0; bi < L.nbundles; ++bi) {
        dwords[bi + 1] += dwords[bi];
        vchunks[bi + 1] += vchunks[bi];
        cwords[bi + 1] += cwords[bi];
    }
    DV_REQUIRE(dwords[L.nbundles] < 0xFFFFFFFFull && vchunks[L.nbundles] < 0xFFFFFFFFull && cwords[L.nbundles] < 0xFFFFFFFFull,
               DV_ERR_FORMAT, "lane layout exceeds 32-bit offsets");
    L.dist.assign(dwords[L.nbundles], 0);
    L.vi.assign(vchunks[L.nbundles] * chunk, 0);
    L.cols.assign(cwords[L.nbundles], 0);
#pragma omp parallel for schedule(static)
    for (int64_t bi = 0; bi < L.nbundles; ++bi) {
        L.meta[5 * bi + 0] = (uint32_t)dwords[bi];
        L.meta[5 * bi + 1] = (uint32_t)vchunks[bi];
        L.meta[5 * bi + 2] = (uint32_t)cwords[bi];
        const uint32_t words = L.meta[5 * bi + 3];
        for (int t = 0; t < 32; ++t) {
            int64_t gi = bi * 32 + t;
            if (gi >= L.ngroups) break;
            const int32_t r0 = (int32_t)(gi * g);
            const uint32_t d0 = h.row_to_dist[r0], ne = h.row_to_dist[r0 + 1] - d0;
            uint32_t nlb = 0;
            walk_lane_blocks(h, r0, [&](uint32_t e, uint32_t c, bool start, uint32_t byte) {
                const uint32_t w = e / 4, k = e % 4;
                if (L.stencil) {
                    byte = (uint32_t)L.offset_set.find((int64_t)c - r0);
                } else if (start) {
                    byte = 255u;
                    L.cols[cwords[bi] + (uint64_t)nlb * 32 + t] = c;
                    ++nlb;
                }
                L.dist[dwords[bi] + (uint64_t)w * 32 + t] |= byte << (8 * k);
            });
            (void)d0;
            if (L.tuples) {
                for (uint32_t e = 0; e < ne; ++e) {
                    uint32_t key = 0;
                    for (int d = 0; d < g; ++d) key |= h.vidx[h.row_to_dist[r0 + d] + e] << (8 * d);
                    const uint32_t w = e / 4, k = e % 4;
                    const uint64_t c = vchunks[bi] + (uint64_t)w * 32 + t;
                    L.vi[c * chunk + k] = (uint8_t)L.tuple_id[key];
                }
            } else {
                for (int d = 0; d < g; ++d) {
                    const uint32_t rd = h.row_to_dist[r0 + d];
                    for (uint32_t e = 0; e < ne; ++e) {
                        uint32_t w = e / 4, k = e % 4;
                        uint64_t c = vchunks[bi] + ((uint64_t)w * g + d) * 32 + t;
                        uint32_t v = h.vidx[rd + e];
                        if (L.scaled) v *= (uint32_t)value_bytes;
                        std::memcpy(&L.vi[c * chunk + k * vib], &v, vib);   // little-endian low bytes
                    }
                }
            }
            (void)words;
        }
    }
    std::vector<int16_t>().swap(L.tuple_id);
    L.offset_set = OffsetSet();
}

void dv_build_duvi_patterns(const DuviHost &h, int32_t n, int32_t n_cols, int g, int shift, int max_patterns,
                            int max_entries, DuviPatternHost &P) {
    P = DuviPatternHost();
    if (g < 1 || n % g != 0 || n == 0) return;
    const bool based = shift || n_cols != n;
    // group signature: entry count, then per entry the column offset and the g value indices
    const int64_t ngroups = n / g;
    std::vector<uint64_t> sig(ngroups);
    if (based) P.base.assign(ngroups, 0);
    auto entries = [&](int64_t gi, std::vector<int64_t> &out) {
        out.clear();
        const int32_t r0 = (int32_t)(gi * g);
        const int64_t b0 = based ? (int64_t)(h.row_to_col[r0 + 1] > h.row_to_col[r0] ? h.col_idx[h.row_to_col[r0]] : 0) : r0;
        walk_lane_blocks(h, r0, [&](uint32_t e, uint32_t c, bool, uint32_t) {
            out.push_back((int64_t)c - b0);
            for (int d = 0; d < g; ++d) out.push_back(h.vidx[h.row_to_dist[r0 + d] + e]);
        });
    };
    if (based)
        for (int64_t gi = 0; gi < ngroups; ++gi) {
            const int32_t r0 = (int32_t)(gi * g);
            if (h.row_to_col[r0 + 1] > h.row_to_col[r0]) P.base[gi] = h.col_idx[h.row_to_col[r0]];
        }
#pragma omp parallel
    {
        std::vector<int64_t> buf;
#pragma omp for schedule(static)
        for (int64_t gi = 0; gi < ngroups; ++gi) {
            entries(gi, buf);
            uint64_t x = 1469598103934665603ull ^ buf.size();
            for (int64_t v : buf) x = (x ^ (uint64_t)v) * 1099511628211ull;
            sig[gi] = x;
        }
    }
    // First-occurrence numbering by signature, then every group's entries confirmed
    // against its pattern's (in parallel).  Two different entry lists with one 64-bit
    // signature would fail the confirmation; the sequential numbering that compares
    // entry lists on every signature match then runs instead.
    std::vector<uint64_t> phash;
    std::vector<std::vector<int64_t>> pent;
    std::vector<int64_t> buf;
    P.id.resize(ngroups);
    bool by_signature = true;
    for (int64_t gi = 0; gi < ngroups && by_signature; ++gi) {
        int found = -1;
        for (size_t p = 0; p < phash.size(); ++p)
            if (phash[p] == sig[gi]) { found = (int)p; break; }
        if (found < 0) {
            if ((int)phash.size() == max_patterns) return;
            entries(gi, buf);
            phash.push_back(sig[gi]);
            pent.push_back(buf);
            found = (int)phash.size() - 1;
        }
        P.id[gi] = (uint16_t)found;
    }
    {
        std::atomic<bool> mismatch(false);
#pragma omp parallel
        {
            std::vector<int64_t> mine;
#pragma omp for schedule(static)
            for (int64_t gi = 0; gi < ngroups; ++gi) {
                if (mismatch.load(std::memory_order_relaxed)) continue;
                entries(gi, mine);
                if (mine != pent[P.id[gi]]) mismatch.store(true, std::memory_order_relaxed);
            }
        }
        by_signature = !mismatch.load();
    }
    if (!by_signature) {
        phash.clear();
        pent.clear();
        for (int64_t gi = 0; gi < ngroups; ++gi) {
            int found = -1;
            for (size_t p = 0; p < phash.size(); ++p)
                if (phash[p] == sig[gi]) {
                    entries(gi, buf);
                    if (buf == pent[p]) { found = (int)p; break; }
                }
            if (found < 0) {
                if ((int)phash.size() == max_patterns) return;
                entries(gi, buf);
                phash.push_back(sig[gi]);
                pent.push_back(buf);
                found = (int)phash.size() - 1;
            }
            P.id[gi] = (uint16_t)found;
        }
    }
    int64_t total = 0;
    for (auto &e : pent) total += (int64_t)e.size() / (1 + g);
    if (total > max_entries) return;
    P.start.assign(1, 0);
    for (auto &e : pent) {
        const size_t m = e.size() / (1 + g);
        for (size_t k = 0; k < m; ++k) {
            P.off.push_back((int32_t)e[k * (1 + g)]);
            for (int d = 0; d < g; ++d) P.vi.push_back((uint32_t)e[k * (1 + g) + 1 + d]);
        }
        P.start.push_back((uint32_t)P.off.size());
    }
    P.group = g;
    P.shift = shift;
    P.based = based ? 1 : 0;
    P.ngroups = ngroups;
    P.ok = 1;
}

bool dv_grid_geometry(const DuviPatternHost &P, int hot, int64_t ng, int32_t &lxo, int32_t &lyo, int32_t &lzo) {
    if (P.group != 3 || P.based || P.shift || ng < 27 || hot < 0 || hot + 1 >= (int)P.start.size()) return false;
    const uint32_t s0 = P.start[hot];
    if (P.start[hot + 1] - s0 != 81) return false;
    // the 27 neighbour groups, each with its 3 consecutive columns, in column order
    int64_t no[27];
    for (int j = 0; j < 27; ++j) {
        const int64_t o = P.off[s0 + 3 * j];
        for (int c = 1; c < 3; ++c)
            if (P.off[s0 + 3 * j + c] != o + c) return false;
        if (((o % 3) + 3) % 3 != 0) return false;
        no[j] = o / 3;
    }
    const int64_t lx = no[16], lxy = no[22];   // offsets of the +y and +z neighbours
    if (lx < 3 || lxy < 3 * lx || lxy % lx != 0) return false;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (no[9 * (dz + 1) + 3 * (dy + 1) + dx + 1] != dx + lx * dy + lxy * dz) return false;
    const int64_t ly = lxy / lx;
    if (ly < 3 || ng % lxy != 0 || ng / lxy < 3 || lx > INT32_MAX || ly > INT32_MAX) return false;
    lxo = (int32_t)lx;
    lyo = (int32_t)ly;
    lzo = (int32_t)(ng / lxy);
    return true;
}

void dv_build_duvi_grid(const DuviPatternHost &P, DuviGridHost &G) {
    G = DuviGridHost();
    if (!P.ok || P.group != 3 || P.based || P.shift || P.ngroups < 27) return;
    const int npat = (int)P.start.size() - 1;
    std::vector<int64_t> cnt(npat, 0);
    for (uint16_t id : P.id) cnt[id]++;
    const int hot = (int)(std::max_element(cnt.begin(), cnt.end()) - cnt.begin());
    int32_t lx, ly, lz;
    if (!dv_grid_geometry(P, hot, P.ngroups, lx, ly, lz)) return;
    const int64_t ng = P.ngroups, lxy = (int64_t)lx * ly;
    bool all_hot = true;
    for (int64_t gi = 0; gi < ng; ++gi) {
        const int64_t ix = gi % lx, iy = (gi / lx) % ly, iz = gi / lxy;
        const bool inner = ix >= 1 && ix <= lx - 2 && iy >= 1 && iy <= ly - 2 && iz >= 1 && iz <= lz - 2;
        if (inner && P.id[gi] == hot) continue;
        if (inner) all_hot = false;
        G.boundary.push_back((uint32_t)gi);
    }
    const uint32_t s0 = P.start[hot];
    G.vi.assign(P.vi.begin() + 3 * (size_t)s0, P.vi.begin() + 3 * (size_t)(s0 + 81));
    G.lx = lx;
    G.ly = ly;
    G.lz = lz;
    G.hot = hot;
    G.all_hot = all_hot ? 1 : 0;
    G.ok = 1;
}

void dv_extract_diag(const dv_csr_host &a, std::vector<double> &d) {
    d.assign(a.n_rows, 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < a.n_rows; ++i)
        for (int32_t k = a.rowptr[i]; k < a.rowptr[i + 1]; ++k)
            if (a.col[k] == i) d[i] = a.val[k];
}

double dv_row_ratio_bound(const dv_csr_host &a) {
    double l = 0;
    for (int32_t i = 0; i < a.n_rows; ++i) {
        double s = 0.0, mx = 0.0;
        for (int32_t k = a.rowptr[i]; k < a.rowptr[i + 1]; ++k) {
            double v = std::fabs(a.val[k]);
            s += v;
            mx = std::max(mx, v);
        }
        if (mx > 0) l = std::max(l, s / mx);
    }
    return l;
}

// In-place inverse of a dense SPD matrix through A = L D L^T: factor, then
// solve for the unit vectors (columns in parallel).
bool dv_dense_inverse(int32_t n, std::vector<double> &a, double pivot_tol) {
    std::vector<double> f = a;   // factor in place: strict lower L, diagonal D
    std::vector<double> v(n);
    for (int32_t j = 0; j < n; ++j) {
        double d = f[(size_t)j * n + j];
        for (int32_t k = 0; k < j; ++k) {
            v[k] = f[(size_t)j * n + k] * f[(size_t)k * n + k];
            d -= f[(size_t)j * n + k] * v[k];
        }
        if (!(std::fabs(d) >= pivot_tol)) return false;
        f[(size_t)j * n + j] = d;
#pragma omp parallel for schedule(static)
        for (int32_t i = j + 1; i < n; ++i) {
            double s = f[(size_t)i * n + j];
            const double *fi = &f[(size_t)i * n];
            for (int32_t k = 0; k < j; ++k) s -= fi[k] * v[k];
            f[(size_t)i * n + j] = s / d;
        }
    }
    // the strict upper triangle is free after the factorisation: L^T there lets the
    // backward substitution read rows instead of columns (same operations, same order)
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = i + 1; k < n; ++k) f[(size_t)i * n + k] = f[(size_t)k * n + i];
#pragma omp parallel for schedule(dynamic, 8)
    for (int32_t c = 0; c < n; ++c) {
        std::vector<double> x(n, 0.0);
        x[c] = 1.0;
        for (int32_t i = c + 1; i < n; ++i) {
            double s = 0.0;
            const double *fi = &f[(size_t)i * n];
            for (int32_t k = c; k < i; ++k) s += fi[k] * x[k];
            x[i] = -s;
        }
        for (int32_t i = 0; i < n; ++i) x[i] /= f[(size_t)i * n + i];
        for (int32_t i = n - 1; i >= 0; --i) {
            double s = x[i];
            const double *lti = &f[(size_t)i * n];
            for (int32_t k = i + 1; k < n; ++k) s -= lti[k] * x[k];
            x[i] = s;
        }
        for (int32_t i = 0; i < n; ++i) a[(size_t)i * n + c] = x[i];
    }
    return true;
}

int dv_block_coloring(const dv_csr_host &a, int bs, std::vector<int32_t> &color) {
    int32_t nb = (a.n_rows + bs - 1) / bs;
    color.assign(nb, -1);
    std::vector<int32_t> mark;
    int ncolors = 0;
    for (int32_t b = 0; b < nb; ++b) {
        mark.assign(ncolors + 1, 0);
        for (int32_t r = b * bs; r < std::min<int32_t>((b + 1) * bs, a.n_rows); ++r)
            for (int32_t k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) {
                int32_t nbk = a.col[k] / bs;
                if (nbk != b && color[nbk] >= 0) mark[color[nbk]] = 1;
            }
        int c = 0;
        while (c < ncolors && mark[c]) ++c;
        color[b] = c;
        if (c == ncolors) ++ncolors;
    }
    return ncolors;
}

int dv_gs_level_sets(const dv_csr_host &a, std::vector<int32_t> &perm, std::vector<int32_t> &offsets) {
    int32_t n = a.n_rows;
    std::vector<int32_t> lev(n, 0);
    int32_t maxl = 0;
    for (int32_t i = 0; i < n; ++i) {
        int32_t l = 0;
        for (int32_t k = a.rowptr[i]; k < a.rowptr[i + 1]; ++k) {
            int32_t j = a.col[k];
            if (j < i) l = std::max(l, lev[j] + 1);
        }
        lev[i] = l;
        maxl = std::max(maxl, l);
    }
    offsets.assign(maxl + 2, 0);
    for (int32_t i = 0; i < n; ++i) offsets[lev[i] + 1]++;
    for (int32_t l = 0; l <= maxl; ++l) offsets[l + 1] += offsets[l];
    perm.resize(n);
    std::vector<int32_t> fill(offsets.begin(), offsets.end() - 1);
    for (int32_t i = 0; i < n; ++i) perm[fill[lev[i]]++] = i;
    return maxl + 1;
}

// ---------------------------------------------------------------------------
// structured hex workload generator
// ---------------------------------------------------------------------------
// Element stiffness of FemCantilever3D.cs:225-313 (top3d), row-major 24x24.
static void hex_ke(double E, double v, double *ke) {
    static const double A[2][14] = {{32, 6, -8, 6, -6, 4, 3, -6, -10, 3, -3, -3, -4, -8},
                                    {-48, 0, 0, -24, 24, 0, 0, 0, 12, -12, 0, 12, 12, 12}};
    double k[15];
    k[0] = 0;
    for (int i = 0; i < 14; ++i) {
        double t = 0.0;
        t += A[0][i] * 1.0;
        t += A[1][i] * v;
        k[i + 1] = t * (1.0 / 72.0);
    }
    static const int K[6][6][6] = {
        {{1, 2, 2, 3, 5, 5}, {2, 1, 2, 4, 6, 7}, {2, 2, 1, 4, 7, 6}, {3, 4, 4, 1, 8, 8}, {5, 6, 7, 8, 1, 2}, {5, 7, 6, 8, 2, 1}},
        {{9, 8, 12, 6, 4, 7}, {8, 9, 12, 5, 3, 5}, {10, 10, 13, 7, 4, 6}, {6, 5, 11, 9, 2, 10}, {4, 3, 5, 2, 9, 12}, {11, 4, 6, 12, 10, 13}},
        {{6, 7, 4, 9, 12, 8}, {7, 6, 4, 10, 13, 10}, {5, 5, 3, 8, 12, 9}, {9, 10, 2, 6, 11, 5}, {12, 13, 10, 11, 6, 4}, {2, 12, 9, 4, 5, 3}},
        {{14, 11, 11, 13, 10, 10}, {11, 14, 11, 12, 9, 8}, {11, 11, 14, 12, 8, 9}, {13, 12, 12, 14, 7, 7}, {10, 9, 8, 7, 14, 11}, {10, 8, 9, 7, 11, 14}},
        {{1, 2, 8, 3, 5, 4}, {2, 1, 8, 4, 6, 11}, {8, 8, 1, 5, 11, 6}, {3, 4, 5, 1, 8, 2}, {5, 6, 11, 8, 1, 8}, {4, 11, 6, 2, 8, 1}},
        {{14, 11, 7, 13, 10, 12}, {11, 14, 7, 12, 9, 2}, {7, 7, 14, 10, 2, 9}, {13, 12, 10, 14, 7, 11}, {10, 9, 2, 7, 14, 7}, {12, 2, 9, 11, 7, 14}}};
    // block (bi,bj) -> (matrix id, transposed): {K1,K2,K3,K4; K2',K5,K6,K3'; K3',K6,K5',K2'; K4,K3,K2,K1'}
    static const int id[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 2}, {2, 5, 4, 1}, {3, 2, 1, 0}};
    static const bool tr[4][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {1, 0, 1, 1}, {0, 0, 0, 1}};
    double f = E / ((v + 1) * (1 - 2 * v));
    for (int bi = 0; bi < 4; ++bi)
        for (int bj = 0; bj < 4; ++bj)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    int m = tr[bi][bj] ? K[id[bi][bj]][j][i] : K[id[bi][bj]][i][j];
                    ke[(bi * 6 + i) * 24 + bj * 6 + j] = k[m] * f;
                }
}

void dv_hex_ke(double E, double nu, double *ke) { hex_ke(E, nu, ke); }

static inline int32_t hex_row_nodes(int32_t i, int32_t j, int32_t k, int32_t nx, int32_t ny, int32_t nz) {
    int ci = (i > 1 ? 1 : 0) + 1 + (i + 1 < nx ? 1 : 0);   // x neighbours among free nodes (x index >= 1)
    int cj = (j > 0 ? 1 : 0) + 1 + (j + 1 < ny ? 1 : 0);
    int ck = (k > 0 ? 1 : 0) + 1 + (k + 1 < nz ? 1 : 0);
    return ci * cj * ck;
}

extern "C" DV_API int dv_duvi_encode(const dv_csr_host *a, int32_t value_index_bits, double dedup_tol,
                                     int64_t *nblocks, int64_t *nuniq, int32_t *bits, uint32_t *row_to_col,
                                     uint32_t *row_to_dist, uint32_t *col_idx, uint8_t *dist,
                                     uint32_t *value_indices, double *values) {
    return dv_guard([&] {
        DV_REQUIRE(a && nblocks && nuniq && bits, DV_ERR_ARG, "null argument");
        dv_check_csr(*a);
        DuviHost h;
        dv_encode_duvi(*a, dedup_tol, value_index_bits, h);
        *nblocks = (int64_t)h.col_idx.size();
        *nuniq = (int64_t)h.values.size();
        *bits = h.vi_bits;
        if (!row_to_col) return;   // sizes only
        DV_REQUIRE(row_to_dist && col_idx && values && ((dist && value_indices) || h.vidx.empty()), DV_ERR_ARG,
                   "null output array");
        std::copy(h.row_to_col.begin(), h.row_to_col.end(), row_to_col);
        std::copy(h.row_to_dist.begin(), h.row_to_dist.end(), row_to_dist);
        std::copy(h.col_idx.begin(), h.col_idx.end(), col_idx);
        std::copy(h.dist.begin(), h.dist.end(), dist);
        std::copy(h.vidx.begin(), h.vidx.end(), value_indices);
        std::copy(h.values.begin(), h.values.end(), values);
    });
}

extern "C" DV_API int dv_hex_csr_size(const int32_t *ne, int32_t *n_rows, int64_t *nnz) {
    return dv_guard([&] {
        DV_REQUIRE(ne && ne[0] > 0 && ne[1] > 0 && ne[2] > 0, DV_ERR_ARG, "element counts must be positive");
        int64_t nx = ne[0] + 1, ny = ne[1] + 1, nz = ne[2] + 1;
        int64_t rows = 3 * (nx - 1) * ny * nz;
        DV_REQUIRE(rows < INT32_MAX, DV_ERR_ARG, "mesh too large for int32 rows");
        // nnz = 9 * (sum over x of free neighbours) * (sum over y) * (sum over z), separable
        auto s1 = [](int64_t n, bool clamp) {
            int64_t s = 0;
            for (int64_t i = clamp ? 1 : 0; i < n; ++i)
                s += (clamp ? (i > 1) : (i > 0)) + 1 + (i + 1 < n);
            return s;
        };
        int64_t z = 9 * s1(nx, true) * s1(ny, false) * s1(nz, false);
        DV_REQUIRE(z < INT32_MAX, DV_ERR_ARG, "nnz exceeds int32 offsets");
        *n_rows = (int32_t)rows;
        *nnz = z;
    });
}

// Row-wise assembly; each entry sums its element contributions in increasing
// element id, starting from 0.0 + first term, exactly as DokRowMajor.AddSubmatrix
// accumulates (DokRowMajor.cs:182-207) when FemCantileverBase.AssembleGlobalMatrix
// visits the elements in order (FemCantileverBase.cs:95-101).
extern "C" DV_API int dv_hex_assemble(const int32_t *ne, const double *elem_E, double scale, double E, double nu,
                                      int32_t *rowptr, int32_t *col, double *val) {
    return dv_guard([&] {
        int32_t nrows;
        int64_t nnz;
        int st = dv_hex_csr_size(ne, &nrows, &nnz);
        DV_REQUIRE(st == DV_OK, st, "bad mesh");
        DV_REQUIRE(rowptr && col && val, DV_ERR_ARG, "null output array");
        double ke[576];
        hex_ke(E, nu, ke);
        const int32_t nx = ne[0] + 1, ny = ne[1] + 1, nz = ne[2] + 1;
        auto fidx = [&](int32_t i, int32_t j, int32_t k) { return 3 * ((i - 1) + (nx - 1) * (j + ny * k)); };
        // row offsets (plane by plane prefix)
        rowptr[0] = 0;
        {
            int64_t p = 0;
            for (int32_t k = 0; k < nz; ++k)
                for (int32_t j = 0; j < ny; ++j)
                    for (int32_t i = 1; i < nx; ++i) {
                        int32_t c = 3 * hex_row_nodes(i, j, k, nx, ny, nz);
                        int32_t r = fidx(i, j, k);
                        for (int d = 0; d < 3; ++d) { p += c; rowptr[r + d + 1] = (int32_t)p; }
                    }
        }
        static const int vtk[8] = {0, 1, 3, 2, 4, 5, 7, 6};
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
        for (int32_t k = 0; k < nz; ++k)
            for (int32_t j = 0; j < ny; ++j)
                for (int32_t i = 1; i < nx; ++i) {
                    int32_t r0 = fidx(i, j, k);
                    for (int d = 0; d < 3; ++d) {
                        int64_t p = rowptr[r0 + d];
                        for (int dk = -1; dk <= 1; ++dk)
                            for (int dj = -1; dj <= 1; ++dj)
                                for (int di = -1; di <= 1; ++di) {
                                    int32_t ii = i + di, jj = j + dj, kk = k + dk;
                                    if (ii < 1 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
                                    int32_t c0 = std::max(std::max(k, kk) - 1, 0), c1 = std::min(std::min(k, kk), ne[2] - 1);
                                    int32_t b0 = std::max(std::max(j, jj) - 1, 0), b1 = std::min(std::min(j, jj), ne[1] - 1);
                                    int32_t a0 = std::max(std::max(i, ii) - 1, 0), a1 = std::min(std::min(i, ii), ne[0] - 1);
                                    int32_t cbase = fidx(ii, jj, kk);
                                    for (int d2 = 0; d2 < 3; ++d2) {
                                        double s = 0.0;
                                        bool first = true;
                                        for (int32_t c = c0; c <= c1; ++c)
                                            for (int32_t b = b0; b <= b1; ++b)
                                                for (int32_t a = a0; a <= a1; ++a) {
                                                    int64_t e = a + (int64_t)ne[0] * (b + (int64_t)ne[1] * c);
                                                    int la = vtk[(i - a) + 2 * (j - b) + 4 * (k - c)];
                                                    int lb = vtk[(ii - a) + 2 * (jj - b) + 4 * (kk - c)];
                                                    double ce = elem_E ? scale * elem_E[e] : scale;
                                                    double t = ce * ke[(3 * la + d) * 24 + 3 * lb + d2];
                                                    if (first) { s = t + 0.0; first = false; }
                                                    else s = t + s;
                                                }
                                        col[p] = cbase + d2;
                                        val[p] = s;
                                        ++p;
                                    }
                                }
                    }
                }
    });
}

// Vertex-based factor-2 coarsening of one axis with n elements: coarse nodes
// sit at the even fine nodes and at the last fine node (for odd n the last
// coarse element has length 1).  Fine node i takes 1 or 2 coarse nodes with
// the linear-interpolation weights; for even n this is standard trilinear.
static int coarse_1d(int32_t i, int32_t n, int32_t idx[2], double w[2]) {
    if ((i & 1) && i != n) {
        idx[0] = i / 2;
        idx[1] = i / 2 + 1;
        w[0] = w[1] = 0.5;
        return 2;
    }
    idx[0] = i == n ? (n + 1) / 2 : i / 2;
    w[0] = 1.0;
    return 1;
}

extern "C" DV_API int dv_hex_trilinear_size(const int32_t *nef, int32_t *n_rows, int32_t *n_cols, int64_t *nnz) {
    return dv_guard([&] {
        DV_REQUIRE(nef && nef[0] >= 1 && nef[1] >= 1 && nef[2] >= 1, DV_ERR_ARG, "element counts must be >= 1");
        int64_t nx = nef[0] + 1, ny = nef[1] + 1, nz = nef[2] + 1;
        int64_t cx = (nef[0] + 1) / 2 + 1, cy = (nef[1] + 1) / 2 + 1, cz = (nef[2] + 1) / 2 + 1;
        int64_t sx = 0, sy = 0, sz = 0;
        int32_t idx[2];
        double w[2];
        for (int32_t i = 1; i < nx; ++i) {   // coarse x = 0 is clamped
            const int m = coarse_1d(i, nef[0], idx, w);
            for (int a = 0; a < m; ++a) sx += idx[a] != 0;
        }
        for (int32_t j = 0; j < ny; ++j) sy += coarse_1d(j, nef[1], idx, w);
        for (int32_t k = 0; k < nz; ++k) sz += coarse_1d(k, nef[2], idx, w);
        *n_rows = (int32_t)(3 * (nx - 1) * ny * nz);
        *n_cols = (int32_t)(3 * (cx - 1) * cy * cz);
        *nnz = 3 * sx * sy * sz;
    });
}

extern "C" DV_API int dv_hex_trilinear(const int32_t *nef, int32_t *rowptr, int32_t *col, double *val) {
    return dv_guard([&] {
        int32_t nr, nc;
        int64_t nnz;
        int st = dv_hex_trilinear_size(nef, &nr, &nc, &nnz);
        DV_REQUIRE(st == DV_OK, st, "bad mesh");
        int32_t nx = nef[0] + 1, ny = nef[1] + 1, nz = nef[2] + 1;
        int32_t cx = (nef[0] + 1) / 2 + 1, cy = (nef[1] + 1) / 2 + 1;
        int64_t p = 0;
        int32_t r = 0;
        rowptr[0] = 0;
        for (int32_t k = 0; k < nz; ++k)
            for (int32_t j = 0; j < ny; ++j)
                for (int32_t i = 1; i < nx; ++i)
                    for (int d = 0; d < 3; ++d) {
                        int32_t ci[2], cj[2], ck[2];
                        double wi[2], wj[2], wk[2];
                        const int ni = coarse_1d(i, nef[0], ci, wi), nj = coarse_1d(j, nef[1], cj, wj),
                                  nk = coarse_1d(k, nef[2], ck, wk);
                        for (int c = 0; c < nk; ++c)
                            for (int b = 0; b < nj; ++b)
                                for (int a = 0; a < ni; ++a) {
                                    if (ci[a] == 0) continue;
                                    col[p] = 3 * ((ci[a] - 1) + (cx - 1) * (cj[b] + cy * ck[c])) + d;
                                    val[p] = wi[a] * wj[b] * wk[c];
                                    ++p;
                                }
                        rowptr[++r] = (int32_t)p;
                    }
        DV_REQUIRE(p == nnz && r == nr, DV_ERR_ARG, "internal size mismatch");
    });
}

// ---------------------------------------------------------------------------
// Galerkin coarse operator P^T A P (sorted rows).  Row I of the result sums,
// in order, over the entries (r, I) of P, the entries (r, j) of A and the
// entries (j, J) of P, each term ((P_rI A_rj) P_jJ).
// ---------------------------------------------------------------------------
void dv_csr_transpose(const dv_csr_host &a, std::vector<int32_t> &rp, std::vector<int32_t> &ci, std::vector<double> &va) {
    const int64_t nnz = a.rowptr[a.n_rows];
    rp.assign((size_t)a.n_cols + 1, 0);
    ci.resize(nnz);
    va.resize(nnz);
#ifdef _OPENMP
    const int64_t nc = std::max<int32_t>(a.n_cols, 1);
    const int T = (int)std::min<int64_t>(omp_get_max_threads(), std::max<int64_t>(1, ((int64_t)1 << 26) / nc));
    if (T > 1 && nnz >= ((int64_t)1 << 20)) {
        // Thread t counts, then places, the entries of rows [n t / T, n (t + 1) / T): inside a
        // column its entries follow those of threads before it, so every transposed row
        // lists its entries by increasing original row, as the sequential pass does.
        std::vector<int32_t> cnt((size_t)T * nc, 0);
        auto rows = [&](int t) {
            return std::make_pair((int32_t)((int64_t)a.n_rows * t / T), (int32_t)((int64_t)a.n_rows * (t + 1) / T));
        };
#pragma omp parallel for schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            int32_t *ct = cnt.data() + (size_t)t * nc;
            const auto [r0, r1] = rows(t);
            for (int64_t k = a.rowptr[r0]; k < a.rowptr[r1]; ++k) ct[a.col[k]]++;
        }
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < a.n_cols; ++c) {
            int32_t run = 0;
            for (int t = 0; t < T; ++t) {
                const int32_t v = cnt[(size_t)t * nc + c];
                cnt[(size_t)t * nc + c] = run;
                run += v;
            }
            rp[c + 1] = run;
        }
        for (int32_t c = 0; c < a.n_cols; ++c) rp[c + 1] += rp[c];
#pragma omp parallel for schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            int32_t *ct = cnt.data() + (size_t)t * nc;
            const auto [r0, r1] = rows(t);
            for (int32_t r = r0; r < r1; ++r)
                for (int32_t k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) {
                    const int32_t c = a.col[k];
                    const int64_t pos = rp[c] + ct[c]++;
                    ci[pos] = r;
                    va[pos] = a.val[k];
                }
        }
        return;
    }
#endif
    for (int64_t k = 0; k < nnz; ++k) rp[a.col[k] + 1]++;
    for (int32_t i = 0; i < a.n_cols; ++i) rp[i + 1] += rp[i];
    std::vector<int32_t> fill(rp.begin(), rp.end() - 1);
    for (int32_t r = 0; r < a.n_rows; ++r)
        for (int32_t k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) {
            const int32_t c = a.col[k];
            ci[fill[c]] = r;
            va[fill[c]] = a.val[k];
            fill[c]++;
        }
}

static void galerkin_rows(const dv_csr_host &A, const dv_csr_host &P, const std::vector<int32_t> &tp,
                          const std::vector<int32_t> &tc, const std::vector<double> &tv, int32_t *count,
                          const int32_t *rowptr, int32_t *col, double *val) {
    const int32_t nc = P.n_cols;
#pragma omp parallel
    {
        std::vector<double> acc(nc, 0.0);
        std::vector<char> mark(nc, 0);
        std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 64)
        for (int32_t I = 0; I < nc; ++I) {
            cols.clear();
            for (int32_t k = tp[I]; k < tp[I + 1]; ++k) {
                const int32_t r = tc[k];
                const double pr = tv[k];
                for (int32_t q = A.rowptr[r]; q < A.rowptr[r + 1]; ++q) {
                    const int32_t j = A.col[q];
                    const double ar = pr * A.val[q];
                    for (int32_t s = P.rowptr[j]; s < P.rowptr[j + 1]; ++s) {
                        const int32_t J = P.col[s];
                        if (!mark[J]) {
                            mark[J] = 1;
                            acc[J] = 0.0;
                            cols.push_back(J);
                        }
                        acc[J] += ar * P.val[s];
                    }
                }
            }
            std::sort(cols.begin(), cols.end());
            if (count) count[I] = (int32_t)cols.size();
            int64_t p = rowptr ? rowptr[I] : 0;
            for (int32_t J : cols) {
                if (col) {
                    col[p] = J;
                    val[p] = acc[J];
                    ++p;
                }
                mark[J] = 0;
            }
        }
    }
}

static void check_galerkin_args(const dv_csr_host *A, const dv_csr_host *P) {
    DV_REQUIRE(A && P && A->rowptr && A->col && A->val && P->rowptr && P->col && P->val, DV_ERR_ARG, "null argument");
    DV_REQUIRE(A->n_rows == A->n_cols && P->n_rows == A->n_rows && P->n_cols >= 1, DV_ERR_ARG,
               "need square A and P with as many rows as A");
}

extern "C" DV_API int dv_galerkin_size(const dv_csr_host *A, const dv_csr_host *P, int32_t *n, int64_t *nnz) {
    return dv_guard([&] {
        check_galerkin_args(A, P);
        DV_REQUIRE(n && nnz, DV_ERR_ARG, "null output");
        std::vector<int32_t> tp, tc;
        std::vector<double> tv;
        dv_csr_transpose(*P, tp, tc, tv);
        std::vector<int32_t> cnt(P->n_cols);
        galerkin_rows(*A, *P, tp, tc, tv, cnt.data(), nullptr, nullptr, nullptr);
        int64_t t = 0;
        for (int32_t c : cnt) t += c;
        DV_REQUIRE(t < INT32_MAX, DV_ERR_ARG, "coarse operator too large for int32 offsets");
        *n = P->n_cols;
        *nnz = t;
    });
}

extern "C" DV_API int dv_galerkin(const dv_csr_host *A, const dv_csr_host *P, int32_t *rowptr, int32_t *col,
                                  double *val) {
    return dv_guard([&] {
        check_galerkin_args(A, P);
        DV_REQUIRE(rowptr && col && val, DV_ERR_ARG, "null output array");
        std::vector<int32_t> tp, tc;
        std::vector<double> tv;
        dv_csr_transpose(*P, tp, tc, tv);
        std::vector<int32_t> cnt(P->n_cols);
        galerkin_rows(*A, *P, tp, tc, tv, cnt.data(), nullptr, nullptr, nullptr);
        rowptr[0] = 0;
        for (int32_t i = 0; i < P->n_cols; ++i) rowptr[i + 1] = rowptr[i] + cnt[i];
        galerkin_rows(*A, *P, tp, tc, tv, nullptr, rowptr, col, val);
    });
}

// Power-method bound of D^-1 A (GeometricMultigridSolver.cs:80-103): iterate
// until the growth ratio is within 5 %, then extrapolate.
double dv_power_bound_ref(const dv_csr_host &a, const std::vector<double> &inv_diag) {
    const double percent = 0.05;
    const int32_t n = a.n_rows;
    std::vector<double> x(n, 1 / std::sqrt((double)n)), y(n);
    double l = 1;
    for (int it = 0; it < 100000; ++it) {
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int32_t k = a.rowptr[i]; k < a.rowptr[i + 1]; ++k) s += a.val[k] * x[a.col[k]];
            y[i] = s * inv_diag[i];
        }
        double l2 = 0.0;
        for (int32_t i = 0; i < n; ++i) l2 += y[i] * y[i];
        l2 = std::sqrt(l2);
        const double sc = 1 / l2;
        for (int32_t i = 0; i < n; ++i) x[i] = y[i] * sc;
        const double ratio = l2 / l;
        if (ratio > 1 - percent && ratio < 1 + percent) {
            return ratio > 1 ? l2 * std::pow(ratio, 1 / std::sqrt(percent)) : (l2 * 9 + l) / 10;
        }
        l = l2;
    }
    return l;
}

// ---------------------------------------------------------------------------
// Restriction / interpolation of structured Cartesian meshes
// (IGeometricMultigridModel.cs:76-194): radial influence 1 - |(w - c)/h| of
// the fine nodes in a window around each coarse node, restriction rows and
// interpolation rows normalised to sum 1 before the fixed dofs are removed,
// the same weight for every dof of a node, free-dof submatrices.
// ---------------------------------------------------------------------------
namespace {
struct TransferBuild {
    std::vector<std::vector<std::pair<int32_t, double>>> R, P;   // free rows: (free col, value)
};
void build_transfer(int dim, const int32_t *nef, const int32_t *nec, int dpn, int32_t nff, const int32_t *ff,
                    int32_t ncf, const int32_t *cf, TransferBuild &out) {
    DV_REQUIRE(dim == 2 || dim == 3, DV_ERR_ARG, "dim must be 2 or 3");
    DV_REQUIRE(dpn >= 1, DV_ERR_ARG, "dofs per node must be positive");
    int nfn[3] = {1, 1, 1}, ncn[3] = {1, 1, 1};
    double dist[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i) {
        DV_REQUIRE(nef[i] >= 1 && nec[i] >= 1, DV_ERR_ARG, "element counts must be positive");
        dist[i] = (double)nef[i] / nec[i];
        nfn[i] = nef[i] + 1;
        ncn[i] = nec[i] + 1;
    }
    const int64_t nf_nodes = (int64_t)nfn[0] * nfn[1] * nfn[2], nc_nodes = (int64_t)ncn[0] * ncn[1] * ncn[2];
    std::vector<int32_t> fmap(nf_nodes * dpn, -1), cmap(nc_nodes * dpn, -1);
    for (int32_t i = 0; i < nff; ++i) {
        DV_REQUIRE(ff[i] >= 0 && ff[i] < nf_nodes * dpn, DV_ERR_ARG, "fine free dof out of range");
        fmap[ff[i]] = i;
    }
    for (int32_t i = 0; i < ncf; ++i) {
        DV_REQUIRE(cf[i] >= 0 && cf[i] < nc_nodes * dpn, DV_ERR_ARG, "coarse free dof out of range");
        cmap[cf[i]] = i;
    }
    struct Tri { int32_t c, f; double v; };
    std::vector<Tri> tris;
    std::vector<double> sum_r(nc_nodes, 0.0), sum_i(nf_nodes, 0.0);
    int a[3] = {0, 0, 0}, start[3] = {0, 0, 0}, end[3] = {0, 0, 0}, w[3] = {0, 0, 0};
    double cursor[3] = {0, 0, 0};
    if (dim < 3) end[2] = 1;
    for (a[0] = 0; a[0] < ncn[0]; ++a[0])
        for (a[2] = 0; a[2] < ncn[2]; ++a[2])
            for (a[1] = 0; a[1] < ncn[1]; ++a[1]) {
                for (int i = 0; i < dim; ++i) {
                    cursor[i] = a[i] * dist[i];
                    start[i] = (int)std::ceil(std::nextafter(cursor[i] - dist[i], INFINITY));
                    if (start[i] < 0) start[i] = 0;
                    end[i] = (int)std::floor(std::nextafter(cursor[i] + dist[i], -INFINITY)) + 1;
                    if (end[i] > nfn[i]) end[i] = nfn[i];
                }
                int32_t cnode = a[0] + a[1] * ncn[0] + (dim == 3 ? a[2] * ncn[0] * ncn[1] : 0);
                double s = 0;
                for (w[0] = start[0]; w[0] < end[0]; ++w[0])
                    for (w[2] = start[2]; w[2] < end[2]; ++w[2])
                        for (w[1] = start[1]; w[1] < end[1]; ++w[1]) {
                            int32_t fnode = w[0] + w[1] * nfn[0] + (dim == 3 ? w[2] * nfn[0] * nfn[1] : 0);
                            double infl = 0;
                            for (int i = 0; i < dim; ++i) {
                                double d0 = (w[i] - cursor[i]) / dist[i];
                                infl += d0 * d0;
                            }
                            infl = 1 - std::sqrt(infl);
                            s += infl;
                            sum_i[fnode] += infl;
                            tris.push_back({cnode, fnode, infl});
                        }
                sum_r[cnode] = s;
            }
    out.R.assign(ncf, {});
    out.P.assign(nff, {});
    for (const Tri &t : tris) {
        double rv = t.v / sum_r[t.c], pv = t.v / sum_i[t.f];
        for (int d = 0; d < dpn; ++d) {
            int32_t cr = cmap[(int64_t)t.c * dpn + d], fr = fmap[(int64_t)t.f * dpn + d];
            if (cr >= 0 && fr >= 0) {
                out.R[cr].push_back({fr, rv});
                out.P[fr].push_back({cr, pv});
            }
        }
    }
    for (auto &row : out.R) std::sort(row.begin(), row.end(), [](auto &x, auto &y) { return x.first < y.first; });
    for (auto &row : out.P) std::sort(row.begin(), row.end(), [](auto &x, auto &y) { return x.first < y.first; });
}
}  // namespace

extern "C" DV_API int dv_cartesian_transfer_size(int32_t dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                                                 int32_t dofs_per_node, int32_t n_fine_free, const int32_t *fine_free,
                                                 int32_t n_coarse_free, const int32_t *coarse_free, int64_t *nnz_r,
                                                 int64_t *nnz_p) {
    return dv_guard([&] {
        DV_REQUIRE(ne_fine && ne_coarse && fine_free && coarse_free && nnz_r && nnz_p, DV_ERR_ARG, "null argument");
        TransferBuild t;
        build_transfer(dim, ne_fine, ne_coarse, dofs_per_node, n_fine_free, fine_free, n_coarse_free, coarse_free, t);
        int64_t r = 0, p = 0;
        for (auto &row : t.R) r += (int64_t)row.size();
        for (auto &row : t.P) p += (int64_t)row.size();
        *nnz_r = r;
        *nnz_p = p;
    });
}

extern "C" DV_API int dv_cartesian_transfer(int32_t dim, const int32_t *ne_fine, const int32_t *ne_coarse,
                                            int32_t dofs_per_node, int32_t n_fine_free, const int32_t *fine_free,
                                            int32_t n_coarse_free, const int32_t *coarse_free, int32_t *r_rowptr,
                                            int32_t *r_col, double *r_val, int32_t *p_rowptr, int32_t *p_col,
                                            double *p_val) {
    return dv_guard([&] {
        DV_REQUIRE(ne_fine && ne_coarse && fine_free && coarse_free && r_rowptr && r_col && r_val && p_rowptr &&
                       p_col && p_val, DV_ERR_ARG, "null argument");
        TransferBuild t;
        build_transfer(dim, ne_fine, ne_coarse, dofs_per_node, n_fine_free, fine_free, n_coarse_free, coarse_free, t);
        auto emit = [](const std::vector<std::vector<std::pair<int32_t, double>>> &rows, int32_t *rp, int32_t *ci, double *va) {
            int64_t k = 0;
            rp[0] = 0;
            for (size_t i = 0; i < rows.size(); ++i) {
                for (auto &cv : rows[i]) { ci[k] = cv.first; va[k] = cv.second; ++k; }
                rp[i + 1] = (int32_t)k;
            }
        };
        emit(t.R, r_rowptr, r_col, r_val);
        emit(t.P, p_rowptr, p_col, p_val);
    });
}
