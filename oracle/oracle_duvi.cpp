// CPU oracle: DuVi formats (GPU SoA and CPU Unit stream).  Test infrastructure only.
#include "oracle_internal.hpp"

#include <cmath>
#include <stdexcept>

// ---------------------------------------------------------------------------
// .NET double hashing and the DuVi tolerance dictionary
// ---------------------------------------------------------------------------
// double.GetHashCode (.NET 8): NaNs and both zeros are normalised, then the two
// 32-bit halves of the bit pattern are xor-ed.
int32_t dotnet_double_hash(double x) {
    uint64_t bits;
    std::memcpy(&bits, &x, 8);
    const uint64_t sign = 0x8000000000000000ull, pinf = 0x7FF0000000000000ull;
    if (((bits - 1) & ~sign) >= pinf) bits &= pinf;
    return (int32_t)(uint32_t)bits ^ (int32_t)(uint32_t)(bits >> 32);
}

// ToleranceComparer.GetHashCode = Math.Round(x / (2 * tolerance)).GetHashCode()
// (round half to even); Equals = |x - y| < tolerance.  Without a tolerance the
// default comparer: x == y or both NaN.
int32_t DoubleIndexMap::hash(double x) const {
    if (tol > 0) return dotnet_double_hash(std::nearbyint(x / (2 * tol)));
    return dotnet_double_hash(x);
}
bool DoubleIndexMap::equal(double stored, double key) const {
    if (tol > 0) return std::fabs(stored - key) < tol;
    return stored == key || (std::isnan(stored) && std::isnan(key));
}
// Dictionary.FindValue walks the bucket chain newest-first and accepts the
// first entry with an equal 32-bit hash code and Equals() true.
int32_t DoubleIndexMap::find(double v) const {
    auto it = classes.find(hash(v));
    if (it == classes.end()) return -1;
    const auto &ids = it->second;
    for (size_t i = ids.size(); i-- > 0;)
        if (equal(keys[ids[i]], v)) return ids[i];
    return -1;
}
int32_t DoubleIndexMap::insert(double v) {
    int32_t id = (int32_t)keys.size();
    keys.push_back(v);
    classes[hash(v)].push_back(id);
    return id;
}

// ---------------------------------------------------------------------------
// GPU SoA DuVi (OpenCLDuViGeometricMultigridSolver.cs:16-31, 753-851)
// ---------------------------------------------------------------------------
struct or_duvi {
    int32_t n_rows = 0;
    std::vector<uint32_t> row_to_col, row_to_dist, col_idx, vidx;
    std::vector<uint8_t> dist;
    std::vector<double> values;
    int vi_bits = 8;
};

extern "C" or_duvi *or_duvi_encode(const or_csr *a, double tol, int force_bits) {
    or_duvi *B = new or_duvi;
    int32_t n = a->n_rows;
    int64_t nnz = (int64_t)a->val.size();
    B->n_rows = n;
    B->row_to_col.assign(n + 1, 0);
    B->row_to_dist.assign(n + 1, 0);
    B->dist.assign(nnz, 0);
    // "DU" part: blocks of column runs with gaps below 256 and at most 256 entries.
    int64_t value_index = 0, value_begin = 0;
    for (int32_t i = 0;; ++i) {
        B->row_to_col[i] = (uint32_t)B->col_idx.size();
        B->row_to_dist[i] = (uint32_t)value_index;
        if (i == n) break;
        int32_t from = a->rowptr[i], to = a->rowptr[i + 1];
        for (int32_t j = from; j < to; ++j) {
            int block_count = 0;
            B->col_idx.push_back((uint32_t)a->col[j]);
            for (; j + 1 < to && block_count < 255; ++j) {
                int32_t diff = a->col[j + 1] - a->col[j] - 1;
                if (diff < 256) {
                    ++block_count;
                    ++value_index;
                    B->dist[value_index] = (uint8_t)diff;
                } else break;
            }
            B->dist[value_begin] = (uint8_t)block_count;
            ++value_index;
            value_begin = value_index;
        }
    }
    // "VI" part: value dedup in CSR order.  Up to 256 distinct values this is
    // the reference encoder; beyond that the reference promotion is broken
    // (:818-824 copies with the wrong index, :814 returns an unusable matrix),
    // so wider indices keep the same first-occurrence numbering.
    DoubleIndexMap map(tol);
    B->vidx.resize(nnz);
    for (int64_t i = 0; i < nnz; ++i) {
        double v = a->val[i];
        int32_t idx = map.find(v);
        if (idx < 0) idx = map.insert(v);
        B->vidx[i] = (uint32_t)idx;
    }
    B->values = map.keys;
    int64_t nu = (int64_t)B->values.size();
    int bits = nu <= 256 ? 8 : (nu <= 65536 ? 16 : 32);
    if (force_bits > bits) bits = force_bits;
    B->vi_bits = bits;
    return B;
}
extern "C" void or_duvi_free(or_duvi *d) { delete d; }
extern "C" void or_duvi_info(const or_duvi *d, int64_t *s) {
    s[0] = d->n_rows; s[1] = (int64_t)d->col_idx.size(); s[2] = (int64_t)d->dist.size();
    s[3] = (int64_t)d->values.size(); s[4] = d->vi_bits;
}
extern "C" void or_duvi_copy(const or_duvi *d, uint32_t *rc, uint32_t *rd, uint32_t *ci, uint8_t *dist,
                             uint32_t *vidx, double *values) {
    if (rc) std::memcpy(rc, d->row_to_col.data(), 4 * d->row_to_col.size());
    if (rd) std::memcpy(rd, d->row_to_dist.data(), 4 * d->row_to_dist.size());
    if (ci) std::memcpy(ci, d->col_idx.data(), 4 * d->col_idx.size());
    if (dist) std::memcpy(dist, d->dist.data(), d->dist.size());
    if (vidx) std::memcpy(vidx, d->vidx.data(), 4 * d->vidx.size());
    if (values) std::memcpy(values, d->values.data(), 8 * d->values.size());
}
// matrix_vector_product_partial (DuViGeometricMultigrid.cl:57-99): accumulate
// straight into y[row].
extern "C" void or_duvi_spmv(const or_duvi *d, const double *x, double *y, int clear) {
    for (int32_t row = 0; row < d->n_rows; ++row) {
        if (clear) y[row] = 0;
        uint32_t ci = d->row_to_col[row], ci_to = d->row_to_col[row + 1];
        uint32_t di = d->row_to_dist[row];
        for (; ci < ci_to; ++ci) {
            uint32_t column = d->col_idx[ci];
            uint32_t di_to = di + d->dist[di] + 1;
            for (;;) {
                y[row] += d->values[d->vidx[di]] * x[column];
                ++di;
                if (di == di_to) break;
                column += d->dist[di] + 1u;
            }
        }
    }
}
// Dense decode in the walk order of DuVi2Mat (OpenCLDuViGeometricMultigridSolver.cs:394-415).
// That debug-only routine leaves its cursor on a block's last entry, so from
// the second block of a row on it reads a gap byte as the block count; the
// decode here advances past the block as the kernels do
// (DuViGeometricMultigrid.cl:84-98).
extern "C" void or_duvi_to_dense(const or_duvi *d, int32_t n_cols, double *B) {
    std::memset(B, 0, sizeof(double) * (size_t)d->n_rows * n_cols);
    for (int32_t row = 0; row < d->n_rows; ++row) {
        uint32_t cb = d->row_to_col[row], ce = d->row_to_col[row + 1];
        uint32_t di = d->row_to_dist[row];
        for (uint32_t j = cb; j < ce; ++j) {
            uint32_t column = d->col_idx[j];
            for (int blk = d->dist[di]; blk > 0; --blk) {
                B[(size_t)row * n_cols + column] = d->values[d->vidx[di]];
                column += 1 + d->dist[++di];
            }
            B[(size_t)row * n_cols + column] = d->values[d->vidx[di]];
            ++di;   // DuVi2Mat leaves dstIdx on the last entry; the next block starts after it
        }
    }
}

// ---------------------------------------------------------------------------
// CPU Unit stream (DuViCompressedSparseMatrix.cs:11-152, 176-441)
// ---------------------------------------------------------------------------
struct or_units {
    std::vector<uint8_t> bytes;
    std::vector<int64_t> offsets;   // unit start offsets (n_units + 1)
    std::vector<int32_t> vidx;
    std::vector<double> values;
};

enum DeltaBytes { ONE = 0, TWO = 1, FOUR = 2 };
static const int LOW2 = 1 << 7, LOW3 = (1 << 14) + LOW2, LOW4 = (1 << 21) + LOW3, LOW5 = (1 << 29) + LOW4;

// Unit constructor (DuViCompressedSparseMatrix.cs:13-88).
static void push_unit(or_units *u, bool new_row, int db, int next_col, const std::vector<int> &deltas) {
    if (next_col >= LOW5) throw std::runtime_error("unit column gap not representable");
    int vbytes = next_col >= LOW4 ? 4 : next_col >= LOW3 ? 3 : next_col >= LOW2 ? 2 : 1;
    size_t total = 2 + vbytes + (size_t)(1 << db) * deltas.size();
    size_t o = u->bytes.size();
    u->offsets.push_back((int64_t)o);
    u->bytes.resize(o + total);
    uint8_t *data = u->bytes.data() + o;
    data[0] = (uint8_t)((new_row ? 1 : 0) | (db << 1));
    data[1] = (uint8_t)deltas.size();
    int nc = next_col, t;
    if (nc >= LOW4) { nc -= LOW4; data[2] = (uint8_t)((nc >> 24) | 128 | 64 | 32); data[3] = (uint8_t)(nc >> 16); data[4] = (uint8_t)(nc >> 8); data[5] = (uint8_t)nc; t = 6; }
    else if (nc >= LOW3) { nc -= LOW3; data[2] = (uint8_t)((nc >> 16) | 128 | 64); data[3] = (uint8_t)(nc >> 8); data[4] = (uint8_t)nc; t = 5; }
    else if (nc >= LOW2) { nc -= LOW2; data[2] = (uint8_t)((nc >> 8) | 128); data[3] = (uint8_t)nc; t = 4; }
    else { data[2] = (uint8_t)nc; t = 3; }
    for (int dlt : deltas) {
        data[t++] = (uint8_t)dlt;
        if (db >= TWO) data[t++] = (uint8_t)(dlt >> 8);
        if (db == FOUR) { data[t++] = (uint8_t)(dlt >> 16); data[t++] = (uint8_t)(dlt >> 24); }
    }
}

// ExtractVariableInteger (:108-119): returns (value, size).
static std::pair<int, int> extract_varint(const uint8_t *data, int index) {
    if ((data[index] & 128) == 0) return {data[index], 1};
    if ((data[index] & 64) == 0) return {LOW2 + (((data[index] & 63) << 8) | data[index + 1]), 2};
    if ((data[index] & 32) == 0) return {LOW3 + (((data[index] & 31) << 16) | (data[index + 1] << 8) | data[index + 2]), 3};
    return {LOW4 + (((data[index] & 31) << 24) | (data[index + 1] << 16) | (data[index + 2] << 8) | data[index + 3]), 4};
}
// GetIndex (:138-151).
static int get_index(const uint8_t *data, int index, int db, int off) {
    if (db == ONE) return data[off + index];
    if (db == TWO) { off += index * 2; return data[off] | (data[off + 1] << 8); }
    off += index * 4;
    return data[off] | (data[off + 1] << 8) | (data[off + 2] << 16) | (data[off + 3] << 24);
}

static void add_value(DoubleIndexMap &map, or_units *u, double v) {
    int32_t idx = map.find(v);
    if (idx < 0) idx = map.insert(v);
    u->vidx.push_back(idx);
}

// Per-row delta grouping shared by both constructors (:214-277 and :319-394).
struct UnitBuilder {
    or_units *u;
    int db = ONE;
    bool new_row = true;
    int delta_next_unit = -1;
    std::vector<int> delta_cols;
    void step(int delta) {
        int want = delta < 256 ? ONE : delta < 65536 ? TWO : FOUR;
        if (db != want) {
            if (!delta_cols.empty()) {
                push_unit(u, new_row, db, delta_next_unit, delta_cols);
                new_row = false;
                delta_next_unit = delta;
                delta_cols.clear();
            } else delta_cols.push_back(delta);
            db = want;
        } else delta_cols.push_back(delta);
    }
};

extern "C" or_units *or_units_from_dense(int32_t h, int32_t w, const double *values, double tol) {
    or_units *u = new or_units;
    DoubleIndexMap map(tol > 0 ? tol : 0);
    int64_t in = 0;
    for (int32_t y = 0; y < h; ++y) {
        UnitBuilder ub{u};
        int x_old = -1, x;
        for (x = 0; x < w; ++x) {
            double v = values[in++];
            if (std::fabs(v) > tol) {
                add_value(map, u, v);
                x_old = x; ub.delta_next_unit = x;
                ++x;
                break;
            }
        }
        for (; x < w; ++x) {
            double v = values[in++];
            if (std::fabs(v) > tol) {
                add_value(map, u, v);
                ub.step(x - x_old);
                x_old = x;
            }
        }
        if (ub.delta_next_unit != -1) push_unit(u, ub.new_row, ub.db, ub.delta_next_unit, ub.delta_cols);
    }
    u->offsets.push_back((int64_t)u->bytes.size());
    u->values = map.keys;
    return u;
}

extern "C" or_units *or_units_from_csr(const or_csr *a, double tol) {
    or_units *u = new or_units;
    DoubleIndexMap map(tol > 0 ? tol : 0);
    for (int32_t y = 0; y < a->n_rows; ++y) {
        int32_t rs = a->rowptr[y];
        if (a->rowptr[y + 1] - rs == 0) {
            add_value(map, u, 0.0);
            push_unit(u, true, ONE, 0, {});
            continue;
        }
        UnitBuilder ub{u};
        int x_old = a->col[rs];
        ub.delta_next_unit = x_old;
        add_value(map, u, a->val[rs]);
        for (int32_t idx = rs + 1; idx < a->rowptr[y + 1]; ++idx) {
            add_value(map, u, a->val[idx]);
            int x = a->col[idx];
            ub.step(x - x_old);
            x_old = x;
        }
        push_unit(u, ub.new_row, ub.db, ub.delta_next_unit, ub.delta_cols);
    }
    u->offsets.push_back((int64_t)u->bytes.size());
    u->values = map.keys;
    return u;
}
extern "C" void or_units_free(or_units *u) { delete u; }
extern "C" void or_units_info(const or_units *u, int64_t *s) {
    s[0] = (int64_t)u->offsets.size() - 1; s[1] = (int64_t)u->bytes.size();
    s[2] = (int64_t)u->vidx.size(); s[3] = (int64_t)u->values.size();
}
extern "C" void or_units_copy(const or_units *u, uint8_t *bytes, int64_t *off, int32_t *vidx, double *values) {
    if (bytes) std::memcpy(bytes, u->bytes.data(), u->bytes.size());
    if (off) std::memcpy(off, u->offsets.data(), 8 * u->offsets.size());
    if (vidx) std::memcpy(vidx, u->vidx.data(), 4 * u->vidx.size());
    if (values) std::memcpy(values, u->values.data(), 8 * u->values.size());
}
// Multiply (:421-441).
extern "C" void or_units_multiply(const or_units *u, const double *x, double *y) {
    int row = -1, col = 0, vi = 0;
    size_t nu = u->offsets.size() - 1;
    for (size_t k = 0; k < nu; ++k) {
        const uint8_t *d = u->bytes.data() + u->offsets[k];
        if (d[0] & 1) { ++row; col = 0; y[row] = 0; }
        int total = d[1];
        auto [delta, size] = extract_varint(d, 2);
        size += 2;
        col += delta;
        double value = u->values[u->vidx[vi++]];
        y[row] += value * x[col];
        int db = d[0] >> 1;
        for (int i = 0; i < total; ++i) {
            col += get_index(d, i, db, size);
            value = u->values[u->vidx[vi++]];
            y[row] += value * x[col];
        }
    }
}
// Indexer get (:450-484).
extern "C" double or_units_get(const or_units *u, int32_t row_idx, int32_t col_idx) {
    int row = -1, col = 0, vi = 0;
    size_t nu = u->offsets.size() - 1;
    for (size_t k = 0; k < nu; ++k) {
        const uint8_t *d = u->bytes.data() + u->offsets[k];
        if (d[0] & 1) { ++row; col = 0; }
        int total = d[1];
        auto [delta, size] = extract_varint(d, 2);
        size += 2;
        col += delta;
        if (row == row_idx) {
            if (col == col_idx) return u->values[u->vidx[vi]];
            else if (col > col_idx) return 0;
        } else if (row > row_idx) return 0;
        ++vi;
        int db = d[0] >> 1;
        for (int i = 0; i < total; ++i) {
            col += get_index(d, i, db, size);
            if (row == row_idx) {
                if (col == col_idx) return u->values[u->vidx[vi]];
                else if (col > col_idx) return 0;
            } else if (row > row_idx) return 0;
            ++vi;
        }
    }
    return 0;
}
// GaussSeidelIterationCsrDuVi.Execute (GaussSeidelIterationCsrDuVi.cs:22-50).
extern "C" void or_units_gs(const or_units *u, const double *b, double *x) {
    int row = -1, col = 0, k = 0;
    double divisor = 0;
    size_t nu = u->offsets.size() - 1;
    for (size_t q = 0; q < nu; ++q) {
        const uint8_t *d = u->bytes.data() + u->offsets[q];
        int db = d[0] >> 1;
        if (d[0] & 1) {
            if (row != -1) x[row] /= divisor;
            ++row; col = 0;
            x[row] = b[row];
        }
        auto [delta, offset] = extract_varint(d, 2);
        offset += 2;
        col += delta;
        int total = d[1], i = 0;
        for (;;) {
            double a = u->values[u->vidx[k++]];
            if (row != col) x[row] -= a * x[col];
            else divisor = a;
            if (i == total) break;
            col += get_index(d, i++, db, offset);
        }
    }
    x[row] /= divisor;
}
