// The CPU DuVi "Unit" stream of the reference (DuViCompressedSparseMatrix,
// DuViCompressedSparseMatrix.cs:11-152 units, :285-400 CSR constructor,
// :419-441 Multiply), as a flat byte stream for storage and interchange.
//
// A row is one or more units.  A unit holds a run of column steps of one
// width: byte 0 = new-row flag (bit 0) | step width class << 1 (0: 1 byte,
// 1: 2 bytes, 2: 4 bytes); byte 1 = number of steps; then the column gap to
// the unit's first entry (from column 0 for a row's first unit, else from the
// previous unit's last entry) as a big-endian prefix code of 1-4 bytes
// (0xxxxxxx; 10xxxxxx +128; 110xxxxx +16,512; 111xxxxx +2,113,664); then the
// steps, little-endian.  A unit ends where the step width changes; a step
// that changes the width of a unit with no steps yet joins that unit.  An
// empty row is one unit with no steps and gap 0 whose value is 0.0.  Values
// are numbered in entry order through the reference's Dictionary semantics
// (int32 indices into a table of distinct values).
//
// The reference stores the step count in one byte and wraps above 255; its
// units are separate arrays, so only that row's tail is lost.  In one flat
// stream a wrapped count would misplace every later unit, so such rows are
// rejected here (DV_ERR_FORMAT), as are gaps of 2^29 + 2,113,664 or more
// (the reference throws NotImplementedException).
#include "dv_internal.cuh"

#include <algorithm>
#include <numeric>

namespace {

constexpr int64_t kLow2 = 1 << 7;
constexpr int64_t kLow3 = (1 << 14) + kLow2;
constexpr int64_t kLow4 = (1 << 21) + kLow3;
constexpr int64_t kLow5 = (1 << 29) + kLow4;

int width_class(int64_t step) { return step < 256 ? 0 : step < 65536 ? 1 : 2; }
int gap_bytes(int64_t gap) { return gap >= kLow4 ? 4 : gap >= kLow3 ? 3 : gap >= kLow2 ? 2 : 1; }

// Walks the units of one row as the reference constructor forms them:
// emit(new_row, width class, gap, first step index, step count) per unit,
// steps being col[k + 1] - col[k] for k in [first, first + count).
template <class Emit>
void row_units(const int32_t *col, int32_t b, int32_t e, Emit emit) {
    if (b == e) {
        emit(true, 0, 0, b, 0);
        return;
    }
    bool new_row = true;
    int cls = 0;
    int64_t gap = col[b];
    int32_t first = b, count = 0;   // steps of the open unit: first .. first + count - 1
    for (int32_t k = b; k + 1 < e; ++k) {
        const int64_t step = (int64_t)col[k + 1] - col[k];
        const int want = width_class(step);
        if (want != cls && count > 0) {
            emit(new_row, cls, gap, first, count);
            new_row = false;
            gap = step;
            first = k + 1;
            count = 0;
        } else {
            ++count;
        }
        cls = want;
    }
    emit(new_row, cls, gap, first, count);
}

}  // namespace

extern "C" DV_API int dv_units_encode(const dv_csr_host *a, double dedup_tol, int64_t *n_units, int64_t *n_bytes,
                                      int64_t *n_indices, int64_t *nuniq, uint8_t *bytes, int64_t *unit_offsets,
                                      int32_t *value_indices, double *values) {
    return dv_guard([&] {
        DV_REQUIRE(a && n_units && n_bytes && n_indices && nuniq, DV_ERR_ARG, "null argument");
        dv_check_csr(*a);
        const int32_t n = a->n_rows;
        // units and bytes per row
        std::vector<int64_t> ru(n + 1, 0), rb(n + 1, 0);
        int32_t bad_row = INT32_MAX;
#pragma omp parallel for schedule(static) reduction(min : bad_row)
        for (int32_t i = 0; i < n; ++i) {
            int64_t u = 0, by = 0;
            bool ok = true;
            row_units(a->col, a->rowptr[i], a->rowptr[i + 1], [&](bool, int cls, int64_t gap, int32_t, int32_t cnt) {
                ok = ok && cnt <= 255 && gap < kLow5;
                ++u;
                by += 2 + gap_bytes(gap) + ((int64_t)1 << cls) * cnt;
            });
            if (!ok) bad_row = std::min(bad_row, i);
            ru[i + 1] = u;
            rb[i + 1] = by;
        }
        DV_REQUIRE(bad_row == INT32_MAX, DV_ERR_FORMAT,
                   "row " + std::to_string(bad_row) +
                       ": a unit of more than 255 column steps or a column gap of 2^29 + 2,113,664 or more is not "
                       "representable in the DuVi Unit stream");
        std::partial_sum(ru.begin(), ru.end(), ru.begin());
        std::partial_sum(rb.begin(), rb.end(), rb.begin());
        // the values in the constructor's order: each entry, and 0.0 for an empty row
        const int64_t nnz = a->rowptr[n];
        int64_t empty = 0;
#pragma omp parallel for schedule(static) reduction(+ : empty)
        for (int32_t i = 0; i < n; ++i) empty += a->rowptr[i + 1] == a->rowptr[i];
        *n_units = ru[n];
        *n_bytes = rb[n];
        *n_indices = nnz + empty;
        std::vector<double> seq;
        const double *vals = a->val;
        if (empty > 0) {
            seq.reserve(nnz + empty);
            for (int32_t i = 0; i < n; ++i) {
                if (a->rowptr[i + 1] == a->rowptr[i]) seq.push_back(0.0);
                else seq.insert(seq.end(), a->val + a->rowptr[i], a->val + a->rowptr[i + 1]);
            }
            vals = seq.data();
        }
        std::vector<uint32_t> idx(nnz + empty);
        const std::vector<double> keys = dv_number_values(vals, nnz + empty, dedup_tol, idx.data());
        *nuniq = (int64_t)keys.size();
        if (!bytes) return;   // sizes only
        DV_REQUIRE(unit_offsets && value_indices && values, DV_ERR_ARG, "null output array");
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            int64_t u = ru[i], o = rb[i];
            row_units(a->col, a->rowptr[i], a->rowptr[i + 1],
                      [&](bool new_row, int cls, int64_t gap, int32_t first, int32_t cnt) {
                          unit_offsets[u++] = o;
                          uint8_t *d = bytes + o;
                          d[0] = (uint8_t)((new_row ? 1 : 0) | (cls << 1));
                          d[1] = (uint8_t)cnt;
                          int t = 2;
                          if (gap >= kLow4) {
                              const int64_t g = gap - kLow4;
                              d[t++] = (uint8_t)((g >> 24) | 0xE0);
                              d[t++] = (uint8_t)(g >> 16);
                              d[t++] = (uint8_t)(g >> 8);
                              d[t++] = (uint8_t)g;
                          } else if (gap >= kLow3) {
                              const int64_t g = gap - kLow3;
                              d[t++] = (uint8_t)((g >> 16) | 0xC0);
                              d[t++] = (uint8_t)(g >> 8);
                              d[t++] = (uint8_t)g;
                          } else if (gap >= kLow2) {
                              const int64_t g = gap - kLow2;
                              d[t++] = (uint8_t)((g >> 8) | 0x80);
                              d[t++] = (uint8_t)g;
                          } else {
                              d[t++] = (uint8_t)gap;
                          }
                          const int w = 1 << cls;
                          for (int32_t s = 0; s < cnt; ++s) {
                              const uint32_t step = (uint32_t)(a->col[first + s + 1] - a->col[first + s]);
                              for (int q = 0; q < w; ++q) d[t++] = (uint8_t)(step >> (8 * q));
                          }
                          o += t;
                      });
        }
        unit_offsets[ru[n]] = rb[n];
        for (int64_t k = 0; k < nnz + empty; ++k) value_indices[k] = (int32_t)idx[k];
        std::copy(keys.begin(), keys.end(), values);
    });
}

extern "C" DV_API int dv_units_decode(int32_t n_rows, int32_t n_cols, const uint8_t *bytes, int64_t n_bytes,
                                      const int32_t *value_indices, int64_t n_indices, const double *values,
                                      int64_t nuniq, int64_t *nnz, int32_t *rowptr, int32_t *col, double *val) {
    return dv_guard([&] {
        DV_REQUIRE(n_rows >= 0 && n_cols >= 0 && nnz && (bytes || n_bytes == 0) && (value_indices || n_indices == 0) &&
                       (values || nuniq == 0),
                   DV_ERR_ARG, "null argument");
        // one walk over the units (Multiply's order); with rowptr == NULL it only counts
        int64_t o = 0, k = 0;
        int32_t row = -1;
        int64_t c = 0;
        auto need = [&](int64_t m) { DV_REQUIRE(o + m <= n_bytes, DV_ERR_FORMAT, "unit stream ends inside a unit"); };
        auto put = [&](int64_t column) {
            DV_REQUIRE(row >= 0, DV_ERR_FORMAT, "unit stream does not start a row");
            DV_REQUIRE(column < n_cols, DV_ERR_FORMAT, "column beyond the matrix width");
            DV_REQUIRE(k < n_indices, DV_ERR_FORMAT, "fewer value indices than entries");
            const int32_t vi = value_indices[k];
            DV_REQUIRE(vi >= 0 && vi < nuniq, DV_ERR_FORMAT, "value index out of range");
            if (rowptr) {
                col[k] = (int32_t)column;
                val[k] = values[vi];
            }
            ++k;
        };
        while (o < n_bytes) {
            need(3);
            const uint8_t h = bytes[o], cnt = bytes[o + 1];
            const int cls = h >> 1;
            DV_REQUIRE(cls <= 2 && (h & ~0x7u) == 0, DV_ERR_FORMAT, "bad unit header");
            if (h & 1) {
                ++row;
                DV_REQUIRE(row < n_rows, DV_ERR_FORMAT, "more rows than the matrix height");
                if (rowptr) rowptr[row] = (int32_t)k;
                c = 0;
            }
            o += 2;
            const uint8_t b0 = bytes[o];
            int64_t gap;
            if (!(b0 & 0x80)) {
                gap = b0;
                o += 1;
            } else if (!(b0 & 0x40)) {
                need(2);
                gap = kLow2 + (((int64_t)(b0 & 63) << 8) | bytes[o + 1]);
                o += 2;
            } else if (!(b0 & 0x20)) {
                need(3);
                gap = kLow3 + (((int64_t)(b0 & 31) << 16) | ((int64_t)bytes[o + 1] << 8) | bytes[o + 2]);
                o += 3;
            } else {
                need(4);
                gap = kLow4 + (((int64_t)(b0 & 31) << 24) | ((int64_t)bytes[o + 1] << 16) |
                               ((int64_t)bytes[o + 2] << 8) | bytes[o + 3]);
                o += 4;
            }
            DV_REQUIRE(gap > 0 || (h & 1), DV_ERR_FORMAT, "columns of a row not increasing (zero gap between units)");
            c += gap;
            put(c);
            const int w = 1 << cls;
            need((int64_t)w * cnt);
            for (int s = 0; s < cnt; ++s) {
                uint32_t step = 0;
                for (int q = 0; q < w; ++q) step |= (uint32_t)bytes[o + q] << (8 * q);
                o += w;
                DV_REQUIRE(step > 0, DV_ERR_FORMAT, "columns of a row not increasing (zero step)");
                c += step;
                put(c);
            }
        }
        DV_REQUIRE(row == n_rows - 1, DV_ERR_FORMAT, "fewer rows than the matrix height");
        DV_REQUIRE(k == n_indices, DV_ERR_FORMAT, "more value indices than entries");
        DV_REQUIRE(k <= INT32_MAX, DV_ERR_FORMAT, "too many entries for int32 row offsets");
        *nnz = k;
        if (rowptr) rowptr[n_rows] = (int32_t)k;
    });
}
