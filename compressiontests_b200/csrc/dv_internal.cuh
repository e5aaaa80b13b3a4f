// Internal declarations of libduvigpu.so (B200 sparse solver path).
#pragma once

#include "../../include/duvi_gpu.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <climits>
#include <vector>

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct DvError : std::runtime_error {
    int code;
    DvError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define DV_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw DvError(e_ == cudaErrorMemoryAllocation ? DV_ERR_NOMEM : DV_ERR_CUDA,        \
                          std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

#define DV_REQUIRE(cond, code, msg)                   \
    do {                                              \
        if (!(cond)) throw DvError((code), (msg));    \
    } while (0)

void dv_set_last_error(const std::string &m);

// Runs f, converting exceptions into status codes and the thread-local message.
template <class F>
int dv_guard(F &&f) {
    try {
        f();
        return DV_OK;
    } catch (const DvError &e) {
        dv_set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        dv_set_last_error("host allocation failed");
        return DV_ERR_NOMEM;
    } catch (const std::exception &e) {
        dv_set_last_error(e.what());
        return DV_ERR_ARG;
    }
}

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
struct DevMem {
    void *p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    explicit DevMem(size_t b) { alloc(b); }
    DevMem(const DevMem &) = delete;
    DevMem &operator=(const DevMem &) = delete;
    DevMem(DevMem &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevMem &operator=(DevMem &&o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevMem() { release(); }
    void alloc(size_t b) {
        release();
        // 64 bytes of tail padding: staged loads round ranges up to 16-byte units.
        // The zero fill runs on the legacy stream, which does not order against the
        // non-blocking context streams: finish it before anyone writes the buffer.
        if (b) {
            DV_CUDA(cudaMalloc(&p, b + 64));
            DV_CUDA(cudaMemsetAsync(p, 0, b + 64, 0));
            DV_CUDA(cudaStreamSynchronize(0));
        }
        bytes = b;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Grid-wide deterministic reduction workspace: per-block partials and a ticket.
struct ReduceWs {
    double *partials = nullptr;   // [max_blocks * 8]
    unsigned *ticket = nullptr;
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct dv_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    int max_smem_optin = 0;
    // Kernel launches, counted by where they go: work done for the caller (dv_context_launch_count),
    // the autotuner's trial launches at matrix upload, and launches recorded into a CUDA graph
    // (counted into `launches` each time the graph runs).
    enum CountInto { kCountWork = 0, kCountTuning = 1, kCountCapture = 2 };
    int64_t launches = 0, tuning_launches = 0, captured_launches = 0;
    int count_into = kCountWork;
    DevMem red;          // default grid-reduction workspace (ticket + partials)
    void count(int64_t n = 1) {
        if (count_into == kCountTuning) tuning_launches += n;
        else if (count_into == kCountCapture) captured_launches += n;
        else launches += n;
    }
};

// Sends the context's launch counts to `into` while in scope.
struct CountScope {
    dv_context *ctx;
    int saved;
    CountScope(dv_context *c, int into) : ctx(c), saved(c->count_into) { c->count_into = into; }
    ~CountScope() { ctx->count_into = saved; }
};

void dv_ctx_check(dv_context *ctx);   // throws DV_ERR_NO_DEVICE / DV_ERR_CUDA

// ---------------------------------------------------------------------------
// matrices
// ---------------------------------------------------------------------------
struct DuviHost {   // host copy of the SoA encoding (export / parity)
    std::vector<uint32_t> row_to_col, row_to_dist, col_idx, vidx;
    std::vector<uint8_t> dist;
    std::vector<double> values;
    int vi_bits = 8;
};

// Lane-interleaved derived layout of a DuVi matrix for the "lanes" kernel.
// Rows are grouped `group` at a time when consecutive rows share their column
// structure (the dofs of one mesh node); one lane owns one group, 32 groups
// form a bundle, and each bundle stores its streams word-interleaved by lane so
// that every warp load is one coalesced 128-byte transaction:
//   dist word w of lane t     at dist[d_base + w*32 + t]      (leader row, 4 entries per word)
//   value-index chunk (w, d)  at vi[v_base + (w*group + d)*32 + t]  (row d of the group, 4 entries)
//   block start b of lane t   at cols[c_base + b*32 + t]      (leader row)
// The canonical SoA stays on the device (export, Gauss-Seidel, SpMM).
// Set of at most 256 int64 keys (open addressing); find returns the insertion rank.
struct OffsetSet {
    static constexpr int kSlots = 2048;
    std::vector<int64_t> slot_key = std::vector<int64_t>(kSlots, INT64_MIN);
    std::vector<int16_t> slot_id = std::vector<int16_t>(kSlots, -1);
    std::vector<int64_t> keys;
    static int h(int64_t k) { return (int)(((uint64_t)k * 0x9E3779B97F4A7C15ull) >> 53); }
    bool insert(int64_t k) {   // false when a 257th key arrives
        for (int i = h(k);; i = (i + 1) & (kSlots - 1)) {
            if (slot_key[i] == k) return true;
            if (slot_key[i] == INT64_MIN) {
                if (keys.size() == 256) return false;
                slot_key[i] = k;
                slot_id[i] = (int16_t)keys.size();
                keys.push_back(k);
                return true;
            }
        }
    }
    int find(int64_t k) const {
        for (int i = h(k);; i = (i + 1) & (kSlots - 1)) {
            if (slot_key[i] == k) return slot_id[i];
            if (slot_key[i] == INT64_MIN) return -1;
        }
    }
};

struct DuviLanesHost {
    int group = 1;
    int scaled = 0;                // 1: value-index bytes hold index * value size (byte offsets into the table)
    int shift = 0;                 // 1: row d of a group reads columns of the leader row + d
    int tuples = 0;                // 1: one 8-bit tuple index per node-entry (tuple_vi: g value indices per tuple)
    std::vector<uint32_t> tuple_vi;
    std::vector<int16_t> tuple_id; // build-time map from packed value indices to tuple numbers
    int stencil = 0;               // 1: entry bytes index `offsets` (column - first row of the group); no column list
    std::vector<int32_t> offsets;
    OffsetSet offset_set;
    int64_t ngroups = 0, nbundles = 0;
    std::vector<uint32_t> meta;    // per bundle: d_base, v_base, c_base, words, blocks
    std::vector<uint32_t> dist;    // leader entry bytes, 4 per word: 255 at a block start, else gap - 1
    std::vector<uint8_t> vi;       // chunks of 4 value indices (4 * vi_bits / 8 bytes each)
    std::vector<uint32_t> cols;    // leader block column starts
    std::vector<uint32_t> nent;    // entries per leader row
};

struct dv_matrix {
    dv_context *ctx = nullptr;
    int32_t n_rows = 0, n_cols = 0;
    int64_t nnz = 0;
    int format = DV_FORMAT_CSR;
    int precision = DV_F64;
    // CSR
    DevMem rowptr, col, val;
    int csr_tpr = 16;          // threads per row (autotuned)
    // DuVi SoA
    int vi_bits = 8;
    int64_t nblocks = 0, nuniq = 0;
    DevMem row_to_col, row_to_dist, col_idx, dist, vidx, values;
    DevMem bundles;            // int32 row starts of row bundles (+ sentinel)
    int32_t nbundles = 0;
    int duvi_batch = 4;        // entries per gather batch in the decode loop (9 when most blocks hold 9)
    int duvi_variant = 0;      // 0: shared-memory staged rows, 1: lane-interleaved groups, 2: node patterns,
                               // 3: grid stencil (autotuned)
    int lanes_group = 1;
    int lanes_scaled = 0;
    int lanes_shift = 0;
    int lanes_tuples = 0;      // node-tuple mode: lanes_tup holds 4 values (padded) per tuple
    DevMem lanes_tup;
    int32_t lanes_ntup = 0;
    int pat_ok = 0;            // node-pattern layout available (duvi_variant 2)
    DevMem pat_id, pat_start, pat_rec;   // u16 per group, u32 per pattern, records {off, values} per entry
    DevMem pat_base;                     // u32 first column per group (based patterns)
    int pat_based = 0, pat_shift = 0;
    int32_t pat_count = 0, pat_entries = 0, pat_maxlen = 0;
    int grid_ok = 0;           // grid-stencil layout in use (duvi_variant 3), see DuviGridHost
    int32_t grid_lx = 0, grid_ly = 0, grid_lz = 0;
    int grid_hot = -1, grid_all_hot = 0;
    std::vector<double> grid_coef;       // 81 x 3 values of the hot pattern (entry k, row d at 3 * k + d)
    int grid_hex = 0;                    // 1: grid_coef has the hex stencil structure (dvk::hex_class)
    double grid_cls[10] = {};            // its class values
    DevMem grid_bnode;                   // u32 boundary groups
    int64_t grid_nb = 0;
    int32_t hex_ne[3] = {0, 0, 0};       // DV_FORMAT_HEX: elements per axis (of the first mesh)
    DevMem hex_factor;                   // per-element factor scale * E_e, matrix precision, meshes in order
    DevMem hex_meshes;                   // dvk::HexMesh per mesh (tiles, first row, first factor)
    int32_t hex_nmesh = 0, hex_ntile = 0;
    int32_t tri_ne[3] = {0, 0, 0};       // DV_FORMAT_TRILINEAR: fine element counts (even)
    int tri_restrict = 0;                // 1: restriction P^T, 0: prolongation P
    double hex_cls[14] = {};             // value classes of Ke (dvk::ke_class)
    int lanes_ok = 0;          // lane layout built (host-encoded matrices)
    int lanes_stencil = 0;     // stencil mode: lanes_off holds the column offsets (int32)
    DevMem lanes_off;
    int32_t lanes_noff = 0;
    int64_t lanes_bundles = 0, lanes_groups = 0;
    DevMem lanes_meta, lanes_dist, lanes_vi, lanes_cols, lanes_nent;
    int64_t lanes_bytes = 0;   // bytes one product reads from the lane layout
    // shared
    int row_group = 1;         // g consecutive rows share one column list (node dofs); 1 otherwise
    DevMem diag;               // FP64 diagonal (0 where absent)
    std::vector<double> host_diag;
    int zero_diag = 0;         // 1 when a diagonal entry is 0 or absent (square matrices)
    int64_t device_bytes = 0;
};

// Node-pattern layout (derived, read-only): every group of g rows whose entry list
// (column offsets from the group's first row, and the g value indices of each
// entry) repeats elsewhere shares one pattern; the matrix is then one pattern id
// per group plus a table of patterns.
struct DuviPatternHost {
    int ok = 0;
    int group = 1;
    int shift = 0;                   // 1: row d of a group reads columns + d
    int based = 0;                   // 1: offsets are from the group's first column (stored in base)
    int64_t ngroups = 0;
    std::vector<uint16_t> id;        // pattern of each group
    std::vector<uint32_t> base;      // first column of each group (based only)
    std::vector<uint32_t> start;     // first entry of each pattern (+ end)
    std::vector<int32_t> off;        // column - first row of the group, per pattern entry
    std::vector<uint32_t> vi;        // g value indices per pattern entry
};
// Grid-stencil layout (derived from the node patterns, read-only).  A square operator
// with 3 rows per node group, groups numbered x-fastest on an lx x ly x lz box, whose most
// frequent pattern ("hot") couples a group with its 27 box neighbours (3 columns each, in
// column order).  Groups off the box faces with the hot pattern are computed by a stencil
// that streams the box plane by plane, with the hot pattern's values as kernel parameters;
// every other group (faces, and interior groups of other patterns) keeps its pattern
// records and is listed in `boundary`.
struct DuviGridHost {
    int ok = 0;
    int32_t lx = 0, ly = 0, lz = 0;
    int hot = -1;                    // pattern id of the stencil groups
    int all_hot = 0;                 // 1: every group off the faces has the hot pattern
    std::vector<uint32_t> vi;        // value indices of the hot pattern, entry k, row d at 3 * k + d
    std::vector<uint32_t> boundary;  // groups computed from their pattern records, ascending
};
void dv_build_duvi_grid(const DuviPatternHost &P, DuviGridHost &out);

// Builds the pattern layout for rows in groups of `group` (identical or, with shift,
// shifted columns) when at most max_patterns patterns of max_entries entries in all
// exist.  Square operators without shift take offsets from the group's first row;
// otherwise from the group's first column, which is stored per group.
void dv_build_duvi_patterns(const DuviHost &h, int32_t n_rows, int32_t n_cols, int group, int shift,
                            int max_patterns, int max_entries, DuviPatternHost &out);

// Row bundles for the staged DuVi kernel: at most kBundleRows rows and at most
// kBundleBytes entry bytes / kBundleBlocks blocks (a longer single row forms its own bundle).
constexpr int kBundleRows = 32;
constexpr int kBundleBytes = 3008;    // entries (+ up to 32 bytes of 16-byte alignment slack)
constexpr int kBundleBlocks = 480;    // block column starts (+ alignment slack)

// Host helpers (dv_host.cpp)
void dv_encode_duvi(const dv_csr_host &a, double tol, int force_bits, DuviHost &out);
void dv_make_bundles(const DuviHost &h, int32_t n_rows, int vi_bits, std::vector<int32_t> &bundles);
// Value numbering of the reference's DuVi constructors: every value, in order, looked up in
// (or added to) a .NET Dictionary<double,int> with the ToleranceComparer of tolerance tol
// (default double comparer for tol == 0); idx[i] receives the value's key, the keys are
// returned in insertion order.
std::vector<double> dv_number_values(const double *val, int64_t n, double tol, uint32_t *idx);
// The same numbering from the distinct bit patterns of the values, given in order of first
// occurrence: key_of[i] receives the key of distinct[i], keys the keys in insertion order.
// Equal to the sequential walk unless a value could match two keys of its hash code or a
// non-finite value meets a tolerance: then returns false (number every value instead).
bool dv_number_distinct(const double *distinct, int64_t nd, double tol, uint32_t *key_of, std::vector<double> &keys);
// Node-pattern layout from its pattern table (off, vi, start, group, shift, based) without the
// per-group ids: the hot pattern's grid geometry (see DuviGridHost), or false.
bool dv_grid_geometry(const DuviPatternHost &P, int hot, int64_t ngroups, int32_t &lx, int32_t &ly, int32_t &lz);
// Throws DV_ERR_ARG / DV_ERR_FORMAT unless a is a valid CSR matrix with strictly
// increasing columns in every row.
void dv_check_csr(const dv_csr_host &a);
void dv_build_duvi_lanes(const DuviHost &h, int32_t n_rows, int32_t n_cols, int value_bytes, DuviLanesHost &out);
void dv_extract_diag(const dv_csr_host &a, std::vector<double> &diag);
// CSR transpose (rows sorted by column of the input).
void dv_csr_transpose(const dv_csr_host &a, std::vector<int32_t> &rp, std::vector<int32_t> &ci, std::vector<double> &va);
// 3 or 2 when every run of that many consecutive rows has one column list, else 1.
int dv_csr_row_group(const dv_csr_host &a);
// Row-ratio bound max_i sum_j |a_ij| / max_j |a_ij| (GeometricMultigridSolver.cs:144-151).
double dv_row_ratio_bound(const dv_csr_host &a);
// Dense inverse of an SPD matrix via LDL^T (no pivoting); returns false on a tiny pivot.
bool dv_dense_inverse(int32_t n, std::vector<double> &a, double pivot_tol);
// 24 x 24 unit-cube hexahedron stiffness (row-major, local nodes in VTK hexa order, 3 dofs per node).
void dv_hex_ke(double E, double nu, double *ke);
// Greedy coloring of node blocks (bs consecutive rows) for multicolor Gauss-Seidel.
int dv_block_coloring(const dv_csr_host &a, int bs, std::vector<int32_t> &color_of_block);
// Level sets of the forward Gauss-Seidel dependency graph (row i depends on j < i).
int dv_gs_level_sets(const dv_csr_host &a, std::vector<int32_t> &perm, std::vector<int32_t> &offsets);

// Pattern tables (records, starts, bases) of P with the given value table, and the grid-stencil
// fields of Gd (false when the stencil does not apply to this matrix); pattern ids and the
// boundary list are uploaded by the caller (dv_matrix.cu).
void dv_upload_patterns(dv_matrix *m, const DuviPatternHost &P, const std::vector<double> &values, cudaStream_t s);
bool dv_set_grid(dv_matrix *m, const DuviGridHost &Gd, const std::vector<double> &values);
// DuVi arrays, value table, diagonal and node-pattern / grid layouts of m (n_rows, n_cols, nnz,
// precision set) from a device CSR matrix, on the device (dv_encode_device.cu).
void dv_duvi_from_device_csr(dv_matrix *m, const int32_t *rp, const int32_t *col, const double *val, int force_bits,
                             double tol);

// Trilinear prolongation (restrict = 0) or restriction (restrict = 1) of the factor-2 coarsening of
// an even grid of ne_fine elements, applied without a matrix (dv_assemble.cu).
dv_matrix *dv_trilinear_build(dv_context *ctx, const int32_t *ne_fine, int restrict_, int32_t precision);
// Matrix-free hexahedral operator of nmesh meshes placed block-diagonally (dv_assemble.cu).
dv_matrix *dv_hex_operator_build(dv_context *ctx, int32_t nmesh, const int32_t *ne, const double *elem_E, double scale,
                                 double E, double nu, int32_t precision);
// Times the launch shapes of m's product and keeps the fastest (matrices of >= 100k rows).
void dv_autotune(dv_matrix *m);

// Matrix creation (dv_matrix.cu)
// encoded: a DuVi encoding of a made with the same vi_bits and tol, used instead of
// encoding again (one encoding serves matrices of both precisions).
dv_matrix *dv_matrix_build(dv_context *ctx, const dv_csr_host &a, int format, int precision,
                           int vi_bits, double tol, const DuviHost *encoded = nullptr);
