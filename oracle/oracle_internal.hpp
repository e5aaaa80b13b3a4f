// Internal types of the CPU oracle (test infrastructure only).
#pragma once
#include "oracle.h"

#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

struct or_csr {
    int32_t n_rows = 0, n_cols = 0;
    std::vector<int32_t> rowptr, col;
    std::vector<double> val;
};

// Dictionary-of-keys row builder that keeps .NET Dictionary insertion order
// (DokRowMajor.cs rows are Dictionary<int,double>; enumeration order is the
// order in which keys were first added, as no key is ever removed).
struct DokRow {
    std::vector<std::pair<int32_t, double>> entries;
    std::unordered_map<int32_t, int32_t> pos;
    // rows[r][c] = value (set), DokRowMajor indexer.
    void set(int32_t c, double v) {
        auto it = pos.find(c);
        if (it == pos.end()) { pos.emplace(c, (int32_t)entries.size()); entries.emplace_back(c, v); }
        else entries[it->second].second = v;
    }
    // rows[r][c] = sub + old (old = 0.0 when absent), DokRowMajor.cs:199-205.
    void add(int32_t c, double v) {
        auto it = pos.find(c);
        if (it == pos.end()) { pos.emplace(c, (int32_t)entries.size()); entries.emplace_back(c, v + 0.0); }
        else { double &o = entries[it->second].second; o = v + o; }
    }
    bool get(int32_t c, double &v) const {
        auto it = pos.find(c);
        if (it == pos.end()) return false;
        v = entries[it->second].second;
        return true;
    }
};

struct Dok {
    int32_t n_rows = 0, n_cols = 0;
    std::vector<DokRow> rows;
    Dok(int32_t r, int32_t c) : n_rows(r), n_cols(c), rows(r) {}
    // GetSubmatrix (DokRowMajor.cs:471-501): rows in rowsToKeep order, each row
    // in source insertion order filtered by the column map.
    Dok submatrix(const std::vector<int32_t> &keep_rows, const std::vector<int32_t> &keep_cols) const;
    // BuildCsrArrays(sorted) (DokRowMajor.cs:286-324).
    or_csr *to_csr(bool sorted) const;
};

// .NET Dictionary<double,int> with the DuVi ToleranceComparer
// (DuViCompressedSparseMatrix.cs:168-174) or the default double comparer.
struct DoubleIndexMap {
    double tol;
    std::unordered_map<int32_t, std::vector<int32_t>> classes;  // hash code -> entry ids (insertion order)
    std::vector<double> keys;
    explicit DoubleIndexMap(double t) : tol(t) {}
    int32_t hash(double x) const;
    bool equal(double stored, double key) const;
    int32_t find(double v) const;       // -1 when absent (newest matching entry first, as the bucket chain)
    int32_t insert(double v);           // returns the new index (== Count before insertion)
    int32_t count() const { return (int32_t)keys.size(); }
};

int32_t dotnet_double_hash(double x);
extern int g_or_threads;

// Element stiffness (FemCantilever3D.cs:225-313, FemCantilever2D.cs:29-49),
// row-major, (nodes*dofs)^2 entries.
std::vector<double> element_stiffness(int dim, double E, double nu);

// Structured mesh helpers (x-fastest numbering, VTK corner order).
struct Mesh {
    int dim = 3;
    int32_t ne[3] = {1, 1, 1};
    int32_t nn[3] = {1, 1, 1};
    double len[3] = {1, 1, 1};
    int32_t nodes_total() const { return nn[0] * nn[1] * nn[2]; }
    int32_t elements_total() const { return ne[0] * ne[1] * ne[2]; }
    int32_t node_id(int32_t i, int32_t j, int32_t k) const { return i + j * nn[0] + k * nn[0] * nn[1]; }
    void element_nodes(int32_t e, int32_t *out) const;   // 4 or 8 node ids
    int nodes_per_element() const { return dim == 3 ? 8 : 4; }
};
