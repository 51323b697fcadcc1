// Sparse Schur complement: which form B takes, the ordering of its rows,
// its symbolic factor, and the 64 x 64 tile schedule the device factor and
// solves run on.
//
// The reference decides in Chordal::ordering_bMat (sdpa_chordal.cpp:348-438)
// and lays the sparse B out in Newton::initialize_sparse_bMat
// (sdpa_newton.cpp:225-340): the rows of B are renumbered by a fill-reducing
// ordering (SPOOLES minimum degree there), and row b of the factor keeps the
// entries (b, a), a in {b} + struct(b), ascending in the new numbering
// ("diagonalIndex" / "column_index").  The SPOOLES library is not part of
// the reference's sources; the ordering here is an exact minimum-degree
// ordering with a fixed tie rule (smallest original index), so the symbolic
// factor is the exact elimination structure of that ordering.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "problem.h"

namespace sddd {

constexpr int SP_T = 64; // tile order of the device factor and solves

// Schur form selection: the reference's thresholds (sdpa_chordal.cpp:42-45),
// always dense, or the reference's "SPARSE computation for debugging"
// thresholds (sdpa_chordal.cpp:53-58: every problem sparse).
enum SchurMode { SCHUR_AUTO = 0, SCHUR_DENSE = 1, SCHUR_SPARSE = 2 };

// Row-wise upper (equivalently column-wise lower) storage of the factor in
// the new numbering: row b holds col[rowptr[b]] = b, then struct(b) ascending.
struct SparseStructure {
    int m = 0;
    std::vector<int> rowptr; // m + 1
    std::vector<int> col;
    long nnz() const { return rowptr.empty() ? 0 : rowptr[m]; }
};

struct SparsePlan {
    bool sparse = false;
    // why the dense form was kept (empty when sparse)
    const char *dense_reason = "";
    long aggregate = 0; // entries of the aggregate pattern, diagonal included
    long extended = 0;  // 2 nnz(L) - m for the ordering (Chordal::countNonZero)
    std::vector<int> order; // new -> old
    SparseStructure s;
};

// The decision and, when sparse, the ordering and symbolic factor.
SparsePlan plan_schur(const Problem &p, int mode);

// Minimum-degree ordering of the graph adj (no self entries): at every step
// the live vertex of least current degree, ties to the smallest original
// index, is eliminated and its live neighbours made a clique.  Returns the
// order (new -> old); structs[v] receives v's live neighbours at its
// elimination (original numbering).
std::vector<int> min_degree_order(int m, const std::vector<std::vector<int>> &adj, std::vector<std::vector<int>> *structs);

// Checks that s is a valid symbolic factor (rows start with their diagonal,
// ascending, closed under elimination); returns an empty string or the
// first violation.
std::string check_structure(const SparseStructure &s);

// Tiles of the lower triangle of the factor (tile (I, J): rows I*64..,
// columns J*64..).
struct TileSchedule {
    int m = 0, nblk = 0, ntiles = 0;
    std::vector<int> tile_of;    // I + nblk * J for I >= J; -1 when the tile has no entry
    std::vector<int> tI, tJ;     // per tile
    std::vector<uint64_t> mask;  // ntiles * 64: word j, bit i = (64I+i, 64J+j) in the structure
    std::vector<int> col_ptr;    // nblk + 1: off-diagonal tiles (I, J), I > J ascending, of column block J
    std::vector<int> col_tiles;
    std::vector<int> row_ptr;    // nblk + 1: off-diagonal tiles (I, J), J < I ascending, of row block I
    std::vector<int> row_tiles;
    // trailing update of panel J: targets (I, K), K > J, I >= K, that some
    // column of J reaches in both I and K; three ints per target: target
    // tile, source tile (I, J), source tile (K, J)
    std::vector<int> upd_ptr; // nblk + 1
    std::vector<int> upd;
    long update_terms = 0;  // sum over panels of targets x 64 x 64 x 64 (upper bound of masked terms)
    long exact_terms = 0;   // dd multiply-subtracts of the factor (Lal::getCholesky's inner updates)
};

TileSchedule make_tile_schedule(const SparseStructure &s);

} // namespace sddd
