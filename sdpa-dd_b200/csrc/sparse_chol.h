// Sparse Schur complement on the device: the factor of the reordered B in
// 64 x 64 tiles (only the tiles the symbolic factor reaches are stored), the
// reference's sparse Cholesky (Lal::getCholesky(SparseMatrix&, int*),
// sdpa_linear.cpp:353-395) and sparse solve (Lal::solveSystems(Vector&,
// SparseMatrix&, Vector&), sdpa_linear.cpp:654-810) with the permutation
// around it (Newton::permuteVec / reverse_permuteVec, sdpa_newton.cpp:1258-1278).
#pragma once

#include "context.h"
#include "sparse_schur.h"

namespace sddd {

struct SparseDev {
    bool active = false;
    SparsePlan plan;     // decision, order and symbolic factor
    TileSchedule sched;  // tiles of the factor
    DBuf<dd_t> tiles;    // ntiles x 64 x 64, column-major within a tile
    DBuf<unsigned long long> mask; // ntiles x 64 structure words
    DBuf<int> tIJ;       // per tile: I, J
    DBuf<int> tile_of;   // nblk x nblk
    DBuf<int> diag;      // per block: its diagonal tile
    DBuf<int> col_ptr, col_tiles, row_ptr, row_tiles, upd;
    DBuf<int> order;     // new -> old
    DBuf<int> ent_b, ent_a; // per entry of the reference layout: column b, row a >= b
    DBuf<dd_t> xp;       // the permuted right-hand side
    DBuf<int> panel_done; // per panel: its CTAs that finished (sp_panel_kernel)
    // the factorisation's panel and update launches as one graph whose
    // edges are the tiles' data dependencies, built once per structure
    cudaGraphExec_t graph = nullptr;
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    ~SparseDev() { drop_graph(); }
};

// Plans the Schur form of the attached problem for c.schur_mode and, when
// it is sparse, uploads the factor's structure.
void sparse_setup(Context &c);
// The same for a given symbolic factor in its own numbering (identity
// order); throws on a structure that is not a symbolic factor.
void sparse_setup_structure(Context &c, const SparseStructure &s);
// Factor of the problem's B (gathered through the order) in the tiles.
void sparse_factor_B(Context &c);
// The entries vals (reference layout, device) into the tiles, and their
// factor in the tiles.
void sparse_load_values(Context &c, const dd_t *vals);
void sparse_factor_values(Context &c, const dd_t *vals);
// The tiles' entries in the reference layout (device).
void sparse_values(Context &c, dd_t *vals);
// x <- B^-1 x with the problem's order around the two triangular solves.
void sparse_solve(Context &c, dd_t *x);
// x <- (L L^T)^-1 x in the factor's own numbering.
void sparse_solve_raw(Context &c, dd_t *x);
// dd multiply-subtracts of one factorisation and of one pair of solves
double sparse_chol_terms(const Context &c);

} // namespace sddd
