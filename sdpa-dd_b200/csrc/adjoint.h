// Adjoint of a finished solve (adjoint.cu): the transpose of the solution's
// linearisation at the final iterate, through the Cholesky of the Schur
// matrix B at that iterate.
#pragma once
#include "context.h"

namespace sddd {

// Weights on the outputs (host arrays, each may be null): g_x on the file's
// x (m), g_Y on its Y (a block space: the internal X), g_X on its X (the
// internal Z), g_obj on the optimal value c.x.  Leaves u and R in the
// context; returns 0, or the failing column of the Cholesky of B.
// Overwrites B, Dx, Dz and the work spaces.
int adjoint(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj);
// The same at the optimum: the adjoint at exactly central points built
// from the iterate's eigendecomposition, extrapolated to mu -> 0
// (adjoint.cu); the solution gradients are those of the optimal solution.
int adjoint_limit(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj);
// The adjoint for mixed weights (linear in them): the optimal value's part at
// the iterate (adjoint), the solution's part at the limit (adjoint_limit).
int adjoint_combined(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj);
// Gradients from the stored adjoint (device outputs).
void adjoint_grad_c(Context &c, dd_t g_obj, dd_t *out_dev);   // m
void adjoint_grad_F0(Context &c, dd_t *out_dev);              // block space
void adjoint_grad_F(Context &c, int k, dd_t *out_dev);        // block space, constraint k (0-based)

} // namespace sddd
