// Device pieces of one interior-point iteration, each matching one routine
// of the reference (see newton.cu for the file:line of each).
#pragma once
#include "context.h"

namespace sddd {

// Solutions::initialize (sdpa_dataset.cpp:35-60): X = Z = lambda I, y = 0,
// L_X^-1 = L_Z^-1 = I / sqrt(lambda), Z^-1 = I / lambda.
void init_point(Context &c, dd_t lambda);
// Solutions::computeInverse (sdpa_dataset.cpp:96-118); false when a
// Cholesky factorisation of X or Z fails.  The _async form enqueues the
// same work and leaves the two failure words in c.info.
bool compute_inverse(Context &c);
void compute_inverse_async(Context &c);

// Several reductions' results side by side in c.scal, read back with one
// copy (one host round trip): each call enqueues its kernels and returns a
// group; after fetch(), sum(g) is the group's slots summed in order from
// zero with "+=" (the reference's per-block sums) and value(g) a one-slot
// group's value as it is.
struct ScalarBatch {
    Context &c;
    int used = 0;
    std::vector<std::pair<int, int>> groups; // (first slot, count)
    std::vector<dd_t> host;
    explicit ScalarBatch(Context &cc) : c(cc) {}
    int group(int count);
    int inner_space(const Space &a, const Space &b);
    int inner_C(const Space &x);
    int inner_b(const dd_t *v);
    int lambda_trace(const Space &s, double lambda);
    int maxabs_of(const dd_t *x, long n, int scratch);
    void residuals(int &gPrimal, int &gDual);
    // the failure words of compute_inverse_async (two ints in one slot)
    int inverse_info();
    void fetch();
    dd_t sum(int g) const;
    dd_t value(int g) const;
    bool inverse_ok(int g) const;
};
// Newton::compute_rMat + Newton::Make_gVec (sdpa_newton.cpp:821-893).
// dual_infeasible: phase is pFEAS or noINFO.
void make_rhs(Context &c, bool corrector, dd_t beta_mu, bool dual_infeasible);
// Newton::Make_bMat (schur.cu).
void schur_build(Context &c);
// Lal::choleskyFactorWithAdjust on B; returns LAPACK's info.
int schur_factor(Context &c);
// Dy = B^-1 g from the factor (Lal::solveSystems, sdpa_linear.cpp:639-651).
void solve_dy(Context &c);
// x = B^-1 x from the factor of B in place: the reference's two Rtrsv
// (bit for bit) after a plain factorisation, blocked solves with the
// inverted diagonal blocks after a split one.
void solve_B(Context &c, dd_t *x);
// Newton::compute_DzMat + compute_DxMat (sdpa_newton.cpp:1318-1343).
void make_dz_dx(Context &c, bool dual_infeasible);
// Inner products of the reference's Lal::let(ret, '=', a, '.', b).
dd_t inner_space(Context &c, const Space &a, const Space &b);
dd_t inner_C(Context &c, const Space &x);
dd_t inner_b(Context &c, const dd_t *v);
// Solutions::update's three axpys (sdpa_dataset.cpp:120-131).
void update_point(Context &c, dd_t alphaP, dd_t alphaD);
// Residuals::compute (sdpa_dataset.cpp:625-645); returns the two max norms.
void residuals(Context &c, dd_t &normPrimal, dd_t &normDual);
// sum_l sum_i lambda * M_l(i,i) (SolveInfo::update, sdpa_parts.cpp:684-690)
dd_t lambda_trace(Context &c, const Space &s, double lambda);
// Jal::getMinEigen(L, D) over the SDP blocks (sdpa_jordan.cpp:55-88).
dd_t min_eig(Context &c, const Space &L, const Space &D);
// The same for two spaces at once (their Lanczos side by side).
void min_eig_pair(Context &c, const Space &L1, const Space &D1, const Space &L2, const Space &D2, dd_t &out1, dd_t &out2);

// Building blocks shared with the adjoint (adjoint.cu):
// out_k = -(A_k . M) + addv_k (InputData::multi_InnerProductToA, then the
// callers' "v = -v + w").
void constraint_inner(Context &c, const Space &M, const dd_t *addv, dd_t *out);
// out = -sum_k y_k A_k (+ D) (mode 0) or C - Z - sum_k y_k A_k (mode 1).
void sum_yA(Context &c, const dd_t *y, Space &out, int mode, const Space *D, const Space *Z);
// out = A B C per block (Jal::ns_jordan_triple_product); uses W2.
void triple(Context &c, const Space &A, const Space &B, const Space &C, Space &out);

} // namespace sddd
