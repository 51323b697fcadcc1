/* CPU restatement of the SDPA-DD dd Newton hot path (test infrastructure).
 *
 * This is the checker the GPU kernels are compared against: plain C,
 * single-threaded, written from the reference's algorithm with every
 * reduction in the reference's order, so that given the same inputs it
 * reproduces the reference's dd results bit for bit.  It is itself pinned
 * against the reference build (oracle/_ref) by the CPU test suite.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may use
 * it; the product never does.
 *
 * dd values are struct { double hi, lo; }, matrices column-major with
 * leading dimension = rows unless stated otherwise.
 */
#ifndef SDDD_ORACLE_H
#define SDDD_ORACLE_H
#include <stdint.h>

typedef struct {
    double hi, lo;
} odd;

/* dd arithmetic in the QD 2.3.23 default shapes (dd_inline.h). */
odd o_add(odd a, odd b);    /* operator+ (sloppy) */
odd o_acc(odd x, odd a);    /* operator+= */
odd o_sub(odd a, odd b);    /* operator- / -= */
odd o_mul(odd a, odd b);    /* operator* */
odd o_muleq(odd x, odd a);  /* operator*= */
odd o_div(odd a, odd b);    /* sloppy_div */
odd o_sqrt(odd a);          /* dd_real.cpp sqrt */
odd o_mul_d(odd a, double b);
odd o_add_d(odd a, double b);
odd o_sub_d(odd a, double b);
odd o_d_sub(double a, odd b);
odd o_div_d(odd a, double b);
odd o_d_div(double a, odd b);
odd o_sqr(odd a);
odd o_npwr(odd a, int n);
int o_lt(odd a, odd b);

/* Apply dd operation `op` elementwise (same numbering as ref_dd_op). */
void o_dd_op(int op, long n, const odd *a, const odd *b, odd *out);

/* Decimal string -> dd exactly as QD's dd_real::read (dd_real.cpp:1198).
 * Returns 0 on success, -1 on a malformed string. */
int o_dd_read(const char *s, odd *out);

/* ---------------- dense kernels in the reference's accumulation order --- */
/* C = op(A) * op(B) with alpha = 1, beta = 0 (Rgemm_{NN,TN,NT}_omp). */
void o_gemm(char ta, char tb, long m, long n, long k, const odd *A, long lda, const odd *B, long ldb, odd *C, long ldc);
/* Lower Cholesky in place (Rpotrf "Lower", any blocking).  Returns info. */
long o_potrf(long n, odd *A, long lda);
/* Solve with a lower factor: trans 'N' forward, 'T' backward (Rtrsv). */
void o_trsv(char trans, long n, const odd *L, long lda, odd *x);
/* X = inv(L) by Rtrsm("Left","Lower","N","N") on the identity. */
void o_inv_lower(long n, const odd *L, long lda, odd *X, long ldx);
/* B := L^T * B in place, L lower, non-unit (Rtrmm "L","L","T","N"). */
void o_trmm_lt(long n, const odd *L, long lda, odd *B, long ldb);
/* x := L^T x and x := L x for lower L (Rtrmv, unit stride). */
void o_trmv(char trans, long n, const odd *L, long lda, odd *x);
/* y = A x (Rgemv "N", alpha 1, beta 0). */
void o_gemv(long m, long n, const odd *A, long lda, const odd *x, odd *y);
/* Sequential dot product (Rdot with one thread). */
odd o_dot(long n, const odd *x, long incx, const odd *y, long incy);
/* (A + A^T)/2 in place (Lal::getSymmetrize). */
void o_symmetrize(long n, odd *A);

/* ---------------- Schur complement (Newton::compute_bMat_dense_SDP) ------ */
/* One SDP block: constraint matrices A_k (k = 0..nc-1 in the block's
 * constraint order) given either as COO upper-triangle entries in input
 * order (dense == 0) or as full n x n column-major (dense == 1). */
typedef struct {
    int con;           /* constraint index i in 0..m-1 */
    int dense;         /* 1 if stored dense (changeToDense happened) */
    int nnz;           /* stored COO entries (sparse) */
    int effect;        /* NonZeroEffect */
    int formula;       /* 0 F1, 1 F2, 2 F3 */
    const int *row, *col;
    const odd *val;    /* nnz values (sparse) or n*n (dense) */
} o_amat;

/* B += contribution of one block (B is m x m, column-major, ld m). */
void o_schur_block(long m, long n, int nc, const o_amat *A, const odd *X, const odd *invZ, odd *B);
/* A • D for one block (Lal::getInnerProduct(SparseMatrix, DenseMatrix)). */
odd o_inner_sparse_dense(long n, const o_amat *a, const odd *D);
/* Formula choice for one block (Newton::computeFormula_SDP). */
void o_formula(long n, int nc, const int *con, const int *dense, const int *effect, double kappa, int *formula_out);

/* ---------------- step-length eigenvalue (Lal::getMinEigen) ------------- */
/* Lanczos on L X L^T with the reference's start vector, checkpoints and
 * stopping rule; the tridiagonal eigenproblems are solved by bisection
 * plus inverse iteration instead of QR, which agrees to dd rounding. */
odd o_lanczos_min_eig(long n, const odd *L, const odd *X);

#endif
