/* CPU restatement of the SDPA-DD dd hot path; see oracle.h.
 * Test infrastructure only.  Compiled with -ffp-contract=off so every
 * double operation rounds as written. */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ primitives */
static double two_sum(double a, double b, double *e) {
    double s = a + b, v = s - a;
    *e = (a - (s - v)) + (b - v);
    return s;
}
static double two_diff(double a, double b, double *e) {
    double s = a - b, v = s - a;
    *e = (a - (s - v)) - (b + v);
    return s;
}
static double quick(double a, double b, double *e) {
    double s = a + b;
    *e = b - (s - a);
    return s;
}
/* Dekker's exact product (Veltkamp split), as QD builds without FMA. */
static void split(double a, double *hi, double *lo) {
    const double SPLITTER = 134217729.0; /* 2^27 + 1 */
    const double THRESH = 6.69692879491417e+299;
    double t;
    if (a > THRESH || a < -THRESH) {
        a *= 3.7252902984619140625e-09;
        t = SPLITTER * a;
        *hi = t - (t - a);
        *lo = a - *hi;
        *hi *= 268435456.0;
        *lo *= 268435456.0;
    } else {
        t = SPLITTER * a;
        *hi = t - (t - a);
        *lo = a - *hi;
    }
}
static double two_prod(double a, double b, double *e) {
    double p = a * b, ah, al, bh, bl;
    split(a, &ah, &al);
    split(b, &bh, &bl);
    *e = ((ah * bh - p) + ah * bl + al * bh) + al * bl;
    return p;
}
static odd mk(double h, double l) {
    odd r;
    r.hi = h;
    r.lo = l;
    return r;
}
static const odd ZERO = {0.0, 0.0};
static const odd ONE = {1.0, 0.0};

odd o_add(odd a, odd b) {
    double e, s = two_sum(a.hi, b.hi, &e);
    e += (a.lo + b.lo);
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_acc(odd x, odd a) {
    double e, s = two_sum(x.hi, a.hi, &e);
    e += x.lo;
    e += a.lo;
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_sub(odd a, odd b) {
    double e, s = two_diff(a.hi, b.hi, &e);
    e += a.lo;
    e -= b.lo;
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_mul(odd a, odd b) {
    double e, p = two_prod(a.hi, b.hi, &e);
    e += (a.hi * b.lo + a.lo * b.hi);
    p = quick(p, e, &e);
    return mk(p, e);
}
odd o_muleq(odd x, odd a) {
    double e, p = two_prod(x.hi, a.hi, &e);
    e += a.lo * x.hi;
    e += a.hi * x.lo;
    p = quick(p, e, &e);
    return mk(p, e);
}
odd o_mul_d(odd a, double b) {
    double e, p = two_prod(a.hi, b, &e);
    e += a.lo * b;
    p = quick(p, e, &e);
    return mk(p, e);
}
odd o_add_d(odd a, double b) {
    double e, s = two_sum(a.hi, b, &e);
    e += a.lo;
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_sub_d(odd a, double b) {
    double e, s = two_diff(a.hi, b, &e);
    e += a.lo;
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_d_sub(double a, odd b) {
    double e, s = two_diff(a, b.hi, &e);
    e -= b.lo;
    s = quick(s, e, &e);
    return mk(s, e);
}
odd o_div(odd a, odd b) {
    double q1 = a.hi / b.hi;
    odd r = o_mul_d(b, q1);
    double s2, s1 = two_diff(a.hi, r.hi, &s2);
    s2 -= r.lo;
    s2 += a.lo;
    double q2 = (s1 + s2) / b.hi, e;
    double q = quick(q1, q2, &e);
    return mk(q, e);
}
odd o_div_d(odd a, double b) {
    double q1 = a.hi / b, p2, p1 = two_prod(q1, b, &p2), e;
    double s = two_diff(a.hi, p1, &e);
    e += a.lo;
    e -= p2;
    double q2 = (s + e) / b, r2;
    double r1 = quick(q1, q2, &r2);
    return mk(r1, r2);
}
odd o_d_div(double a, odd b) { return o_div(mk(a, 0.0), b); }
odd o_sqr(odd a) {
    double p2, p1 = two_prod(a.hi, a.hi, &p2);
    p2 += 2.0 * a.hi * a.lo;
    p2 += a.lo * a.lo;
    double s2, s1 = quick(p1, p2, &s2);
    return mk(s1, s2);
}
odd o_sqrt(odd a) {
    if (a.hi == 0.0) return ZERO;
    if (a.hi < 0.0) return mk(NAN, NAN);
    double x = 1.0 / sqrt(a.hi);
    double ax = a.hi * x;
    double e2, p = two_prod(ax, ax, &e2);
    odd d = o_sub(a, mk(p, e2));
    double e, s = two_sum(ax, d.hi * (x * 0.5), &e);
    return mk(s, e);
}
odd o_npwr(odd a, int n) {
    if (n == 0) return ONE;
    odd r = a, s = ONE;
    int N = n < 0 ? -n : n;
    if (N > 1) {
        while (N > 0) {
            if (N % 2 == 1) s = o_muleq(s, r);
            N /= 2;
            if (N > 0) r = o_sqr(r);
        }
    } else {
        s = r;
    }
    if (n < 0) return o_d_div(1.0, s);
    return s;
}
int o_lt(odd a, odd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
static int o_gt(odd a, odd b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }
static int o_le_d(odd a, double b) { return a.hi < b || (a.hi == b && a.lo <= 0.0); }
static int o_gt_d(odd a, double b) { return a.hi > b || (a.hi == b && a.lo > 0.0); }
static int o_is_zero(odd a) { return a.hi == 0.0 && a.lo == 0.0; }
static odd o_neg(odd a) { return mk(-a.hi, -a.lo); }
static odd o_abs(odd a) { return a.hi < 0.0 ? o_neg(a) : a; }
static odd o_from(double d) { return mk(d, 0.0); }
/* double-vs-dd comparisons of QD (dd_inline.h operator< / operator>) */
static int d_lt_dd(double a, odd b) { return a < b.hi || (a == b.hi && b.lo > 0.0); }
static int d_gt_dd(double a, odd b) { return a > b.hi || (a == b.hi && b.lo < 0.0); }

void o_dd_op(int op, long n, const odd *a, const odd *b, odd *out) {
    for (long i = 0; i < n; ++i) {
        odd x = a[i], y = b[i], r;
        switch (op) {
        case 0: r = o_add(x, y); break;
        case 1: r = o_acc(x, y); break;
        case 2: r = o_sub(x, y); break;
        case 3: r = o_sub(x, y); break;
        case 4: r = o_mul(x, y); break;
        case 5: r = o_muleq(x, y); break;
        case 6: r = o_div(x, y); break;
        case 7: r = o_sqrt(x); break;
        case 8: r = o_mul_d(x, y.hi); break;
        case 9: r = o_add_d(x, y.hi); break;
        case 10: r = o_sub_d(x, y.hi); break;
        case 11: r = o_d_sub(x.hi, y); break;
        case 12: r = o_div_d(x, y.hi); break;
        case 13: r = o_d_div(x.hi, y); break;
        case 14: r = o_neg(x); break;
        case 15: r = o_abs(x); break;
        case 16: r = o_sqr(x); break;
        case 17: {
            double e, s = two_sum(x.hi, y.hi, &e);
            r = mk(s, e);
        } break;
        default: r = ZERO; break;
        }
        out[i] = r;
    }
}

/* QD dd_real::read (dd_real.cpp:1198-1259): digits accumulated by
 * r *= 10; r += d, then one multiplication by 10^e computed by npwr. */
int o_dd_read(const char *s, odd *out) {
    const char *p = s;
    int sign = 0, point = -1, nd = 0, e = 0, done = 0;
    odd r = ZERO;
    while (*p == ' ') p++;
    while (!done && *p != '\0') {
        char ch = *p;
        if (ch >= '0' && ch <= '9') {
            r = o_mul_d(r, 10.0);
            r = o_add_d(r, (double)(ch - '0'));
            nd++;
        } else {
            switch (ch) {
            case '.':
                if (point >= 0) return -1;
                point = nd;
                break;
            case '-':
            case '+':
                if (sign != 0 || nd > 0) return -1;
                sign = (ch == '-') ? -1 : 1;
                break;
            case 'E':
            case 'e':
                if (sscanf(p + 1, "%d", &e) != 1) return -1;
                done = 1;
                break;
            default:
                return -1;
            }
        }
        p++;
    }
    if (point >= 0) e -= (nd - point);
    if (e != 0) r = o_muleq(r, o_npwr(o_from(10.0), e));
    *out = (sign == -1) ? o_neg(r) : r;
    return 0;
}

/* ------------------------------------------------------------- kernels */
#define AT(M, ld, i, j) (M)[(i) + (long)(ld) * (j)]

/* Rgemm_NN/TN/NT_omp (mplapack/Rgemm_*_omp.cpp) with alpha = 1, beta = 0:
 * every C(i,j) is a sequential sum over l of operator+= steps. */
void o_gemm(char ta, char tb, long m, long n, long k, const odd *A, long lda, const odd *B, long ldb, odd *C, long ldc) {
    for (long j = 0; j < n; ++j)
        for (long i = 0; i < m; ++i) AT(C, ldc, i, j) = ZERO;
    if (ta == 'N') {
        for (long j = 0; j < n; ++j)
            for (long l = 0; l < k; ++l) {
                odd temp = o_mul(ONE, tb == 'N' ? AT(B, ldb, l, j) : AT(B, ldb, j, l));
                for (long i = 0; i < m; ++i) AT(C, ldc, i, j) = o_acc(AT(C, ldc, i, j), o_mul(temp, AT(A, lda, i, l)));
            }
    } else { /* 'T', tb 'N' */
        for (long j = 0; j < n; ++j)
            for (long i = 0; i < m; ++i) {
                odd temp = ZERO;
                for (long l = 0; l < k; ++l) temp = o_acc(temp, o_mul(AT(A, lda, l, i), AT(B, ldb, l, j)));
                AT(C, ldc, i, j) = o_acc(AT(C, ldc, i, j), o_mul(ONE, temp));
            }
    }
}

/* Rpotrf("Lower") (mplapack/Rpotrf.cpp:124-142, Rpotrf2.cpp).  Whatever
 * the blocking, each entry receives the terms L(j,k) L(i,k), k ascending,
 * as "x = x - p" steps (Rsyrk/Rgemm add the negated product, which rounds
 * identically); the diagonal then takes sqrt and the column below is
 * multiplied by 1/L(j,j) (Rtrsm "Right","Lower","Transpose"). */
long o_potrf(long n, odd *A, long lda) {
    for (long j = 0; j < n; ++j) {
        odd d = AT(A, lda, j, j);
        for (long k = 0; k < j; ++k) d = o_sub(d, o_mul(AT(A, lda, j, k), AT(A, lda, j, k)));
        if (o_le_d(d, 0.0) || d.hi != d.hi || d.lo != d.lo) return j + 1;
        odd ljj = o_sqrt(d);
        AT(A, lda, j, j) = ljj;
        odd r = o_div(ONE, ljj);
        for (long i = j + 1; i < n; ++i) {
            odd v = AT(A, lda, i, j);
            for (long k = 0; k < j; ++k) v = o_sub(v, o_mul(AT(A, lda, j, k), AT(A, lda, i, k)));
            AT(A, lda, i, j) = o_mul(r, v);
        }
    }
    return 0;
}

/* Rtrsv lower, non-unit (mplapack/Rtrsv.cpp). */
void o_trsv(char trans, long n, const odd *L, long lda, odd *x) {
    if (trans == 'N') {
        for (long j = 0; j < n; ++j) {
            if (!o_is_zero(x[j])) {
                x[j] = o_div(x[j], AT(L, lda, j, j));
                odd t = x[j];
                for (long i = j + 1; i < n; ++i) x[i] = o_sub(x[i], o_mul(t, AT(L, lda, i, j)));
            }
        }
    } else {
        for (long j = n - 1; j >= 0; --j) {
            odd t = x[j];
            for (long i = n - 1; i >= j + 1; --i) t = o_sub(t, o_mul(AT(L, lda, i, j), x[i]));
            x[j] = o_div(t, AT(L, lda, j, j));
        }
    }
}

/* Lal::getInvLowTriangularMatrix (sdpa_linear.cpp:397-412):
 * Rtrsm("Left","Lower","N","N") applied to the identity. */
void o_inv_lower(long n, const odd *L, long lda, odd *X, long ldx) {
    for (long j = 0; j < n; ++j)
        for (long i = 0; i < n; ++i) AT(X, ldx, i, j) = (i == j) ? ONE : ZERO;
    for (long j = 0; j < n; ++j)
        for (long k = 0; k < n; ++k) {
            if (o_is_zero(AT(X, ldx, k, j))) continue;
            AT(X, ldx, k, j) = o_div(AT(X, ldx, k, j), AT(L, lda, k, k));
            for (long i = k + 1; i < n; ++i) AT(X, ldx, i, j) = o_sub(AT(X, ldx, i, j), o_mul(AT(X, ldx, k, j), AT(L, lda, i, k)));
        }
}

/* Rtrmm("Left","Lower","Transpose","NonUnit", alpha = 1). */
void o_trmm_lt(long n, const odd *L, long lda, odd *B, long ldb) {
    for (long j = 0; j < n; ++j)
        for (long i = 0; i < n; ++i) {
            odd t = o_mul(AT(B, ldb, i, j), AT(L, lda, i, i));
            for (long k = i + 1; k < n; ++k) t = o_acc(t, o_mul(AT(L, lda, k, i), AT(B, ldb, k, j)));
            AT(B, ldb, i, j) = o_mul(ONE, t);
        }
}

/* Rtrmv lower, non-unit, unit stride (mplapack/Rtrmv.cpp). */
void o_trmv(char trans, long n, const odd *L, long lda, odd *x) {
    if (trans == 'T') {
        for (long j = 0; j < n; ++j) {
            odd t = o_mul(x[j], AT(L, lda, j, j));
            for (long i = j + 1; i < n; ++i) t = o_acc(t, o_mul(AT(L, lda, i, j), x[i]));
            x[j] = t;
        }
    } else {
        for (long j = n - 1; j >= 0; --j) {
            if (!o_is_zero(x[j])) {
                odd t = x[j];
                for (long i = n - 1; i >= j + 1; --i) x[i] = o_acc(x[i], o_mul(t, AT(L, lda, i, j)));
                x[j] = o_mul(x[j], AT(L, lda, j, j));
            }
        }
    }
}

void o_gemv(long m, long n, const odd *A, long lda, const odd *x, odd *y) {
    for (long i = 0; i < m; ++i) y[i] = ZERO;
    for (long j = 0; j < n; ++j) {
        odd t = o_mul(ONE, x[j]);
        for (long i = 0; i < m; ++i) y[i] = o_acc(y[i], o_mul(t, AT(A, lda, i, j)));
    }
}

/* Rdot with one OpenMP thread (mplapack/Rdot_omp.cpp). */
odd o_dot(long n, const odd *x, long incx, const odd *y, long incy) {
    odd t = ZERO;
    for (long i = 0; i < n; ++i) t = o_acc(t, o_mul(x[i * incx], y[i * incy]));
    return o_acc(ZERO, t);
}

/* Lal::getSymmetrize (sdpa_linear.cpp:414-438). */
void o_symmetrize(long n, odd *A) {
    const odd half = {0.5, 0.0};
    for (long c = 0; c + 1 < n; ++c)
        for (long i = c + 1; i < n; ++i) {
            odd v = o_acc(AT(A, n, i, c), o_mul(ONE, AT(A, n, c, i)));
            v = o_mul(half, v);
            AT(A, n, i, c) = v;
            AT(A, n, c, i) = v;
        }
}

/* ------------------------------------------------------------- Schur */
/* Lal::getInnerProduct(SparseMatrix, DenseMatrix) (sdpa_linear.cpp:202-298):
 * the first nnz % 4 terms one by one, then groups of four summed with
 * operator+ before one operator+=. */
odd o_inner_sparse_dense(long n, const o_amat *a, const odd *D) {
    if (a->dense) return o_dot(n * n, a->val, 1, D, 1);
    odd ret = ZERO;
    int amari = a->nnz % 4, shou = a->nnz / 4;
#define TERM(idx)                                                                                            \
    ((a->row[idx] == a->col[idx]) ? o_mul(a->val[idx], AT(D, n, a->row[idx], a->col[idx]))                   \
                                  : o_mul(a->val[idx], o_add(AT(D, n, a->row[idx], a->col[idx]), AT(D, n, a->col[idx], a->row[idx]))))
    for (int idx = 0; idx < amari; ++idx) ret = o_acc(ret, TERM(idx));
    for (int c = 0, idx = amari; c < shou; ++c, idx += 4) {
        odd r1 = TERM(idx), r2 = TERM(idx + 1), r3 = TERM(idx + 2), r4 = TERM(idx + 3);
        ret = o_acc(ret, o_add(o_add(o_add(r1, r2), r3), r4));
    }
#undef TERM
    return ret;
}

/* Lal::multiply(DenseMatrix, SparseMatrix, DenseMatrix) with scalar NULL
 * (sdpa_linear.cpp:832-893): ret = A * Bm, sparse A as Raxpy row updates. */
static void o_sparse_times_dense(long n, const o_amat *a, const odd *Bm, odd *ret) {
    if (a->dense) {
        o_gemm('N', 'N', n, n, n, a->val, n, Bm, n, ret, n);
        return;
    }
    for (long t = 0; t < n * n; ++t) ret[t] = ZERO;
    for (int idx = 0; idx < a->nnz; ++idx) {
        int i = a->row[idx], j = a->col[idx];
        odd v = a->val[idx];
        if (o_is_zero(v)) continue; /* Raxpy returns when da == 0 */
        if (i != j) {
            for (long t = 0; t < n; ++t) AT(ret, n, i, t) = o_acc(AT(ret, n, i, t), o_mul(v, AT(Bm, n, j, t)));
            for (long t = 0; t < n; ++t) AT(ret, n, j, t) = o_acc(AT(ret, n, j, t), o_mul(v, AT(Bm, n, i, t)));
        } else {
            for (long t = 0; t < n; ++t) AT(ret, n, j, t) = o_acc(AT(ret, n, j, t), o_mul(v, AT(Bm, n, j, t)));
        }
    }
}

/* Newton::calF3 (sdpa_newton.cpp:937-977). */
static odd o_calF3(long n, const odd *X, const odd *invZ, const o_amat *Ai, const o_amat *Aj) {
    odd ret = ZERO;
    for (int i1 = 0; i1 < Aj->nnz; ++i1) {
        int al = Aj->row[i1], be = Aj->col[i1];
        odd v1 = Aj->val[i1], sum = ZERO;
        for (int i2 = 0; i2 < Ai->nnz; ++i2) {
            int ga = Ai->row[i2], de = Ai->col[i2];
            odd v2 = Ai->val[i2];
            sum = o_acc(sum, o_mul(o_mul(v2, AT(invZ, n, de, be)), AT(X, n, al, ga)));
            if (ga != de) sum = o_acc(sum, o_mul(o_mul(v2, AT(invZ, n, ga, be)), AT(X, n, al, de)));
        }
        ret = o_acc(ret, o_mul(v1, sum));
        if (al == be) continue;
        sum = ZERO;
        for (int i2 = 0; i2 < Ai->nnz; ++i2) {
            int ga = Ai->row[i2], de = Ai->col[i2];
            odd v2 = Ai->val[i2];
            sum = o_acc(sum, o_mul(o_mul(v2, AT(invZ, n, de, al)), AT(X, n, be, ga)));
            if (ga != de) sum = o_acc(sum, o_mul(o_mul(v2, AT(invZ, n, ga, al)), AT(X, n, be, de)));
        }
        ret = o_acc(ret, o_mul(v1, sum));
    }
    return ret;
}

/* Newton::compute_bMat_dense_SDP for one block (sdpa_newton.cpp:979-1068). */
void o_schur_block(long m, long n, int nc, const o_amat *A, const odd *X, const odd *invZ, odd *B) {
    odd *F = (odd *)malloc(sizeof(odd) * n * n), *G = (odd *)malloc(sizeof(odd) * n * n);
    for (int k1 = 0; k1 < nc; ++k1) {
        const o_amat *Ai = &A[k1];
        int i = Ai->con, inz = Ai->effect, hasG = 0;
        if (Ai->formula == 0) {
            o_sparse_times_dense(n, Ai, invZ, F);
            o_gemm('N', 'N', n, n, n, X, n, F, n, G, n);
        } else if (Ai->formula == 1) {
            o_sparse_times_dense(n, Ai, invZ, F);
        }
        for (int k2 = 0; k2 < nc; ++k2) {
            const o_amat *Aj = &A[k2];
            int j = Aj->con, jnz = Aj->effect;
            if (inz < jnz || (inz == jnz && i < j)) continue;
            odd value;
            if (Ai->formula == 0) {
                value = o_inner_sparse_dense(n, Aj, G);
            } else if (Ai->formula == 1) {
                if (Aj->dense) {
                    if (!hasG) {
                        o_gemm('N', 'N', n, n, n, X, n, F, n, G, n);
                        hasG = 1;
                    }
                    value = o_inner_sparse_dense(n, Aj, G);
                } else {
                    value = ZERO;
                    for (int idx = 0; idx < Aj->nnz; ++idx) {
                        int al = Aj->row[idx], be = Aj->col[idx];
                        odd v1 = Aj->val[idx];
                        value = o_acc(value, o_mul(v1, o_dot(n, X + al, n, F + n * be, 1)));
                        if (al != be) value = o_acc(value, o_mul(v1, o_dot(n, X + be, n, F + n * al, 1)));
                    }
                }
            } else {
                value = o_calF3(n, X, invZ, Ai, Aj);
            }
            if (i != j) {
                AT(B, m, i, j) = o_acc(AT(B, m, i, j), value);
                AT(B, m, j, i) = o_acc(AT(B, m, j, i), value);
            } else {
                AT(B, m, i, i) = o_acc(AT(B, m, i, i), value);
            }
        }
    }
    free(F);
    free(G);
}

/* Newton::computeFormula_SDP for one block (sdpa_newton.cpp:694-819),
 * including its dd cost arithmetic. */
void o_formula(long n, int nc, const int *con, const int *dense, const int *effect, double kappa, int *formula_out) {
    odd K = o_from(kappa), nn = o_from((double)n);
    for (int k1 = 0; k1 < nc; ++k1) {
        int inz_i = effect[k1], up_i = inz_i;
        for (int k2 = 0; k2 < nc; ++k2) {
            int jnz = effect[k2];
            if (jnz < inz_i) up_i += jnz;
            else if (jnz == inz_i && con[k2] < con[k1]) up_i += jnz;
        }
        odd inz = o_from((double)inz_i), up = o_from((double)up_i);
        odd f1 = o_add(o_add(o_mul(o_mul(K, nn), inz), o_mul(o_mul(nn, nn), nn)), o_mul(K, up));
        odd f2 = o_add(o_mul(o_mul(K, nn), inz), o_mul(o_mul(K, o_add_d(nn, 1.0)), up));
        odd f3 = o_div(o_mul(o_mul(K, o_add_d(o_mul(o_mul_d(K, 2.0), inz), 1.0)), up), K);
        int f;
        if (dense[k1]) f = o_lt(f1, f2) ? 0 : 1;
        else if (o_lt(f1, f2) && o_lt(f1, f3)) f = 0;
        else if (o_lt(f2, f3)) f = 1;
        else f = 2;
        formula_out[k1] = f;
    }
}

/* ---------------------------------------------------------- Lanczos */
/* Number of eigenvalues of the tridiagonal (d, e) below x (Sturm count
 * through the LDL^T pivots). */
static int sturm_count(int k, const odd *d, const odd *e2, odd x) {
    int c = 0;
    odd q = o_sub(d[0], x);
    if (q.hi < 0.0) c++;
    for (int i = 1; i < k; ++i) {
        if (o_is_zero(q)) q = mk(1e-300, 0.0);
        q = o_sub(o_sub(d[i], x), o_div(e2[i - 1], q));
        if (q.hi < 0.0) c++;
    }
    return c;
}

/* Smallest eigenvalue of the k x k symmetric tridiagonal (d, e) and the
 * last component of its unit eigenvector (bisection, then inverse
 * iteration with a partially pivoted tridiagonal solve). */
static void tri_min_eig(int k, const odd *d, const odd *e, odd *lam, odd *last) {
    odd *e2 = (odd *)malloc(sizeof(odd) * (k + 1));
    odd lo = d[0], hi = d[0];
    for (int i = 0; i < k; ++i) {
        odd r = ZERO;
        if (i > 0) r = o_add(r, o_abs(e[i - 1]));
        if (i + 1 < k) r = o_add(r, o_abs(e[i]));
        odd a = o_sub(d[i], r), b = o_add(d[i], r);
        if (o_lt(a, lo)) lo = a;
        if (o_gt(b, hi)) hi = b;
        if (i + 1 < k) e2[i] = o_mul(e[i], e[i]);
    }
    odd width = o_sub(hi, lo);
    lo = o_sub(lo, o_mul_d(width, 1e-10));
    hi = o_add(hi, o_mul_d(width, 1e-10));
    for (int it = 0; it < 400; ++it) {
        odd mid = o_mul_d(o_add(lo, hi), 0.5);
        if (!(o_lt(lo, mid) && o_lt(mid, hi))) break;
        if (sturm_count(k, d, e2, mid) >= 1) hi = mid;
        else lo = mid;
    }
    odd l = o_mul_d(o_add(lo, hi), 0.5);
    *lam = l;
    /* inverse iteration on (T - l I) */
    odd *v = (odd *)malloc(sizeof(odd) * k), *dd = (odd *)malloc(sizeof(odd) * k), *du = (odd *)malloc(sizeof(odd) * k),
        *du2 = (odd *)malloc(sizeof(odd) * k), *dl = (odd *)malloc(sizeof(odd) * k);
    int *piv = (int *)malloc(sizeof(int) * k);
    for (int i = 0; i < k; ++i) v[i] = ONE;
    odd tnorm = o_add(o_abs(lo), o_abs(hi));
    for (int it = 0; it < 3; ++it) {
        for (int i = 0; i < k; ++i) {
            dd[i] = o_sub(d[i], l);
            du[i] = (i + 1 < k) ? e[i] : ZERO;
            dl[i] = (i + 1 < k) ? e[i] : ZERO;
            du2[i] = ZERO;
        }
        for (int i = 0; i + 1 < k; ++i) {
            if (!o_lt(o_abs(dd[i]), o_abs(dl[i]))) {
                piv[i] = 0;
                if (o_is_zero(dd[i])) dd[i] = o_mul_d(tnorm, 1e-32);
                odd f = o_div(dl[i], dd[i]);
                dl[i] = f;
                dd[i + 1] = o_sub(dd[i + 1], o_mul(f, du[i]));
            } else {
                piv[i] = 1;
                odd f = o_div(dd[i], dl[i]);
                dd[i] = dl[i];
                dl[i] = f;
                odd t = du[i];
                du[i] = dd[i + 1];
                dd[i + 1] = o_sub(t, o_mul(f, dd[i + 1]));
                if (i + 2 < k) {
                    du2[i] = du[i + 1];
                    du[i + 1] = o_neg(o_mul(f, du[i + 1]));
                }
            }
        }
        if (o_is_zero(dd[k - 1])) dd[k - 1] = o_mul_d(tnorm, 1e-32);
        for (int i = 0; i + 1 < k; ++i) {
            if (piv[i]) {
                odd t = v[i];
                v[i] = v[i + 1];
                v[i + 1] = o_sub(t, o_mul(dl[i], v[i + 1]));
            } else {
                v[i + 1] = o_sub(v[i + 1], o_mul(dl[i], v[i]));
            }
        }
        for (int i = k - 1; i >= 0; --i) {
            odd t = v[i];
            if (i + 1 < k) t = o_sub(t, o_mul(du[i], v[i + 1]));
            if (i + 2 < k) t = o_sub(t, o_mul(du2[i], v[i + 2]));
            v[i] = o_div(t, dd[i]);
        }
        odd nrm = ZERO;
        for (int i = 0; i < k; ++i) nrm = o_acc(nrm, o_mul(v[i], v[i]));
        nrm = o_sqrt(nrm);
        for (int i = 0; i < k; ++i) v[i] = o_div(v[i], nrm);
    }
    *last = v[k - 1];
    free(e2);
    free(v);
    free(dd);
    free(du);
    free(du2);
    free(dl);
    free(piv);
}

/* Lal::getMinEigen (sdpa_linear.cpp:27-122). */
odd o_lanczos_min_eig(long n, const odd *L, const odd *X) {
    odd min = o_from(1.0e+51), min_old = o_from(1.0e+52), error = o_from(1.0e+10);
    odd *diag = (odd *)malloc(sizeof(odd) * n), *off = (odd *)malloc(sizeof(odd) * n), *q = (odd *)malloc(sizeof(odd) * n),
        *qold = (odd *)malloc(sizeof(odd) * n), *r = (odd *)malloc(sizeof(odd) * n), *w = (odd *)malloc(sizeof(odd) * n),
        *tmp = (odd *)malloc(sizeof(odd) * n);
    for (long i = 0; i < n; ++i) {
        diag[i] = o_from(1.0e+50);
        off[i] = ZERO;
        q[i] = ZERO;
        r[i] = ONE;
    }
    odd beta = o_sqrt(o_from((double)n));
    long k = 0, kk = 0;
    odd sqn10 = o_add_d(o_sqrt(o_from((double)n)), 10.0);
    odd sqn9 = o_sqrt(o_add_d(o_from((double)n), 9.0));
    while (k < n && d_lt_dd((double)k, sqn10) && o_gt_d(beta, 1.0e-16) &&
           (o_gt(o_abs(o_sub(min, min_old)), o_add_d(o_mul_d(o_abs(min), 1.0e-5), 1.0e-8)) ||
            o_gt(o_abs(o_mul(error, beta)), o_add_d(o_mul_d(o_abs(min), 1.0e-2), 1.0e-4)))) {
        for (long i = 0; i < n; ++i) qold[i] = q[i];
        odd value = o_div(ONE, beta);
        for (long i = 0; i < n; ++i) q[i] = o_mul(value, r[i]);
        for (long i = 0; i < n; ++i) w[i] = q[i];
        o_trmv('T', n, L, n, w);
        o_gemv(n, n, X, n, w, tmp);
        for (long i = 0; i < n; ++i) w[i] = tmp[i];
        o_trmv('N', n, L, n, w);
        odd alpha = o_dot(n, q, 1, w, 1);
        diag[k] = alpha;
        for (long i = 0; i < n; ++i) r[i] = w[i];
        odd ma = o_neg(alpha), mb = o_neg(beta);
        if (!o_is_zero(ma))
            for (long i = 0; i < n; ++i) r[i] = o_acc(r[i], o_mul(ma, q[i]));
        if (!o_is_zero(mb))
            for (long i = 0; i < n; ++i) r[i] = o_acc(r[i], o_mul(mb, qold[i]));
        /* int-vs-dd comparisons promote the int to double (QD's
         * operator>=(double, dd_real) and operator>(double, dd_real)) */
        if (o_le_d(o_sqrt(o_from((double)k)), (double)kk) || k == n - 1 || d_gt_dd((double)k, sqn9)) {
            kk = 0;
            odd lam, last;
            tri_min_eig((int)k + 1, diag, off, &lam, &last);
            min_old = min;
            min = lam;
            error = last;
        }
        odd rr = o_dot(n, r, 1, r, 1);
        beta = o_sqrt(rr);
        off[k] = beta;
        ++k;
        ++kk;
    }
    odd ret = o_sub(min, o_abs(o_mul(error, beta)));
    free(diag);
    free(off);
    free(q);
    free(qold);
    free(r);
    free(w);
    free(tmp);
    return ret;
}
