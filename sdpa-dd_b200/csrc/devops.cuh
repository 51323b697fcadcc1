// Device helpers shared by the Newton-step kernels.
#pragma once
#include "common.cuh"

namespace sddd {

// A . D for a sparse block matrix given as COO (upper-triangle entries in
// input order): Lal::getInnerProduct(SparseMatrix, DenseMatrix),
// sdpa_linear.cpp:202-298 - the first nnz % 4 terms one at a time, then
// groups of four summed with operator+ before one operator+=.
__device__ __forceinline__ dd_t sparse_dot_dense(int n, int nnz, const int *row, const int *col, const dd_t *val, const dd_t *D) {
    auto term = [&](int q) -> dd_t {
        int i = row[q], j = col[q];
        dd_t v = val[q];
        if (i == j) return dd_mul(v, ld_dd(D + i + (long)n * j));
        return dd_mul(v, dd_add(ld_dd(D + i + (long)n * j), ld_dd(D + j + (long)n * i)));
    };
    dd_t ret = dd_zero();
    const int amari = nnz % 4, shou = nnz / 4;
    for (int q = 0; q < amari; ++q) ret = dd_acc(ret, term(q));
    for (int c = 0, q = amari; c < shou; ++c, q += 4) {
        dd_t r1 = term(q), r2 = term(q + 1), r3 = term(q + 2), r4 = term(q + 3);
        ret = dd_acc(ret, dd_add(dd_add(dd_add(r1, r2), r3), r4));
    }
    return ret;
}

// Rdot with one OpenMP thread: templ += x[k] y[k]; return 0 + templ
// (mplapack/Rdot_omp.cpp).  The loads of eight steps go out ahead of
// their terms; the sum's order is unchanged.
__device__ __forceinline__ dd_t seq_dot(long n, const dd_t *x, const dd_t *y) {
    dd_t t = dd_zero();
    long k = 0;
    for (; k + 8 <= n; k += 8) {
        dd_t a[8], b[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            a[u] = ld_dd(x + k + u);
            b[u] = ld_dd(y + k + u);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) t = dd_acc(t, dd_mul(a[u], b[u]));
    }
    for (; k < n; ++k) t = dd_acc(t, dd_mul(ld_dd(x + k), ld_dd(y + k)));
    return dd_acc(dd_zero(), t);
}

} // namespace sddd
