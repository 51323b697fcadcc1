// Step-length eigenvalue lambda_min(L D L^T) per SDP block
// (Jal::getMinEigen, sdpa_jordan.cpp:55-88):
//   n > 20   Lanczos of Lal::getMinEigen (sdpa_linear.cpp:27-122) - same
//            start vector, recurrences (Rtrmv/Rgemv/Rdot orders), checkpoint
//            and stopping rules; the k x k tridiagonal eigenproblem at a
//            checkpoint is solved for its smallest eigenpair by Sturm
//            multisection over 15 warps plus inverse iteration (the reference uses
//            implicit QR, Rsteqr; both give the eigenvalue and the last
//            eigenvector component to dd rounding).
//   n <= 20  M = L (D L^T) by two Rgemm, then the smallest eigenvalue of the
//            lower triangle of M (the reference's Rsyev "N","L") by
//            Householder tridiagonalisation (one warp) and Sturm multisection.
// The whole Lanczos loop runs in one CTA per block: no host round trip per
// step.
#include "newton.h"

#include "blas.h"
#include "devops.cuh"
#include "eig_kernels.cuh"
#include "prof.h"

namespace sddd {

// QD double-vs-dd comparisons (dd_inline.h operator< / operator>)
__device__ __forceinline__ bool d_lt_dd(double a, dd_t b) { return a < b.hi || (a == b.hi && b.lo > 0.0); }
__device__ __forceinline__ bool d_gt_dd(double a, dd_t b) { return a > b.hi || (a == b.hi && b.lo < 0.0); }

// Number of eigenvalues of tridiagonal (d, e2 = e^2) below x.
__device__ int sturm_count(int k, const dd_t *d, const dd_t *e2, dd_t x) {
    int c = 0;
    dd_t q = dd_sub(d[0], x);
    if (q.hi < 0.0) c++;
    for (int i = 1; i < k; ++i) {
        if (dd_is_zero(q)) q = dd_make(1e-300, 0.0);
        q = dd_sub(dd_sub(d[i], x), dd_div(e2[i - 1], q));
        if (q.hi < 0.0) c++;
    }
    return c;
}

// The same count on the high parts in double: a quick estimate only.
__device__ int sturm_count_d(int k, const dd_t *d, const dd_t *e2, double x) {
    int c = 0;
    double q = d[0].hi - x;
    if (q < 0.0) c++;
    for (int i = 1; i < k; ++i) {
        if (q == 0.0) q = 1e-300;
        q = (d[i].hi - x) - e2[i - 1].hi / q;
        if (q < 0.0) c++;
    }
    return c;
}

// Smallest eigenvalue of the k x k tridiagonal (d, e) by multisection over
// the lanes of nw warps (warps 0 .. nw-1 of the CTA, all of their threads
// calling; nw = 1 runs on one warp alone); every thread returns the same
// value.  A first multisection in double on the high parts narrows the
// Gershgorin bracket to ~2^-40 of the spectrum's scale; that bracket is
// kept only when dd Sturm counts confirm it (no eigenvalue below its lower
// end, one below its upper end), and the dd multisection then runs from it.
// P = 32 nw points a round; each warp's ballot goes to shared memory (ball:
// 2 nw + 2 words, two alternating halves), so that every thread finds the
// first point with a non-zero count.
__device__ dd_t tri_min_eigenvalue(int k, const dd_t *d, const dd_t *e, dd_t *e2, int nw, unsigned *ball) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = threadIdx.x, P = 32 * nw;
    auto sync = [&]() {
        if (nw == 1)
            __syncwarp();
        else
            asm volatile("bar.sync 1, %0;" ::"r"(P) : "memory");
    };
    // index of the first point (over all warps) whose flag is set, or -1
    int half = 0;
    auto first_set = [&](bool flag) {
        const unsigned b = __ballot_sync(0xffffffffu, flag);
        unsigned *hb = ball + half * nw;
        if (lane == 0) hb[warp] = b;
        sync();
        int first = -1;
        for (int w = 0; w < nw; ++w)
            if (hb[w] != 0u) {
                first = 32 * w + __ffs(hb[w]) - 1;
                break;
            }
        half ^= 1; // the next round writes the other half: no second barrier
        return first;
    };
    dd_t lo = d[0], hi = d[0];
    for (int i = 0; i < k; ++i) {
        dd_t r = dd_zero();
        if (i > 0) r = dd_add(r, dd_abs(e[i - 1]));
        if (i + 1 < k) r = dd_add(r, dd_abs(e[i]));
        dd_t a = dd_sub(d[i], r), b = dd_add(d[i], r);
        if (dd_lt(a, lo)) lo = a;
        if (dd_gt(b, hi)) hi = b;
    }
    if (g == 0)
        for (int i = 0; i + 1 < k; ++i) e2[i] = dd_mul(e[i], e[i]);
    sync();
    dd_t w = dd_sub(hi, lo);
    lo = dd_sub(lo, dd_mul_d(w, 1e-10));
    hi = dd_add(hi, dd_mul_d(w, 1e-10));
    const double PP = (double)(P + 1);
    {
        double dlo = lo.hi, dhi = hi.hi;
        for (int round = 0; round < 12; ++round) {
            const double width = dhi - dlo;
            const double x = dlo + width * (double)(g + 1) / PP;
            const bool below = !(x > dlo) ? false : !(x < dhi) ? true : sturm_count_d(k, d, e2, x) >= 1;
            const int first = first_set(below);
            double nlo, nhi;
            if (first < 0) {
                nlo = dlo + width * (double)P / PP;
                nhi = dhi;
            } else {
                nhi = dlo + width * (double)(first + 1) / PP;
                nlo = first == 0 ? dlo : dlo + width * (double)first / PP;
            }
            if (!(nlo < nhi) || (nlo == dlo && nhi == dhi)) break;
            dlo = nlo;
            dhi = nhi;
        }
        const double rad = (fabs(lo.hi) + fabs(hi.hi) + (hi.hi - lo.hi)) * 0x1p-40;
        const dd_t blo = dd_max(lo, dd_from(dlo - rad)), bhi = dd_min(hi, dd_from(dhi + rad));
        bool bad = false;
        if (g == 0) bad = sturm_count(k, d, e2, blo) != 0;
        if (g == 1) bad = !(dd_lt(blo, bhi) && sturm_count(k, d, e2, bhi) >= 1);
        if (first_set(bad) < 0) {
            lo = blo;
            hi = bhi;
        }
    }
    for (int round = 0; round < 40; ++round) {
        const dd_t width = dd_sub(hi, lo);
        // P interior points x_g = lo + width (g+1)/(P+1); the smallest
        // eigenvalue lies below the first x with a non-zero Sturm count,
        // or above x_(P-1) when there is none.
        const dd_t x = dd_add(lo, dd_div_d(dd_mul_d(width, (double)(g + 1)), PP));
        bool below;
        if (!dd_gt(x, lo))
            below = false;
        else if (!dd_lt(x, hi))
            below = true;
        else
            below = sturm_count(k, d, e2, x) >= 1;
        const int first = first_set(below);
        dd_t nlo, nhi;
        if (first < 0) {
            nlo = dd_add(lo, dd_div_d(dd_mul_d(width, (double)P), PP));
            nhi = hi;
        } else {
            nhi = dd_add(lo, dd_div_d(dd_mul_d(width, (double)(first + 1)), PP));
            nlo = first == 0 ? lo : dd_add(lo, dd_div_d(dd_mul_d(width, (double)first), PP));
        }
        if (!dd_lt(nlo, nhi) || (dd_eq(nlo, lo) && dd_eq(nhi, hi))) break;
        lo = nlo;
        hi = nhi;
    }
    return dd_mul_d(dd_add(lo, hi), 0.5);
}

// Last component of the unit eigenvector of (d, e) for eigenvalue l:
// three steps of inverse iteration with a partially pivoted tridiagonal
// solve (single thread; k <= LZ_KMAX).  T - l I is factored once; each
// step solves with the factors.
__device__ dd_t tri_last_component(int k, const dd_t *d, const dd_t *e, dd_t l, dd_t tnorm, dd_t *v, dd_t *dd_, dd_t *du, dd_t *du2, dd_t *dl, int *piv) {
    for (int i = 0; i < k; ++i) v[i] = dd_from(1.0);
    {
        for (int i = 0; i < k; ++i) {
            dd_[i] = dd_sub(d[i], l);
            du[i] = (i + 1 < k) ? e[i] : dd_zero();
            dl[i] = (i + 1 < k) ? e[i] : dd_zero();
            du2[i] = dd_zero();
        }
        for (int i = 0; i + 1 < k; ++i) {
            if (!dd_lt(dd_abs(dd_[i]), dd_abs(dl[i]))) {
                piv[i] = 0;
                if (dd_is_zero(dd_[i])) dd_[i] = dd_mul_d(tnorm, 1e-32);
                dd_t f = dd_div(dl[i], dd_[i]);
                dl[i] = f;
                dd_[i + 1] = dd_sub(dd_[i + 1], dd_mul(f, du[i]));
            } else {
                piv[i] = 1;
                dd_t f = dd_div(dd_[i], dl[i]);
                dd_[i] = dl[i];
                dl[i] = f;
                dd_t t = du[i];
                du[i] = dd_[i + 1];
                dd_[i + 1] = dd_sub(t, dd_mul(f, dd_[i + 1]));
                if (i + 2 < k) {
                    du2[i] = du[i + 1];
                    du[i + 1] = dd_neg(dd_mul(f, du[i + 1]));
                }
            }
        }
        if (dd_is_zero(dd_[k - 1])) dd_[k - 1] = dd_mul_d(tnorm, 1e-32);
    }
    for (int it = 0; it < 3; ++it) {
        for (int i = 0; i + 1 < k; ++i) {
            if (piv[i]) {
                dd_t t = v[i];
                v[i] = v[i + 1];
                v[i + 1] = dd_sub(t, dd_mul(dl[i], v[i + 1]));
            } else {
                v[i + 1] = dd_sub(v[i + 1], dd_mul(dl[i], v[i]));
            }
        }
        for (int i = k - 1; i >= 0; --i) {
            dd_t t = v[i];
            if (i + 1 < k) t = dd_sub(t, dd_mul(du[i], v[i + 1]));
            if (i + 2 < k) t = dd_sub(t, dd_mul(du2[i], v[i + 2]));
            v[i] = dd_div(t, dd_[i]);
        }
        dd_t nrm = dd_zero();
        for (int i = 0; i < k; ++i) nrm = dd_acc(nrm, dd_mul(v[i], v[i]));
        nrm = dd_sqrt(nrm);
        for (int i = 0; i < k; ++i) v[i] = dd_div(v[i], nrm);
    }
    return v[k - 1];
}

// Warps of the Lanczos CTA that run the checkpoint's multisection; the last
// warp's lane 0 computes r.r beside them.
constexpr int LZ_EIG_WARPS = LZ_THREADS / 32 - 1;
struct LanczosShared {
    dd_t diag[LZ_KMAX], off[LZ_KMAX], e2[LZ_KMAX];
    unsigned ball[2 * LZ_EIG_WARPS + 2];
    dd_t v[LZ_KMAX], t0[LZ_KMAX], t1[LZ_KMAX], t2[LZ_KMAX], t3[LZ_KMAX];
    int piv[LZ_KMAX];
    dd_t alpha, beta, value, mn, mn_old, err, rr;
    int go, check;
};

// One CTA per block: work holds 5 n-vectors (q, qold, r, w, tmp).  With a
// second space (Lsp2, Dsp2), CTAs nb.. take the same blocks of that space,
// so the two step-length eigenvalues run side by side.
__global__ void __launch_bounds__(LZ_THREADS) lanczos_kernel(const int *blk_ids, int nb, const int *sizes, const long *off, const dd_t *Lsp,
                                                             const dd_t *Dsp, const dd_t *Lsp2, const dd_t *Dsp2, dd_t *work, long work_stride, dd_t *out) {
    __shared__ LanczosShared S;
    const bool second = (int)blockIdx.x >= nb;
    const int b = blk_ids[second ? blockIdx.x - nb : blockIdx.x];
    if (second) {
        Lsp = Lsp2;
        Dsp = Dsp2;
    }
    const int n = sizes[b];
    const dd_t *L = Lsp + off[b], *X = Dsp + off[b];
    dd_t *q = work + blockIdx.x * work_stride, *qold = q + n, *r = qold + n, *w = r + n, *tmp = w + n;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < n; i += nt) {
        st_dd(q + i, dd_zero());
        st_dd(r + i, dd_from(1.0));
    }
    if (tid == 0) {
        S.mn = dd_from(1.0e+51);
        S.mn_old = dd_from(1.0e+52);
        S.err = dd_from(1.0e+10);
        S.beta = dd_sqrt(dd_from((double)n));
    }
    __syncthreads();
    const dd_t sqn10 = dd_add_d(dd_sqrt(dd_from((double)n)), 10.0);
    const dd_t sqn9 = dd_sqrt(dd_add_d(dd_from((double)n), 9.0));
    int k = 0, kk = 0;
    while (true) {
        if (tid == 0) {
            const dd_t mn = S.mn, mo = S.mn_old;
            bool c1 = dd_gt(dd_abs(dd_sub(mn, mo)), dd_add_d(dd_mul_d(dd_abs(mn), 1.0e-5), 1.0e-8));
            bool c2 = dd_gt(dd_abs(dd_mul(S.err, S.beta)), dd_add_d(dd_mul_d(dd_abs(mn), 1.0e-2), 1.0e-4));
            S.go = (k < n && k < LZ_KMAX && d_lt_dd((double)k, sqn10) && dd_gt_d(S.beta, 1.0e-16) && (c1 || c2)) ? 1 : 0;
            S.value = dd_div(dd_from(1.0), S.beta);
        }
        __syncthreads();
        if (!S.go) break;
        const dd_t value = S.value;
        // qold = q; q = r * value (Rcopy + Rscal)
        for (int i = tid; i < n; i += nt) {
            st_dd(qold + i, ld_dd(q + i));
            dd_t qi = dd_mul(value, ld_dd(r + i));
            st_dd(q + i, qi);
        }
        __syncthreads();
        // Each product below is a sequential chain per entry; the loads of
        // eight steps go out ahead of their terms (same order of the sums).
        // w = L^T q (Rtrmv "Lower","Transpose")
        for (int j = tid; j < n; j += nt) {
            const dd_t *Lc = L + (long)n * j;
            dd_t t = dd_mul(ld_dd(q + j), ld_dd(Lc + j));
            int i = j + 1;
            for (; i + 8 <= n; i += 8) {
                dd_t a[8], b[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    a[u] = ld_dd(Lc + i + u);
                    b[u] = ld_dd(q + i + u);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) t = dd_acc(t, dd_mul(a[u], b[u]));
            }
            for (; i < n; ++i) t = dd_acc(t, dd_mul(ld_dd(Lc + i), ld_dd(q + i)));
            st_dd(w + j, t);
        }
        __syncthreads();
        // tmp = X w (Rgemv "N", alpha 1, beta 0)
        for (int i = tid; i < n; i += nt) {
            dd_t t = dd_zero();
            int j = 0;
            for (; j + 8 <= n; j += 8) {
                dd_t a[8], b[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    a[u] = ld_dd(w + j + u);
                    b[u] = ld_dd(X + i + (long)n * (j + u));
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) t = dd_acc(t, dd_mul(dd_mul(dd_from(1.0), a[u]), b[u]));
            }
            for (; j < n; ++j) t = dd_acc(t, dd_mul(dd_mul(dd_from(1.0), ld_dd(w + j)), ld_dd(X + i + (long)n * j)));
            st_dd(tmp + i, t);
        }
        __syncthreads();
        // w = L tmp (Rtrmv "Lower","NoTranspose": row i, j descending)
        for (int i = tid; i < n; i += nt) {
            dd_t t = dd_mul(ld_dd(tmp + i), ld_dd(L + i + (long)n * i));
            int j = i - 1;
            for (; j >= 7; j -= 8) {
                dd_t a[8], b[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    a[u] = ld_dd(tmp + j - u);
                    b[u] = ld_dd(L + i + (long)n * (j - u));
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (!dd_is_zero(a[u])) t = dd_acc(t, dd_mul(a[u], b[u]));
            }
            for (; j >= 0; --j) {
                dd_t xj = ld_dd(tmp + j);
                if (!dd_is_zero(xj)) t = dd_acc(t, dd_mul(xj, ld_dd(L + i + (long)n * j)));
            }
            st_dd(w + i, t);
        }
        __syncthreads();
        if (tid == 0) {
            S.alpha = seq_dot(n, q, w);
            S.diag[k] = S.alpha;
        }
        __syncthreads();
        const dd_t ma = dd_neg(S.alpha), mb = dd_neg(S.beta);
        // r = w - alpha q - beta qold (Rcopy, Raxpy, Raxpy)
        for (int i = tid; i < n; i += nt) {
            dd_t ri = ld_dd(w + i);
            if (!dd_is_zero(ma)) ri = dd_acc(ri, dd_mul(ma, ld_dd(q + i)));
            if (!dd_is_zero(mb)) ri = dd_acc(ri, dd_mul(mb, ld_dd(qold + i)));
            st_dd(r + i, ri);
        }
        __syncthreads();
        // checkpoint: kk >= sqrt(k) || k == n-1 || k > sqrt(n+9)
        const dd_t sk = dd_sqrt(dd_from((double)k));
        const bool check = dd_le_d(sk, (double)kk) || k == n - 1 || d_gt_dd((double)k, sqn9);
        if (check) {
            kk = 0;
            if (tid < 32 * LZ_EIG_WARPS) {
                dd_t lam = tri_min_eigenvalue(k + 1, S.diag, S.off, S.e2, LZ_EIG_WARPS, S.ball);
                if (tid == 0) {
                    dd_t lo = S.diag[0], hi = S.diag[0];
                    for (int i = 0; i <= k; ++i) {
                        lo = dd_min(lo, S.diag[i]);
                        hi = dd_max(hi, S.diag[i]);
                    }
                    dd_t tnorm = dd_add(dd_add(dd_abs(lo), dd_abs(hi)), dd_from(1e-300));
                    dd_t last = tri_last_component(k + 1, S.diag, S.off, lam, tnorm, S.v, S.t0, S.t1, S.t2, S.t3, S.piv);
                    S.mn_old = S.mn;
                    S.mn = lam;
                    S.err = last;
                }
            }
        }
        // r.r on the last warp, beside the checkpoint's warps
        if (tid == 32 * LZ_EIG_WARPS) S.rr = seq_dot(n, r, r);
        __syncthreads();
        if (tid == 0) {
            S.beta = dd_sqrt(S.rr);
            S.off[k] = S.beta;
        }
        __syncthreads();
        ++k;
        ++kk;
    }
    if (tid == 0) out[blockIdx.x] = dd_sub(S.mn, dd_abs(dd_mul(S.err, S.beta)));
}

// Smallest eigenvalue of the lower triangle of an n x n symmetric M
// (n <= 32): Householder tridiagonalisation, then the warp multisection of
// tri_min_eigenvalue.  One warp per block: the scalar sums of a reflector
// on lane 0 in sequence, the products with A and the rank-2 update row by
// row over the lanes, A in shared memory.
__global__ void __launch_bounds__(32) small_min_eig_kernel(const int *blk_ids, const int *sizes, const long *off, const dd_t *Msp, dd_t *out) {
    __shared__ dd_t A[32][33];
    __shared__ dd_t v[32], p[32], d[32], e[32], e2[32];
    __shared__ dd_t tau_s, K_s;
    __shared__ int skip;
    const int lane = threadIdx.x;
    const int b = blk_ids[blockIdx.x];
    const int n = sizes[b];
    const dd_t *M = Msp + off[b];
    for (int j = 0; j < n; ++j)
        if (lane >= j && lane < n) {
            const dd_t x = ld_dd(M + lane + (long)n * j);
            A[lane][j] = x;
            A[j][lane] = x;
        }
    __syncwarp();
    for (int k = 0; k + 2 < n; ++k) {
        if (lane == 0) {
            skip = 0;
            dd_t s = dd_zero();
            for (int i = k + 1; i < n; ++i) s = dd_acc(s, dd_mul(A[i][k], A[i][k]));
            const dd_t nrm = dd_sqrt(s);
            if (dd_is_zero(nrm)) {
                skip = 1;
            } else {
                const dd_t alpha = A[k + 1][k].hi < 0.0 ? nrm : dd_neg(nrm);
                for (int i = 0; i < n; ++i) v[i] = dd_zero();
                v[k + 1] = dd_sub(A[k + 1][k], alpha);
                for (int i = k + 2; i < n; ++i) v[i] = A[i][k];
                dd_t vv = dd_zero();
                for (int i = k + 1; i < n; ++i) vv = dd_acc(vv, dd_mul(v[i], v[i]));
                if (dd_is_zero(vv))
                    skip = 1;
                else
                    tau_s = dd_div(dd_from(2.0), vv);
            }
        }
        __syncwarp();
        if (skip) continue;
        const dd_t tau = tau_s;
        // p = tau A v (row i on lane i)
        if (lane < n) {
            dd_t t = dd_zero();
            for (int j = k + 1; j < n; ++j) t = dd_acc(t, dd_mul(A[lane][j], v[j]));
            p[lane] = dd_mul(tau, t);
        }
        __syncwarp();
        // K = tau/2 v^T p ; w = p - K v
        if (lane == 0) {
            dd_t vp = dd_zero();
            for (int i = k + 1; i < n; ++i) vp = dd_acc(vp, dd_mul(v[i], p[i]));
            K_s = dd_mul(dd_mul_d(tau, 0.5), vp);
        }
        __syncwarp();
        if (lane < n) p[lane] = dd_sub(p[lane], dd_mul(K_s, v[lane]));
        __syncwarp();
        // A -= v w^T + w v^T (row i on lane i)
        if (lane < n) {
            const dd_t vi = v[lane], pi = p[lane];
            for (int j = 0; j < n; ++j) A[lane][j] = dd_sub(dd_sub(A[lane][j], dd_mul(vi, p[j])), dd_mul(pi, v[j]));
        }
        __syncwarp();
    }
    if (lane < n) {
        d[lane] = A[lane][lane];
        if (lane + 1 < n) e[lane] = A[lane + 1][lane];
    }
    __syncwarp();
    __shared__ unsigned ball[4];
    const dd_t lam = tri_min_eigenvalue(n, d, e, e2, 1, ball);
    if (lane == 0) out[blockIdx.x] = lam;
}

// The small blocks (n <= 20) of one space: DLS2 = D L^T (Rgemm "N","T"),
// DLS1 = L DLS2 (Rgemm "N","N"), then each block's smallest eigenvalue to
// res[0 ..) in block order.
static void small_blocks(Context &c, const Space &L, const Space &D, const std::vector<int> &small, dd_t *res) {
    cudaStream_t st = c.stream;
    for (const BlockRun &r : c.runs) {
        if (r.n > 20) continue;
        const int n = r.n, l = r.first;
        const long nn = (long)n * n;
        gemm(st, 'N', 'T', GEMM_STORE, n, n, n, D.blk(c.off, l), n, nn, L.blk(c.off, l), n, nn, c.W2.blk(c.off, l), n, nn, r.count, false);
        gemm(st, 'N', 'N', GEMM_STORE, n, n, n, L.blk(c.off, l), n, nn, c.W2.blk(c.off, l), n, nn, c.W1.blk(c.off, l), n, nn, r.count, false);
    }
    small_min_eig_kernel<<<(unsigned)small.size(), 32, 0, st>>>(c.eig_ids_small.p, c.d_sizes.p, c.d_off.p, c.W1.buf.p, res);
    CK_LAUNCH();
}

// min over the blocks of lambda_min(L D L^T) for nsp spaces (1 or 2): the
// big blocks' Lanczos of all spaces in one launch; results per space in
// block order, then the minimum as the reference takes it.
static void min_eig_spaces(Context &c, int nsp, const Space *L[2], const Space *D[2], dd_t out[2]) {
    cudaStream_t st = c.stream;
    PROF_SCOPE("min_eig", st);
    std::vector<int> big, small;
    for (int l = 0; l < c.nSDP; ++l) (c.sizes[l] > 20 ? big : small).push_back(l);
    static_assert(LZ_KMAX >= 64, "Lanczos step bound");
    if (c.eig_ids_big.n != big.size() || c.eig_ids_small.n != small.size() || c.eig_ids_gen != c.upload_gen) {
        c.eig_ids_big.upload(big, st);
        c.eig_ids_small.upload(small, st);
        c.eig_ids_gen = c.upload_gen;
    }
    const size_t nb = big.size(), ns = small.size();
    // result slots: space s at s * nSDP: big blocks first, then the small
    dd_t *res = c.scal.p;
    if (nb > 0) {
        long maxn = 0;
        for (int l : big) maxn = std::max<long>(maxn, c.sizes[l]);
        c.eig_work.alloc(5 * maxn * nb * nsp);
        // the two spaces' CTAs write slots 0 .. 2 nb - 1; spread below
        lanczos_kernel<<<(unsigned)(nb * nsp), LZ_THREADS, 0, st>>>(c.eig_ids_big.p, (int)nb, c.d_sizes.p, c.d_off.p, L[0]->buf.p, D[0]->buf.p,
                                                                   L[nsp - 1]->buf.p, D[nsp - 1]->buf.p, c.eig_work.p, 5 * maxn, res + 2 * c.nSDP);
        CK_LAUNCH();
    }
    for (int sp = 0; sp < nsp && ns > 0; ++sp) small_blocks(c, *L[sp], *D[sp], small, res + (size_t)sp * c.nSDP + nb);
    if (nb > 0) {
        for (int sp = 0; sp < nsp; ++sp)
            CK(cudaMemcpyAsync(res + (size_t)sp * c.nSDP, res + 2 * c.nSDP + sp * nb, sizeof(dd_t) * nb, cudaMemcpyDeviceToDevice, st));
    }
    std::vector<dd_t> h((size_t)nsp * c.nSDP);
    d2h(c, h.data(), res, sizeof(dd_t) * h.size());
    for (int sp = 0; sp < nsp; ++sp) {
        // blocks in order: big blocks' values first in the slots, then the small
        const dd_t *v = h.data() + (size_t)sp * c.nSDP;
        size_t bi = 0, si = 0;
        dd_t mn = dd_from(1.0e50);
        for (int l = 0; l < c.nSDP; ++l) {
            const dd_t x = (c.sizes[l] > 20) ? v[bi++] : v[nb + si++];
            if (dd_lt(x, mn)) mn = x;
        }
        out[sp] = mn;
    }
}

dd_t min_eig(Context &c, const Space &L, const Space &D) {
    const Space *Ls[2] = {&L, &L}, *Ds[2] = {&D, &D};
    dd_t out[2];
    min_eig_spaces(c, 1, Ls, Ds, out);
    return out[0];
}

void min_eig_pair(Context &c, const Space &L1, const Space &D1, const Space &L2, const Space &D2, dd_t &out1, dd_t &out2) {
    const Space *Ls[2] = {&L1, &L2}, *Ds[2] = {&D1, &D2};
    dd_t out[2];
    min_eig_spaces(c, 2, Ls, Ds, out);
    out1 = out[0];
    out2 = out[1];
}

} // namespace sddd
