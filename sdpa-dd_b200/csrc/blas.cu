// Dense dd linear algebra on the FP64 pipe of sm_100a.
//
// Every kernel here reproduces the per-entry operation order of the
// MPLAPACK routine it replaces, so that with the same inputs it returns the
// reference's dd results bit for bit:
//   gemm       Rgemm_{NN,TN,NT}_omp  (mplapack/Rgemm_*_omp.cpp): each C(i,j)
//              is a sequential sum over k of "c += a*b" steps
//   potrf      Rpotrf("Lower") (mplapack/Rpotrf.cpp:124-142 with Rsyrk,
//              Rgemm, Rtrsm, Rpotrf2): entry (i,j) receives the products
//              L(j,k)L(i,k) for k ascending as "x = x - p" steps, the diagonal
//              takes sqrt and the column below is scaled by 1/L(j,j)
//   trsv       Rtrsv("Lower", "N"/"T", "NonUnit") (mplapack/Rtrsv.cpp)
//   inv_lower  Rtrsm("Left","Lower","N","N") on the identity
//              (Lal::getInvLowTriangularMatrix, sdpa_linear.cpp:397-412)
//   trmm_lt    Rtrmm("Left","Lower","Transpose","NonUnit")
//              (Jal::getInvCholAndInv, sdpa_jordan.cpp:154-170)
//   symmetrize Lal::getSymmetrize (sdpa_linear.cpp:414-438)
// The blocking below (tiles, panels) is the B200 schedule; it never
// reorders the operations that land on one entry.
#include "blas.h"
#include "prof.h"

#include <algorithm>

namespace sddd {

// ===================================================================== GEMM
// Tile: BM x BN outputs per CTA, BK-deep k slices staged in shared memory,
// TM x TN outputs per thread.  Shared tiles are k-major and padded by one
// element so that transposed tile loads do not collide on banks.
template <int BM, int BN, int BK, int TM, int TN, bool TA, bool TB, int MODE>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    gemm_kernel(int M, int N, int K, const dd_t *__restrict__ A, long lda, long sA, const dd_t *__restrict__ B, long ldb, long sB, dd_t *C,
                long ldc, long sC, int lower) {
    constexpr int TX = BN / TN, TY = BM / TM, NT = TX * TY;
    __shared__ double2 As[BK][BM + 1];
    __shared__ double2 Bs[BK][BN + 1];
    const long bz = blockIdx.z;
    A += bz * sA;
    B += bz * sB;
    C += bz * sC;
    const int i0 = blockIdx.y * BM, j0 = blockIdx.x * BN;
    if (lower && i0 + BM <= j0) return; // tile entirely above the diagonal
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    dd_t acc[TM][TN];
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) {
            int gi = i0 + ty + TY * r, gj = j0 + tx + TX * c;
            if (MODE == GEMM_STORE || gi >= M || gj >= N)
                acc[r][c] = dd_zero();
            else
                acc[r][c] = ld_dd(C + gi + ldc * (long)gj);
        }
    for (int k0 = 0; k0 < K; k0 += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            int ii, kk;
            if (!TA) {
                ii = e % BM;
                kk = e / BM;
            } else {
                kk = e % BK;
                ii = e / BK;
            }
            int gi = i0 + ii, gk = k0 + kk;
            double2 v = make_double2(0.0, 0.0);
            if (gi < M && gk < K) v = *reinterpret_cast<const double2 *>(TA ? A + gk + lda * (long)gi : A + gi + lda * (long)gk);
            As[kk][ii] = v;
        }
        for (int e = tid; e < BN * BK; e += NT) {
            int jj, kk;
            if (!TB) {
                kk = e % BK;
                jj = e / BK;
            } else {
                jj = e % BN;
                kk = e / BN;
            }
            int gj = j0 + jj, gk = k0 + kk;
            double2 v = make_double2(0.0, 0.0);
            if (gj < N && gk < K) v = *reinterpret_cast<const double2 *>(TB ? B + gj + ldb * (long)gk : B + gk + ldb * (long)gj);
            Bs[kk][jj] = v;
        }
        __syncthreads();
        const int kmax = min(BK, K - k0);
        for (int kk = 0; kk < kmax; ++kk) {
            dd_t a[TM], b[TN];
#pragma unroll
            for (int r = 0; r < TM; ++r) {
                double2 v = As[kk][ty + TY * r];
                a[r] = dd_make(v.x, v.y);
            }
#pragma unroll
            for (int c = 0; c < TN; ++c) {
                double2 v = Bs[kk][tx + TX * c];
                b[c] = dd_make(v.x, v.y);
            }
#pragma unroll
            for (int r = 0; r < TM; ++r)
#pragma unroll
                for (int c = 0; c < TN; ++c) {
                    dd_t p = dd_mul(b[c], a[r]);
                    acc[r][c] = (MODE == GEMM_SUB) ? dd_sub(acc[r][c], p) : dd_acc(acc[r][c], p);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) {
            int gi = i0 + ty + TY * r, gj = j0 + tx + TX * c;
            if (gi < M && gj < N && (!lower || gi >= gj)) st_dd(C + gi + ldc * (long)gj, acc[r][c]);
        }
}

template <bool TA, bool TB, int MODE>
static void gemm_launch(cudaStream_t st, int M, int N, int K, const dd_t *A, long lda, long sA, const dd_t *B, long ldb, long sB, dd_t *C, long ldc,
                        long sC, int batch, bool lower) {
    constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4;
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM), batch);
    gemm_kernel<BM, BN, BK, TM, TN, TA, TB, MODE><<<grid, (BM / TM) * (BN / TN), 0, st>>>(M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, lower ? 1 : 0);
    CK_LAUNCH();
}

void gemm(cudaStream_t st, char ta, char tb, int mode, int M, int N, int K, const dd_t *A, long lda, long sA, const dd_t *B, long ldb, long sB,
          dd_t *C, long ldc, long sC, int batch, bool lower) {
    if (M <= 0 || N <= 0 || batch <= 0) return;
    if (K <= 0 && mode == GEMM_SUB) return;
#define GL(TA_, TB_, MD_) gemm_launch<TA_, TB_, MD_>(st, M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, batch, lower)
    bool a = ta == 'T', b = tb == 'T';
    if (mode == GEMM_STORE) {
        if (!a && !b) GL(false, false, GEMM_STORE);
        else if (a && !b) GL(true, false, GEMM_STORE);
        else if (!a && b) GL(false, true, GEMM_STORE);
        else GL(true, true, GEMM_STORE);
    } else if (mode == GEMM_SUB) {
        if (!a && b) GL(false, true, GEMM_SUB);
        else if (!a && !b) GL(false, false, GEMM_SUB);
        else throw Error(ERR_ARG, "gemm: unsupported SUB variant");
    } else {
        if (!a && !b) GL(false, false, GEMM_ACC);
        else if (a && !b) GL(true, false, GEMM_ACC);
        else throw Error(ERR_ARG, "gemm: unsupported ACC variant");
    }
#undef GL
}

// ==================================================================== POTRF
// Diagonal block: right-looking dd Cholesky of an nb x nb block held in
// shared memory (lower triangle).  On a non-positive or NaN pivot the
// 1-based global column goes to *info and the block stops (Rpotrf2's n=1
// test, mplapack/Rpotrf2.cpp).  1/L(j,j) for the panel goes to rdiag.
__global__ void potrf_diag_kernel(dd_t *A, long lda, int nb, int c0, int *info, dd_t *rdiag) {
    extern __shared__ double2 sm[];
    double2 *S = sm;                // nb x nb, column-major
    __shared__ double2 rk;
    __shared__ int fail;
    if (*info != 0) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nb * nb; e += nt) {
        int i = e % nb, j = e / nb;
        S[e] = (i >= j) ? *reinterpret_cast<const double2 *>(A + (c0 + i) + lda * (long)(c0 + j)) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        if (tid == 0) {
            dd_t d = dd_make(S[k + nb * k].x, S[k + nb * k].y);
            if (dd_le_d(d, 0.0) || dd_isnan(d)) {
                fail = 1;
                *info = c0 + k + 1;
            } else {
                dd_t l = dd_sqrt(d);
                S[k + nb * k] = make_double2(l.hi, l.lo);
                dd_t r = dd_div(dd_from(1.0), l);
                rk = make_double2(r.hi, r.lo);
                rdiag[k] = r;
                fail = 0;
            }
        }
        __syncthreads();
        if (fail) return;
        const dd_t r = dd_make(rk.x, rk.y);
        for (int i = k + 1 + tid; i < nb; i += nt) {
            double2 v = S[i + nb * k];
            dd_t x = dd_mul(r, dd_make(v.x, v.y));
            S[i + nb * k] = make_double2(x.hi, x.lo);
        }
        __syncthreads();
        // trailing update of the block: (i, j) with k < j <= i < nb
        const int w = nb - 1 - k;
        for (int p = tid; p < w * w; p += nt) {
            int i = k + 1 + p % w, j = k + 1 + p / w;
            if (i < j) continue;
            double2 xi = S[i + nb * k], xj = S[j + nb * k], v = S[i + nb * j];
            dd_t y = dd_sub(dd_make(v.x, v.y), dd_mul(dd_make(xj.x, xj.y), dd_make(xi.x, xi.y)));
            S[i + nb * j] = make_double2(y.hi, y.lo);
        }
        __syncthreads();
    }
    for (int e = tid; e < nb * nb; e += nt) {
        int i = e % nb, j = e / nb;
        if (i >= j) *reinterpret_cast<double2 *>(A + (c0 + i) + lda * (long)(c0 + j)) = S[e];
    }
}

// Panel rows below the diagonal block: each CTA takes PR rows and solves
// them against L11 in shared memory, column by column (Rtrsm "Right",
// "Lower", "Transpose": x(i,j) -= L(j,k) x(i,k) for k < j, then
// x(i,j) *= 1/L(j,j)).
constexpr int PANEL_ROWS = 64;
__global__ void potrf_panel_kernel(dd_t *A, long lda, int n, int nb, int c0, const int *info, const dd_t *rdiag) {
    extern __shared__ double2 sm[];
    double2 *L11 = sm;               // nb x nb
    double2 *P = sm + nb * nb;       // PANEL_ROWS x nb, column-major ld PANEL_ROWS
    double2 *R = P + PANEL_ROWS * nb; // nb reciprocals
    if (*info != 0) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int r0 = c0 + nb + blockIdx.x * PANEL_ROWS;
    const int rows = min(PANEL_ROWS, n - r0);
    if (rows <= 0) return;
    for (int e = tid; e < nb * nb; e += nt) {
        int i = e % nb, j = e / nb;
        L11[e] = (i >= j) ? *reinterpret_cast<const double2 *>(A + (c0 + i) + lda * (long)(c0 + j)) : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < PANEL_ROWS * nb; e += nt) {
        int i = e % PANEL_ROWS, j = e / PANEL_ROWS;
        P[e] = (i < rows) ? *reinterpret_cast<const double2 *>(A + (r0 + i) + lda * (long)(c0 + j)) : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < nb; e += nt) R[e] = make_double2(rdiag[e].hi, rdiag[e].lo);
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        const dd_t r = dd_make(R[k].x, R[k].y);
        for (int i = tid; i < rows; i += nt) {
            double2 v = P[i + PANEL_ROWS * k];
            dd_t x = dd_mul(r, dd_make(v.x, v.y));
            P[i + PANEL_ROWS * k] = make_double2(x.hi, x.lo);
        }
        __syncthreads();
        const int w = nb - 1 - k;
        for (int e = tid; e < rows * w; e += nt) {
            int i = e % rows, j = k + 1 + e / rows;
            double2 ljk = L11[j + nb * k], xik = P[i + PANEL_ROWS * k], v = P[i + PANEL_ROWS * j];
            dd_t y = dd_sub(dd_make(v.x, v.y), dd_mul(dd_make(ljk.x, ljk.y), dd_make(xik.x, xik.y)));
            P[i + PANEL_ROWS * j] = make_double2(y.hi, y.lo);
        }
        __syncthreads();
    }
    for (int e = tid; e < PANEL_ROWS * nb; e += nt) {
        int i = e % PANEL_ROWS, j = e / PANEL_ROWS;
        if (i < rows) *reinterpret_cast<double2 *>(A + (r0 + i) + lda * (long)(c0 + j)) = P[e];
    }
}

// Right-looking blocked Cholesky: per panel of POTRF_NB columns, factor the
// diagonal block, solve the rows below, then subtract the panel's outer
// product from the trailing lower triangle (GEMM_SUB keeps each entry's
// k-order).  info is a device int; 0 on success, else the failing column.
void potrf(cudaStream_t st, dd_t *A, long lda, int n, int *info_dev, dd_t *rdiag_dev) {
    if (n <= 0) return;
    static bool attr = false;
    const int nbmax = POTRF_NB;
    const size_t smem_diag = sizeof(double2) * nbmax * nbmax;
    const size_t smem_panel = sizeof(double2) * (nbmax * nbmax + PANEL_ROWS * nbmax + nbmax);
    if (!attr) {
        CK(cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_diag));
        CK(cudaFuncSetAttribute(potrf_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_panel));
        attr = true;
    }
    for (int c0 = 0; c0 < n; c0 += nbmax) {
        const int nb = std::min(nbmax, n - c0);
        {
            PROF_SCOPE("potrf_diag", st);
            potrf_diag_kernel<<<1, 256, sizeof(double2) * nb * nb, st>>>(A, lda, nb, c0, info_dev, rdiag_dev);
            CK_LAUNCH();
        }
        const int below = n - c0 - nb;
        if (below <= 0) break;
        {
            PROF_SCOPE("potrf_panel", st);
            potrf_panel_kernel<<<ceil_div(below, PANEL_ROWS), 256, sizeof(double2) * (nb * nb + PANEL_ROWS * nb + nb), st>>>(A, lda, n, nb, c0, info_dev,
                                                                                                                          rdiag_dev);
            CK_LAUNCH();
        }
        dd_t *panel = A + (c0 + nb) + lda * (long)c0;
        dd_t *trail = A + (c0 + nb) + lda * (long)(c0 + nb);
        PROF_SCOPE("potrf_trailing_update", st);
        gemm(st, 'N', 'T', GEMM_SUB, below, below, nb, panel, lda, 0, panel, lda, 0, trail, lda, 0, 1, true);
    }
}

// Zero the strict upper triangle (Lal::getCholesky, sdpa_linear.cpp:320-343).
__global__ void zero_upper_kernel(dd_t *A, long lda, int n) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    int i = e % n, j = e / n;
    if (i < j) st_dd(A + i + lda * (long)j, dd_zero());
}
void zero_upper(cudaStream_t st, dd_t *A, long lda, int n) {
    zero_upper_kernel<<<ceil_div((long)n * n, 256), 256, 0, st>>>(A, lda, n);
    CK_LAUNCH();
}

// ===================================================================== TRSV
constexpr int TRSV_B = 64;

// Forward solve, launch p: rows of blocks c >= p first take block p-1's
// solution (x(i) -= x(j) L(i,j), j ascending); then CTA p solves its own
// diagonal block (x(j) /= L(j,j) when x(j) != 0, then x(i) -= x(j) L(i,j)).
__global__ void trsv_fwd_kernel(const dd_t *L, long lda, int n, dd_t *x, int p) {
    __shared__ double2 xs[TRSV_B];
    const int c = p + blockIdx.x;
    const int r0 = c * TRSV_B, tid = threadIdx.x;
    const int i = r0 + tid;
    dd_t xi = dd_zero();
    if (i < n) xi = ld_dd(x + i);
    if (p > 0) {
        const int j0 = (p - 1) * TRSV_B;
        for (int t = tid; t < TRSV_B; t += blockDim.x) xs[t] = *reinterpret_cast<const double2 *>(x + j0 + t);
        __syncthreads();
        if (i < n)
            for (int t = 0; t < TRSV_B; ++t) {
                dd_t xj = dd_make(xs[t].x, xs[t].y);
                if (!dd_is_zero(xj)) xi = dd_sub(xi, dd_mul(xj, ld_dd(L + i + lda * (long)(j0 + t))));
            }
        __syncthreads();
    }
    if (c == p) {
        const int nb = min(TRSV_B, n - r0);
        xs[tid] = make_double2(xi.hi, xi.lo);
        __syncthreads();
        for (int t = 0; t < nb; ++t) {
            if (tid == t) {
                dd_t v = dd_make(xs[t].x, xs[t].y);
                if (!dd_is_zero(v)) v = dd_div(v, ld_dd(L + (r0 + t) + lda * (long)(r0 + t)));
                xs[t] = make_double2(v.hi, v.lo);
            }
            __syncthreads();
            dd_t xt = dd_make(xs[t].x, xs[t].y);
            if (tid > t && tid < nb && !dd_is_zero(xt)) {
                dd_t v = dd_make(xs[tid].x, xs[tid].y);
                v = dd_sub(v, dd_mul(xt, ld_dd(L + (r0 + tid) + lda * (long)(r0 + t))));
                xs[tid] = make_double2(v.hi, v.lo);
            }
            __syncthreads();
        }
        xi = dd_make(xs[tid].x, xs[tid].y);
    }
    if (i < n) st_dd(x + i, xi);
}

// Backward solve with L^T, launch p (from the last block down): entries of
// blocks c <= p take block p+1's solution (t -= L(i,j) x(i), i descending);
// then CTA p finishes its block (j descending: x(j) = t(j) / L(j,j)).
__global__ void trsv_bwd_kernel(const dd_t *L, long lda, int n, dd_t *x, int p, int nblk) {
    __shared__ double2 xs[TRSV_B];
    const int c = blockIdx.x; // blocks 0..p
    const int r0 = c * TRSV_B, tid = threadIdx.x;
    const int j = r0 + tid;
    dd_t xj = dd_zero();
    if (j < n) xj = ld_dd(x + j);
    if (p + 1 < nblk) {
        const int i0 = (p + 1) * TRSV_B;
        const int ib = min(TRSV_B, n - i0);
        for (int t = tid; t < ib; t += blockDim.x) xs[t] = *reinterpret_cast<const double2 *>(x + i0 + t);
        __syncthreads();
        if (j < n)
            for (int t = ib - 1; t >= 0; --t) xj = dd_sub(xj, dd_mul(ld_dd(L + (i0 + t) + lda * (long)j), dd_make(xs[t].x, xs[t].y)));
        __syncthreads();
    }
    if (c == p) {
        const int nb = min(TRSV_B, n - r0);
        xs[tid] = make_double2(xj.hi, xj.lo);
        __syncthreads();
        for (int t = nb - 1; t >= 0; --t) {
            if (tid == t) {
                dd_t v = dd_div(dd_make(xs[t].x, xs[t].y), ld_dd(L + (r0 + t) + lda * (long)(r0 + t)));
                xs[t] = make_double2(v.hi, v.lo);
            }
            __syncthreads();
            if (tid < t) {
                dd_t v = dd_make(xs[tid].x, xs[tid].y);
                v = dd_sub(v, dd_mul(ld_dd(L + (r0 + t) + lda * (long)(r0 + tid)), dd_make(xs[t].x, xs[t].y)));
                xs[tid] = make_double2(v.hi, v.lo);
            }
            __syncthreads();
        }
        xj = dd_make(xs[tid].x, xs[tid].y);
    }
    if (j < n) st_dd(x + j, xj);
}

void trsv_lower(cudaStream_t st, char trans, const dd_t *L, long lda, int n, dd_t *x) {
    if (n <= 0) return;
    PROF_SCOPE("trsv", st);
    const int nblk = ceil_div(n, TRSV_B);
    if (trans == 'N') {
        for (int p = 0; p < nblk; ++p) {
            trsv_fwd_kernel<<<nblk - p, TRSV_B, 0, st>>>(L, lda, n, x, p);
            CK_LAUNCH();
        }
    } else {
        for (int p = nblk - 1; p >= 0; --p) {
            trsv_bwd_kernel<<<p + 1, TRSV_B, 0, st>>>(L, lda, n, x, p, nblk);
            CK_LAUNCH();
        }
    }
}

// ======================================================= triangular inverse
// X = inv(L): one CTA per column j, right-looking over k = j..n-1
// (Rtrsm "Left","Lower","N","N" on the identity).
__global__ void inv_lower_kernel(const dd_t *L, long lda, int n, dd_t *X, long ldx) {
    extern __shared__ double2 col[];
    const int j = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < n; i += nt) col[i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int k = j; k < n; ++k) {
        dd_t xk = dd_make(col[k].x, col[k].y);
        if (dd_is_zero(xk)) continue; // uniform across the CTA
        __syncthreads();
        if (tid == 0) {
            xk = dd_div(xk, ld_dd(L + k + lda * (long)k));
            col[k] = make_double2(xk.hi, xk.lo);
        }
        __syncthreads();
        xk = dd_make(col[k].x, col[k].y);
        for (int i = k + 1 + tid; i < n; i += nt) {
            dd_t v = dd_make(col[i].x, col[i].y);
            v = dd_sub(v, dd_mul(xk, ld_dd(L + i + lda * (long)k)));
            col[i] = make_double2(v.hi, v.lo);
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += nt) *reinterpret_cast<double2 *>(X + i + ldx * (long)j) = col[i];
}
void inv_lower(cudaStream_t st, const dd_t *L, long lda, int n, dd_t *X, long ldx) {
    if (n <= 0) return;
    const size_t smem = sizeof(double2) * n;
    if (smem > 227 * 1024) throw Error(ERR_UNSUPPORTED, "inv_lower: block too large for one CTA");
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(inv_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    inv_lower_kernel<<<n, 128, smem, st>>>(L, lda, n, X, ldx);
    CK_LAUNCH();
}

// B = M^T M for lower M, entry by entry as Rtrmm("L","L","T","N") does in
// place: t = M(i,j) M(i,i); t += M(k,i) M(k,j), k = i+1..n-1 (terms with
// M(k,j) = 0, k < j, add exact zeros and are skipped).
__global__ void trmm_lt_kernel(const dd_t *M, long ldm, int n, dd_t *B, long ldb) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    int i = e % n, j = e / n;
    dd_t t = dd_mul(ld_dd(M + i + ldm * (long)j), ld_dd(M + i + ldm * (long)i));
    for (int k = max(i + 1, j); k < n; ++k) t = dd_acc(t, dd_mul(ld_dd(M + k + ldm * (long)i), ld_dd(M + k + ldm * (long)j)));
    st_dd(B + i + ldb * (long)j, t);
}
void trmm_lt(cudaStream_t st, const dd_t *M, long ldm, int n, dd_t *B, long ldb) {
    if (n <= 0) return;
    trmm_lt_kernel<<<ceil_div((long)n * n, 128), 128, 0, st>>>(M, ldm, n, B, ldb);
    CK_LAUNCH();
}

// =============================================================== symmetrize
__global__ void symmetrize_kernel(dd_t *A, int n) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    int i = e % n, c = e / n;
    if (i <= c) return;
    dd_t v = dd_acc(ld_dd(A + i + (long)n * c), ld_dd(A + c + (long)n * i));
    v = dd_mul(dd_from(0.5), v);
    st_dd(A + i + (long)n * c, v);
    st_dd(A + c + (long)n * i, v);
}
void symmetrize(cudaStream_t st, dd_t *A, int n) {
    if (n <= 1) return;
    symmetrize_kernel<<<ceil_div((long)n * n, 256), 256, 0, st>>>(A, n);
    CK_LAUNCH();
}

// ================================================================ vector ops
__global__ void fill_kernel(dd_t *x, long n, dd_t v) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) st_dd(x + e, v);
}
void fill(cudaStream_t st, dd_t *x, long n, dd_t v) {
    if (n <= 0) return;
    fill_kernel<<<ceil_div(n, 256), 256, 0, st>>>(x, n, v);
    CK_LAUNCH();
}

// y = a * y (Rscal: da * dx)
__global__ void scal_kernel(dd_t *y, long n, dd_t a) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) st_dd(y + e, dd_mul(a, ld_dd(y + e)));
}
void scal(cudaStream_t st, dd_t *y, long n, dd_t a) {
    if (n <= 0) return;
    scal_kernel<<<ceil_div(n, 256), 256, 0, st>>>(y, n, a);
    CK_LAUNCH();
}

// y = x * a (Rcopy then Rscal)
__global__ void copy_scal_kernel(const dd_t *x, dd_t *y, long n, dd_t a) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) st_dd(y + e, dd_mul(a, ld_dd(x + e)));
}
void copy_scal(cudaStream_t st, const dd_t *x, dd_t *y, long n, dd_t a) {
    if (n <= 0) return;
    copy_scal_kernel<<<ceil_div(n, 256), 256, 0, st>>>(x, y, n, a);
    CK_LAUNCH();
}

// z = x; z += a * y (Rcopy then Raxpy; Raxpy returns early when a == 0)
__global__ void axpy_kernel(const dd_t *x, const dd_t *y, dd_t *z, long n, dd_t a) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) st_dd(z + e, dd_acc(ld_dd(x + e), dd_mul(a, ld_dd(y + e))));
}
void axpy(cudaStream_t st, const dd_t *x, const dd_t *y, dd_t *z, long n, dd_t a) {
    if (n <= 0) return;
    if (dd_is_zero(a)) {
        if (x != z) CK(cudaMemcpyAsync(z, x, sizeof(dd_t) * n, cudaMemcpyDeviceToDevice, st));
        return;
    }
    axpy_kernel<<<ceil_div(n, 256), 256, 0, st>>>(x, y, z, n, a);
    CK_LAUNCH();
}

// ================================================================ reductions
// Deterministic dd dot product.  Up to DOT_SEQ terms: one sequential chain,
// identical to Rdot with one OpenMP thread.  Longer: contiguous chunks summed
// sequentially, then a fixed pairwise tree (same result on every run).
constexpr int DOT_SEQ = 1024;
constexpr int DOT_THREADS = 256;

__global__ void dot_seq_kernel(const dd_t *x, long incx, const dd_t *y, long incy, long n, dd_t *out) {
    if (threadIdx.x != 0) return;
    dd_t t = dd_zero();
    for (long i = 0; i < n; ++i) t = dd_acc(t, dd_mul(ld_dd(x + i * incx), ld_dd(y + i * incy)));
    st_dd(out, dd_acc(dd_zero(), t));
}

__device__ dd_t block_tree(dd_t v, double2 *sh) {
    const int tid = threadIdx.x;
    sh[tid] = make_double2(v.hi, v.lo);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            dd_t a = dd_make(sh[tid].x, sh[tid].y), b = dd_make(sh[tid + s].x, sh[tid + s].y);
            dd_t r = dd_add(a, b);
            sh[tid] = make_double2(r.hi, r.lo);
        }
        __syncthreads();
    }
    return dd_make(sh[0].x, sh[0].y);
}

__global__ void dot_chunk_kernel(const dd_t *x, long incx, const dd_t *y, long incy, long n, dd_t *partial) {
    __shared__ double2 sh[DOT_THREADS];
    const long nthr = (long)gridDim.x * DOT_THREADS;
    const long g = blockIdx.x * (long)DOT_THREADS + threadIdx.x;
    const long q = n / nthr, r = n % nthr;
    const long lo = g * q + min(g, r), hi = lo + q + (g < r ? 1 : 0);
    dd_t t = dd_zero();
    for (long i = lo; i < hi; ++i) t = dd_acc(t, dd_mul(ld_dd(x + i * incx), ld_dd(y + i * incy)));
    dd_t s = block_tree(t, sh);
    if (threadIdx.x == 0) st_dd(partial + blockIdx.x, s);
}
__global__ void tree_final_kernel(const dd_t *partial, int np, dd_t *out) {
    __shared__ double2 sh[DOT_THREADS];
    dd_t v = threadIdx.x < np ? ld_dd(partial + threadIdx.x) : dd_zero();
    dd_t s = block_tree(v, sh);
    if (threadIdx.x == 0) st_dd(out, s);
}

void dot(cudaStream_t st, const dd_t *x, long incx, const dd_t *y, long incy, long n, dd_t *out, dd_t *scratch) {
    if (n <= DOT_SEQ) {
        dot_seq_kernel<<<1, 32, 0, st>>>(x, incx, y, incy, n, out);
        CK_LAUNCH();
        return;
    }
    int nb = (int)std::min<long>(DOT_THREADS, ceil_div(n, 16L * DOT_THREADS));
    dot_chunk_kernel<<<nb, DOT_THREADS, 0, st>>>(x, incx, y, incy, n, scratch);
    CK_LAUNCH();
    tree_final_kernel<<<1, DOT_THREADS, 0, st>>>(scratch, nb, out);
    CK_LAUNCH();
}

// max |x_i| (Residuals::computeMaxNorm) - exact in any order.
__global__ void maxabs_kernel(const dd_t *x, long n, dd_t *partial) {
    __shared__ double2 sh[DOT_THREADS];
    dd_t m = dd_zero();
    for (long i = blockIdx.x * (long)DOT_THREADS + threadIdx.x; i < n; i += (long)gridDim.x * DOT_THREADS) m = dd_max(m, dd_abs(ld_dd(x + i)));
    sh[threadIdx.x] = make_double2(m.hi, m.lo);
    __syncthreads();
    for (int s = DOT_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            dd_t a = dd_make(sh[threadIdx.x].x, sh[threadIdx.x].y), b = dd_make(sh[threadIdx.x + s].x, sh[threadIdx.x + s].y);
            dd_t r = dd_max(a, b);
            sh[threadIdx.x] = make_double2(r.hi, r.lo);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = dd_make(sh[0].x, sh[0].y);
}
__global__ void max_final_kernel(const dd_t *partial, int np, dd_t *out) {
    if (threadIdx.x != 0) return;
    dd_t m = dd_zero();
    for (int i = 0; i < np; ++i) m = dd_max(m, partial[i]);
    *out = m;
}
void maxabs(cudaStream_t st, const dd_t *x, long n, dd_t *out, dd_t *scratch) {
    int nb = (int)std::min<long>(DOT_THREADS, std::max(1u, ceil_div(n, 4L * DOT_THREADS)));
    maxabs_kernel<<<nb, DOT_THREADS, 0, st>>>(x, n, scratch);
    CK_LAUNCH();
    max_final_kernel<<<1, 32, 0, st>>>(scratch, nb, out);
    CK_LAUNCH();
}

} // namespace sddd
