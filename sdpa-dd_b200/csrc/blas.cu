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
#include "bulk.cuh"
#include "ozaki.h"
#include "prof.h"

#include <algorithm>

namespace sddd {

// ===================================================================== GEMM
// Tile: BM x BN outputs per CTA, BK-deep k slices staged in shared memory,
// TM x TN outputs per thread.  Shared tiles are k-major and padded by one
// element so that transposed tile loads do not collide on banks.
// MODE GEMM_AB_PRE (Rgemm_NN/NT_omp with alpha): each B value is multiplied
// by alpha as it is staged ("temp = alpha * B(l,j)"), then c += temp * a
// from the (beta-scaled) C; GEMM_AB_POST (Rgemm_TN/TT_omp): the products
// are summed from zero and C += alpha * sum.
template <int BM, int BN, int BK, int TM, int TN, bool TA, bool TB, int MODE>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    gemm_kernel(int M, int N, int K, const dd_t *__restrict__ A, long lda, long sA, const dd_t *__restrict__ B, long ldb, long sB, dd_t *C,
                long ldc, long sC, int lower, dd_t alpha) {
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
            if (MODE == GEMM_STORE || MODE == GEMM_AB_POST || gi >= M || gj >= N)
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
            if (MODE == GEMM_AB_PRE) {
                const dd_t t = dd_mul(alpha, dd_make(v.x, v.y));
                v = make_double2(t.hi, t.lo);
            }
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
            if (gi < M && gj < N && (!lower || gi >= gj)) {
                dd_t *cp = C + gi + ldc * (long)gj;
                st_dd(cp, MODE == GEMM_AB_POST ? dd_acc(ld_dd(cp), dd_mul(alpha, acc[r][c])) : acc[r][c]);
            }
        }
}

// 64 x 64 tiles (4 x 4 entries a thread) when they fill the GPU; for
// small products (fewer 64 x 64 tiles than half the SMs) 16 x 16 tiles
// with one entry a thread, so the work spreads over more SMs.  Each
// entry's k-order is the same either way.
constexpr long GEMM_SMALL_TILES = 74;
template <bool TA, bool TB, int MODE>
static void gemm_launch(cudaStream_t st, int M, int N, int K, const dd_t *A, long lda, long sA, const dd_t *B, long ldb, long sB, dd_t *C, long ldc,
                        long sC, int batch, bool lower, dd_t alpha = dd_t{1.0, 0.0}) {
    if ((long)ceil_div(N, 64) * ceil_div(M, 64) * batch < GEMM_SMALL_TILES) {
        constexpr int BM = 16, BN = 16, BK = 16, TM = 1, TN = 1;
        dim3 grid(ceil_div(N, BN), ceil_div(M, BM), batch);
        gemm_kernel<BM, BN, BK, TM, TN, TA, TB, MODE>
            <<<grid, (BM / TM) * (BN / TN), 0, st>>>(M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, lower ? 1 : 0, alpha);
        CK_LAUNCH();
        return;
    }
    constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4;
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM), batch);
    gemm_kernel<BM, BN, BK, TM, TN, TA, TB, MODE>
        <<<grid, (BM / TM) * (BN / TN), 0, st>>>(M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, lower ? 1 : 0, alpha);
    CK_LAUNCH();
}

// C = beta C as Rgemm's first loop: zero for beta == 0, unchanged for
// beta == 1, else beta * C(i,j).
__global__ void gemm_beta_kernel(dd_t *C, long ldc, int M, int N, dd_t beta) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)M * N) return;
    dd_t *cp = C + e % M + ldc * (e / M);
    st_dd(cp, (beta.hi == 0.0 && beta.lo == 0.0) ? dd_zero() : dd_mul(beta, ld_dd(cp)));
}

void gemm_ab(cudaStream_t st, char ta, char tb, int M, int N, int K, dd_t alpha, const dd_t *A, long lda, const dd_t *B, long ldb, dd_t beta, dd_t *C,
             long ldc) {
    const bool one_beta = beta.hi == 1.0 && beta.lo == 0.0;
    const bool zero_alpha = alpha.hi == 0.0 && alpha.lo == 0.0;
    if (M <= 0 || N <= 0 || ((zero_alpha || K <= 0) && one_beta)) return; // Rgemm's quick return
    if (!one_beta) {
        gemm_beta_kernel<<<ceil_div((long)M * N, 256), 256, 0, st>>>(C, ldc, M, N, beta);
        CK_LAUNCH();
    }
    if (zero_alpha || K <= 0) return;
    const bool a = ta == 'T', b = tb == 'T';
    if (!a && !b) gemm_launch<false, false, GEMM_AB_PRE>(st, M, N, K, A, lda, 0, B, ldb, 0, C, ldc, 0, 1, false, alpha);
    else if (!a && b) gemm_launch<false, true, GEMM_AB_PRE>(st, M, N, K, A, lda, 0, B, ldb, 0, C, ldc, 0, 1, false, alpha);
    else if (a && !b) gemm_launch<true, false, GEMM_AB_POST>(st, M, N, K, A, lda, 0, B, ldb, 0, C, ldc, 0, 1, false, alpha);
    else gemm_launch<true, true, GEMM_AB_POST>(st, M, N, K, A, lda, 0, B, ldb, 0, C, ldc, 0, 1, false, alpha);
}

void gemm(cudaStream_t st, char ta, char tb, int mode, int M, int N, int K, const dd_t *A, long lda, long sA, const dd_t *B, long ldb, long sB,
          dd_t *C, long ldc, long sC, int batch, bool lower) {
    if (M <= 0 || N <= 0 || batch <= 0) return;
    if (K <= 0 && mode == GEMM_SUB) return;
    if (batch > MAX_GRID_YZ) {
        // grid.z holds at most 65535 matrices per launch
        for (int b0 = 0; b0 < batch; b0 += MAX_GRID_YZ)
            gemm(st, ta, tb, mode, M, N, K, A + b0 * sA, lda, sA, B + b0 * sB, ldb, sB, C + b0 * sC, ldc, sC, std::min(MAX_GRID_YZ, batch - b0), lower);
        return;
    }
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
// Diagonal block: right-looking dd Cholesky of an nb x nb block, nb <= 64.
// On a non-positive or NaN pivot the 1-based global column goes to *info
// and the block is left as it was (Rpotrf2's n = 1 test,
// mplapack/Rpotrf2.cpp).  1/L(j,j) for the panel goes to rdiag.
// Dataflow form, with no CTA-wide barrier between columns: warp w owns
// columns w and w + 32 in registers (lane l holds rows j + l and j + l + 32
// of column j).  When column k is final (pivot, scaling) its owner copies
// it to shared memory and its 32 lanes arrive on column k's mbarrier;
// every warp waits for that barrier, then subtracts column k's term from
// its own columns right of k, the owner of column k + 1 taking that column
// first and finishing it at once, so that one pivot follows the next
// through a single warp.  Every entry sees the same operations in the same
// order as the column-by-column form: x(i,j) -= L(j,k) L(i,k) for k
// ascending, then the sqrt (diagonal) or the scaling by 1/L(j,j).
constexpr int DIAG_THREADS = 1024;
constexpr unsigned long long POTRF_WAIT_NS = 2000000000ull; // one mbarrier wait, at most
static_assert(POTRF_NB <= 64 && DIAG_THREADS == 1024, "two columns a warp, two rows a lane");
// Bounded wait for phase 0 of an mbarrier.
__device__ __forceinline__ bool bar_wait0(uint64_t *b) {
    if (mbar_try_wait(b, 0)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(b, 0))
        if (globaltimer_ns() - t0 > POTRF_WAIT_NS) return false;
    return true;
}
__global__ void __launch_bounds__(DIAG_THREADS) potrf_diag_kernel(dd_t *A, long lda, int nb, int c0, int *info, dd_t *rdiag, long sA) {
    extern __shared__ double2 sm[];
    double2 *S = sm; // nb x nb, column-major: the final columns
    __shared__ uint64_t bar[POTRF_NB];
    __shared__ int fail;
    A += blockIdx.x * sA; // CTA b: matrix b of a batch of equal blocks (rdiag null then)
    if (*info != 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < nb) mbar_init(&bar[tid], 32);
    if (tid == 0) fail = 0;
    __syncthreads();
    volatile int *vfail = &fail;
    dd_t x[2][2];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int j = warp + 32 * c, i = j + lane + 32 * r;
            x[c][r] = (j < nb && i < nb) ? ld_dd(A + (c0 + i) + lda * (long)(c0 + j)) : dd_from(0.0);
        }
    // Column warp + 32 c: pivot (lane 0 holds the diagonal), scaling, copy
    // to shared memory, arrival.  False when the pivot fails.
    auto finish = [&](const int c) -> bool {
        const int j = warp + 32 * c;
        int bad = 0;
        double rh = 0.0, rl = 0.0;
        if (lane == 0) {
            const dd_t d = x[c][0];
            if (dd_le_d(d, 0.0) || dd_isnan(d)) {
                bad = 1;
                *vfail = 1;
                *info = c0 + j + 1;
            } else {
                const dd_t l = dd_sqrt(d);
                x[c][0] = l;
                const dd_t r = dd_div(dd_from(1.0), l);
                if (rdiag) rdiag[j] = r;
                rh = r.hi;
                rl = r.lo;
            }
        }
        bad = __shfl_sync(0xffffffffu, bad, 0);
        if (!bad) {
            const dd_t r = dd_make(__shfl_sync(0xffffffffu, rh, 0), __shfl_sync(0xffffffffu, rl, 0));
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int i = j + lane + 32 * q;
                if (i < nb) {
                    if (i > j) x[c][q] = dd_mul(r, x[c][q]);
                    S[i + nb * j] = make_double2(x[c][q].hi, x[c][q].lo);
                }
            }
        }
        mbar_arrive(&bar[j]);
        return !bad;
    };
    // column warp + 32 c takes column k's term
    auto update = [&](const int c, const int k) {
        const int j = warp + 32 * c;
        const double2 l = S[j + nb * k];
        const dd_t ljk = dd_make(l.x, l.y);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int i = j + lane + 32 * q;
            if (i < nb) {
                const double2 v = S[i + nb * k];
                x[c][q] = dd_sub(x[c][q], dd_mul(ljk, dd_make(v.x, v.y)));
            }
        }
    };
    const bool two = warp + 32 < nb;
    const int last = two ? warp + 32 : (warp < nb ? warp : -1); // the warp's last column
    bool ok = true;
    if (warp == 0 && nb > 0) ok = finish(0);
    for (int k = 0; ok && k < last; ++k) {
        // warp-uniform outcomes: the lanes go on together or stop together
        if (!__all_sync(0xffffffffu, bar_wait0(&bar[k]))) {
            if (lane == 0) {
                *vfail = 2;
                atomicCAS(info, 0, -1);
            }
            break;
        }
        if (__any_sync(0xffffffffu, *vfail != 0)) break;
        if (((k + 1) & 31) == warp) {
            // this warp owns column k + 1
            if (k + 1 < 32) {
                update(0, k);
                ok = finish(0);
                if (ok && two) update(1, k);
            } else {
                update(1, k);
                ok = finish(1);
            }
        } else {
            if (warp > k) update(0, k);
            if (two) update(1, k);
        }
    }
    __syncthreads();
    if (*vfail) return;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int j = warp + 32 * c, i = j + lane + 32 * r;
            if (j < nb && i < nb) st_dd(A + (c0 + i) + lda * (long)(c0 + j), x[c][r]);
        }
}

// Panel rows below the diagonal block (Rtrsm "Right", "Lower", "Transpose":
// x(i,j) -= L(j,k) x(i,k) for k < j ascending, then x(i,j) *= 1/L(j,j)).
// Rows are independent, so a warp solves PANEL_WROWS rows by itself, with
// no barrier: lane = (column class c, row r), c = lane / PANEL_WROWS, and
// the lane holds the row's columns c, c + PANEL_CLASSES, ... in registers.
// At step k the holder of x(r,k) passes it to the row's other lanes by
// shuffle; every lane subtracts the step's term from its columns right of
// k, and the holder of column k + 1 then scales it (the entry is final).
// Rounds of PANEL_CLASSES steps: in round q, slot s holds column
// c + PANEL_CLASSES (q + s) (the slots rotate by one between rounds, and the
// column leaving slot 0 is final and goes back to memory); the rounds are
// unrolled so that each one updates exactly its live slots, without
// branches between the slots' independent chains.  L11 (lower triangle,
// packed by columns, one bulk copy per column) and the reciprocals are
// shared by the CTA's warps.  The panel is POTRF_NB columns wide.
constexpr int PANEL_CLASSES = 16;                           // lanes a row
constexpr int PANEL_WROWS = 32 / PANEL_CLASSES;             // rows a warp
constexpr int PANEL_SLOTS = POTRF_NB / PANEL_CLASSES;       // columns a lane
constexpr int PANEL_THREADS = 128;
constexpr int PANEL_ROWS = PANEL_WROWS * (PANEL_THREADS / 32); // rows a CTA
static_assert(POTRF_NB % PANEL_CLASSES == 0 && 32 % PANEL_CLASSES == 0, "panel lane map");
constexpr size_t PANEL_SMEM = sizeof(double2) * (POTRF_NB * (POTRF_NB + 1) / 2 + POTRF_NB);
// first entry of column k (rows k .. POTRF_NB-1) of a lower triangle packed
// by columns
__device__ __forceinline__ int col_off(int k) { return k * POTRF_NB - k * (k - 1) / 2; }
__global__ void __launch_bounds__(PANEL_THREADS) potrf_panel_kernel(dd_t *A, long lda, int n, int c0, int *info, const dd_t *rdiag) {
    constexpr int NB = POTRF_NB, C = PANEL_CLASSES, W = PANEL_WROWS, NS = PANEL_SLOTS;
    extern __shared__ __align__(16) double2 sm[];
    double2 *L11 = sm;                   // lower triangle of NB x NB, packed by columns
    double2 *R = sm + NB * (NB + 1) / 2; // NB reciprocals
    __shared__ uint64_t lbar;
    __shared__ int lfail;
    if (*info != 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(&lbar, 1);
        mbar_init_fence();
        lfail = 0;
    }
    __syncthreads();
    if (warp == 0) {
        // column k of L11 (rows k .. NB-1) is contiguous in A: one bulk copy
        if (lane == 0) mbar_expect_tx(&lbar, (uint32_t)(sizeof(double2) * NB * (NB + 1) / 2));
        __syncwarp();
        for (int k = lane; k < NB; k += 32)
            bulk_g2s(L11 + col_off(k), A + (c0 + k) + lda * (long)(c0 + k), (uint32_t)(sizeof(double2) * (NB - k)), &lbar);
    }
    for (int e = tid; e < NB; e += PANEL_THREADS) R[e] = make_double2(rdiag[e].hi, rdiag[e].lo);
    const int cls = lane / W, row = lane % W;
    const long gi = (long)c0 + NB + (long)blockIdx.x * PANEL_ROWS + warp * W + row;
    const bool live = gi < n;
    dd_t *arow = A + gi + lda * (long)c0; // the row's panel entries, stride lda
    dd_t x[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) x[s] = live ? ld_dd(arow + lda * (long)(cls + C * s)) : dd_from(0.0);
    if (tid == 0 && !bar_wait0(&lbar)) {
        // the copies did not land in time: report, let them land (bounded)
        lfail = 1;
        atomicCAS(info, 0, -1);
        bar_wait0(&lbar);
    }
    __syncthreads();
    if (lfail) return;
    auto rk = [&](int k) { return dd_make(R[k].x, R[k].y); };
    if (cls == 0) x[0] = dd_mul(rk(0), x[0]); // column 0: scaling only
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        // step k = C q + t; slot s holds column cls + C (q + s), s < NS - q
#pragma unroll 1
        for (int t = 0; t < C; ++t) {
            const int k = C * q + t;
            if (k + 1 >= NB) break;
            const dd_t xk = dd_make(__shfl_sync(0xffffffffu, x[0].hi, t * W + row), __shfl_sync(0xffffffffu, x[0].lo, t * W + row));
            const double2 *lk = L11 + col_off(k) - k; // L(j, k) at lk[j]
            dd_t y[NS];
#pragma unroll
            for (int s = 0; s < NS - q; ++s) {
                const int j = cls + C * (q + s);
                const double2 l = lk[j];
                y[s] = dd_sub(x[s], dd_mul(dd_make(l.x, l.y), xk));
            }
            // slot 0's column lies right of k only for classes above t
            x[0] = cls > t ? y[0] : x[0];
#pragma unroll
            for (int s = 1; s < NS - q; ++s) x[s] = y[s];
            // column k + 1 is final after its scaling: class t + 1 in slot 0,
            // or class 0 in slot 1 at the round's last step
            if (t + 1 < C) {
                if (cls == t + 1) x[0] = dd_mul(rk(k + 1), x[0]);
            } else if (q + 1 < NS) {
                if (cls == 0) x[1] = dd_mul(rk(k + 1), x[1]);
            }
        }
        // column cls + C q is final
        if (live) st_dd(arow + lda * (long)(cls + C * q), x[0]);
#pragma unroll
        for (int s = 0; s + 1 < NS - q; ++s) x[s] = x[s + 1];
    }
}

// The next diagonal block's update by the panel just solved, ahead of the
// trailing update (the split form's lookahead): D(i, j) -= P(j, k) P(i, k)
// for k ascending, i >= j; CTA j takes column j, thread i row i.  D is the
// nb x nb block at c0, P its rows of the nbp panel columns before c0,
// staged in shared memory first (one bulk copy per panel column: its nb
// rows are contiguous) so that the chain of each entry reads no global
// memory.
__global__ void potrf_diag_pre_kernel(dd_t *A, long lda, int c0, int nb, int nbp, int *info) {
    extern __shared__ __align__(16) double2 pre_sp[]; // pre_sp[k * blockDim.x + r] = P(r, k)
    __shared__ uint64_t pbar;
    __shared__ int pfail;
    if (*info != 0) return;
    const int j = blockIdx.x, i = threadIdx.x, w = blockDim.x;
    const dd_t *P = A + c0 + lda * (long)(c0 - nbp);
    if (i == 0) {
        mbar_init(&pbar, 1);
        mbar_init_fence();
        pfail = 0;
    }
    __syncthreads();
    if (i < 32) {
        if (i == 0) mbar_expect_tx(&pbar, (uint32_t)(sizeof(double2) * nb * nbp));
        __syncwarp();
        for (int k = i; k < nbp; k += 32) bulk_g2s(pre_sp + k * w, P + lda * (long)k, (uint32_t)(sizeof(double2) * nb), &pbar);
    }
    if (i == 0 && !bar_wait0(&pbar)) {
        // the copies did not land in time: report, let them land (bounded)
        pfail = 1;
        atomicCAS(info, 0, -1);
        bar_wait0(&pbar);
    }
    __syncthreads();
    if (pfail || i < j || i >= nb) return;
    dd_t *d = A + (c0 + i) + lda * (long)(c0 + j);
    dd_t x = ld_dd(d);
    for (int k = 0; k < nbp; ++k) {
        const double2 pj = pre_sp[k * w + j], pi = pre_sp[k * w + i];
        x = dd_sub(x, dd_mul(dd_make(pj.x, pj.y), dd_make(pi.x, pi.y)));
    }
    st_dd(d, x);
}

// Right-looking blocked Cholesky: per panel of POTRF_NB columns, factor the
// diagonal block, solve the rows below, then subtract the panel's outer
// product from the trailing lower triangle (GEMM_SUB keeps each entry's
// k-order).  info is a device int; 0 on success, else the failing column.
void potrf(cudaStream_t st, dd_t *A, long lda, int n, int *info_dev, dd_t *rdiag_dev, OzakiWork *tc) {
    if (n <= 0) return;
    static thread_local bool attr[64] = {};
    const int nbmax = POTRF_NB;
    const size_t smem_diag = sizeof(double2) * nbmax * nbmax;
    const size_t smem_panel = PANEL_SMEM;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (!attr[dev & 63]) {
        CK(cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_diag));
        CK(cudaFuncSetAttribute(potrf_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_panel));
        CK(cudaFuncSetAttribute(potrf_diag_pre_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double2) * nbmax * nbmax)));
        attr[dev & 63] = true;
    }
    if (tc && tc->side && n > 2 * nbmax) {
        // Split form with one block of lookahead: after panel k, the next
        // diagonal block takes panel k's update in dd (a small kernel) and
        // is factored on the side stream, on an SM the trailing update
        // leaves free, while the trailing update of panel k (all but that
        // block) runs; panel k+1 waits for both.
        {
            PROF_SCOPE("potrf_diag", st);
            potrf_diag_kernel<<<1, DIAG_THREADS, sizeof(double2) * nbmax * nbmax, st>>>(A, lda, nbmax, 0, info_dev, rdiag_dev, 0);
            CK_LAUNCH();
        }
        for (int c0 = 0;; c0 += nbmax) {
            const int nb = std::min(nbmax, n - c0);
            const int below = n - c0 - nb;
            if (below <= 0) break;
            {
                PROF_SCOPE("potrf_panel", st);
                potrf_panel_kernel<<<ceil_div(below, PANEL_ROWS), PANEL_THREADS, PANEL_SMEM, st>>>(A, lda, n, c0, info_dev, rdiag_dev);
                CK_LAUNCH();
            }
            const int c1 = c0 + nb, nb1 = std::min(nbmax, n - c1);
            {
                PROF_SCOPE("potrf_diag_pre", st);
                potrf_diag_pre_kernel<<<nb1, nbmax, sizeof(double2) * nbmax * nb, st>>>(A, lda, c1, nb1, nb, info_dev);
                CK_LAUNCH();
            }
            CK(cudaEventRecord(tc->ev_pre, st));
            CK(cudaStreamWaitEvent(tc->side, tc->ev_pre, 0));
            {
                PROF_SCOPE("potrf_diag", tc->side);
                potrf_diag_kernel<<<1, DIAG_THREADS, sizeof(double2) * nb1 * nb1, tc->side>>>(A, lda, nb1, c1, info_dev, rdiag_dev, 0);
                CK_LAUNCH();
            }
            CK(cudaEventRecord(tc->ev_diag, tc->side));
            if (below > nb1) {
                PROF_SCOPE("potrf_trailing_update_tc", st);
                ozaki_syrk_sub_lower(st, A + c1 + lda * (long)c0, lda, below, nb, A + c1 + lda * (long)c1, lda, *tc, nb1, 1);
            }
            CK(cudaStreamWaitEvent(st, tc->ev_diag, 0));
        }
        return;
    }
    for (int c0 = 0; c0 < n; c0 += nbmax) {
        const int nb = std::min(nbmax, n - c0);
        {
            PROF_SCOPE("potrf_diag", st);
            potrf_diag_kernel<<<1, DIAG_THREADS, sizeof(double2) * nb * nb, st>>>(A, lda, nb, c0, info_dev, rdiag_dev, 0);
            CK_LAUNCH();
        }
        const int below = n - c0 - nb;
        if (below <= 0) break;
        {
            PROF_SCOPE("potrf_panel", st);
            potrf_panel_kernel<<<ceil_div(below, PANEL_ROWS), PANEL_THREADS, PANEL_SMEM, st>>>(A, lda, n, c0, info_dev, rdiag_dev);
            CK_LAUNCH();
        }
        dd_t *panel = A + (c0 + nb) + lda * (long)c0;
        dd_t *trail = A + (c0 + nb) + lda * (long)(c0 + nb);
        if (tc) {
            PROF_SCOPE("potrf_trailing_update_tc", st);
            ozaki_syrk_sub_lower(st, panel, lda, below, nb, trail, lda, *tc);
        } else {
            PROF_SCOPE("potrf_trailing_update", st);
            gemm(st, 'N', 'T', GEMM_SUB, below, below, nb, panel, lda, 0, panel, lda, 0, trail, lda, 0, 1, true);
        }
    }
}

int potrf_info_check(int info) {
    if (info < 0) throw Error(ERR_CUDA, "potrf: a diagonal block's wait for one of its columns ran out");
    return info;
}

void potrf_batched(cudaStream_t st, dd_t *A, long lda, int n, long sA, int batch, int *info_dev) {
    if (n <= 0 || batch <= 0) return;
    if (n > POTRF_NB) throw Error(ERR_ARG, "potrf_batched: order above one diagonal block");
    const size_t smem = sizeof(double2) * n * n;
    CK(cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double2) * POTRF_NB * POTRF_NB)));
    potrf_diag_kernel<<<batch, DIAG_THREADS, smem, st>>>(A, lda, n, 0, info_dev, nullptr, sA);
    CK_LAUNCH();
}

// Zero the strict upper triangle (Lal::getCholesky, sdpa_linear.cpp:320-343).
__global__ void zero_upper_kernel(dd_t *A, long lda, int n, long sA) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    A += blockIdx.y * sA;
    int i = e % n, j = e / n;
    if (i < j) st_dd(A + i + lda * (long)j, dd_zero());
}
void zero_upper(cudaStream_t st, dd_t *A, long lda, int n, int batch, long sA) {
    if (n <= 0 || batch <= 0) return;
    if (batch > MAX_GRID_YZ) {
        for (int b0 = 0; b0 < batch; b0 += MAX_GRID_YZ) zero_upper(st, A + b0 * sA, lda, n, std::min(MAX_GRID_YZ, batch - b0), sA);
        return;
    }
    zero_upper_kernel<<<dim3(ceil_div((long)n * n, 256), batch), 256, 0, st>>>(A, lda, n, sA);
    CK_LAUNCH();
}

// ===================================================================== TRSV
// One cooperative launch per solve.  The matrix is cut into 64 x 64 tiles;
// CTA b owns the 64-entry blocks c = b, b + G, ... of x (forward) or the
// mirror order from the last block down (backward) and publishes each
// finished block through a per-block flag that holds the solve's epoch.
// Each entry keeps the reference's own chain (mplapack/Rtrsv.cpp, the
// reference BLAS loop order):
//   "N": x(i) -= x(j) L(i,j) for j ascending (skipped when x(j) == 0),
//        then x(i) /= L(i,i) when x(i) != 0;
//   "T": t = x(j); t -= L(i,j) x(i) for i descending; x(j) = t / L(j,j).
// Warp 0 holds the 64 entries of the current block, two per lane, and runs
// the chains; the other warps stage the next tile of L in shared memory
// (padded leading dimension 65: conflict-free for rows and columns).
// A CTA waits for a block with an acquire load bounded by the solve's wait
// budget (2 s by default); on expiry it records the block in the error word
// and returns.  Tests of that path name a block whose flag is withheld.
constexpr int TRSV_B = 64;
constexpr int TRSV_LD = 65;
constexpr int TRSV_THREADS = 256;
constexpr int TRSV_ONE_CTA = 8; // solves of at most 8 blocks (512 entries) run in one CTA
constexpr size_t TRSV_SMEM = 2 * sizeof(double2) * TRSV_B * TRSV_LD + sizeof(double2) * TRSV_B;

struct TrsvArgs {
    const dd_t *L;
    long lda;
    int n, nblk, epoch;
    dd_t *x;
    int *flags, *err;
    unsigned long long wait_ns;
    int withhold; // a block whose flag is never published (-1: none)
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v) { asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Lane 0 of the calling warp waits until flags[blk] == epoch; every lane
// returns the outcome.
__device__ bool trsv_wait(const TrsvArgs &a, int blk) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long t0 = global_ns();
        unsigned iter = 0;
        while (ld_acquire_gpu(a.flags + blk) != a.epoch) {
            if (ld_acquire_gpu(a.err) != 0 || ++iter > (1u << 26) || global_ns() - t0 > a.wait_ns) {
                atomicCAS(a.err, 0, blk + 1);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
    }
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// T(i, j) = L(r0 + i, c0 + j) for i, j < 64 (zero outside the matrix).
// Every thread of [t0, t0 + nt) puts all its 16-byte copies in flight at
// once (cp.async; a source size of 0 writes zeros) and waits for them, so a
// tile costs one memory latency rather than one per element; the caller's
// __syncthreads then publishes the tile.
__device__ __forceinline__ void trsv_load_tile(double2 *T, const TrsvArgs &a, int r0, int c0, int t0, int nt) {
    for (int e = t0; e < TRSV_B * TRSV_B; e += nt) {
        const int i = e % TRSV_B, j = e / TRSV_B;
        const int gi = r0 + i, gj = c0 + j;
        const bool in = gi < a.n && gj < a.n;
        const dd_t *src = in ? a.L + gi + a.lda * (long)gj : a.L;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(T + i + TRSV_LD * j)), "l"(src),
                     "r"(in ? 16 : 0)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ dd_t tile_dd(const double2 *T, int i, int j) {
    const double2 v = T[i + TRSV_LD * j];
    return dd_make(v.x, v.y);
}
__device__ __forceinline__ dd_t ldcg_dd(const dd_t *p) {
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return dd_make(v.x, v.y);
}
__device__ __forceinline__ dd_t shfl_dd(dd_t v, int src) {
    return dd_make(__shfl_sync(0xffffffffu, v.hi, src), __shfl_sync(0xffffffffu, v.lo, src));
}

__global__ void __launch_bounds__(TRSV_THREADS) trsv_fwd_wave_kernel(TrsvArgs a) {
    extern __shared__ double2 trsv_sm[];
    double2 *xs = trsv_sm + 2 * TRSV_B * TRSV_LD;
    __shared__ int fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    for (int c = blockIdx.x; c < a.nblk; c += gridDim.x) {
        const int r0 = c * TRSV_B;
        const int i0 = r0 + lane, i1 = r0 + 32 + lane;
        dd_t v0 = dd_zero(), v1 = dd_zero();
        if (warp == 0) {
            if (i0 < a.n) v0 = ld_dd(a.x + i0);
            if (i1 < a.n) v1 = ld_dd(a.x + i1);
        }
        trsv_load_tile(trsv_sm, a, r0, 0, tid, blockDim.x);
        __syncthreads();
        for (int p = 0; p < c; ++p) {
            const double2 *T = trsv_sm + (p & 1) * TRSV_B * TRSV_LD;
            if (warp != 0) {
                trsv_load_tile(trsv_sm + ((p + 1) & 1) * TRSV_B * TRSV_LD, a, r0, (p + 1) * TRSV_B, tid - 32, blockDim.x - 32);
            } else if (!trsv_wait(a, p)) {
                if (lane == 0) fail = 1;
            } else {
                // block p is complete (p < c): 64 entries
                const dd_t xa = ldcg_dd(a.x + p * TRSV_B + lane), xb = ldcg_dd(a.x + p * TRSV_B + 32 + lane);
                xs[lane] = make_double2(xa.hi, xa.lo);
                xs[32 + lane] = make_double2(xb.hi, xb.lo);
                __syncwarp();
                for (int t = 0; t < TRSV_B; ++t) {
                    const dd_t xt = dd_make(xs[t].x, xs[t].y);
                    if (!dd_is_zero(xt)) {
                        v0 = dd_sub(v0, dd_mul(xt, tile_dd(T, lane, t)));
                        v1 = dd_sub(v1, dd_mul(xt, tile_dd(T, 32 + lane, t)));
                    }
                }
                __syncwarp();
            }
            __syncthreads();
            if (fail) return;
        }
        if (warp == 0) {
            // diagonal tile (p == c)
            const double2 *T = trsv_sm + (c & 1) * TRSV_B * TRSV_LD;
            const int nb = min(TRSV_B, a.n - r0);
            for (int t = 0; t < nb; ++t) {
                const int owner = t & 31;
                dd_t mine = t < 32 ? v0 : v1;
                if (lane == owner && !dd_is_zero(mine)) mine = dd_div(mine, tile_dd(T, t, t));
                if (lane == owner) {
                    if (t < 32) v0 = mine;
                    else v1 = mine;
                }
                const dd_t xt = shfl_dd(mine, owner);
                if (!dd_is_zero(xt)) {
                    if (lane > t && lane < nb) v0 = dd_sub(v0, dd_mul(xt, tile_dd(T, lane, t)));
                    if (32 + lane > t && 32 + lane < nb) v1 = dd_sub(v1, dd_mul(xt, tile_dd(T, 32 + lane, t)));
                }
            }
            if (i0 < a.n) st_dd(a.x + i0, v0);
            if (i1 < a.n) st_dd(a.x + i1, v1);
            __threadfence();
            __syncwarp();
            if (lane == 0 && c != a.withhold) st_release_gpu(a.flags + c, a.epoch);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(TRSV_THREADS) trsv_bwd_wave_kernel(TrsvArgs a) {
    extern __shared__ double2 trsv_sm[];
    double2 *xs = trsv_sm + 2 * TRSV_B * TRSV_LD;
    __shared__ int fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    for (int k = blockIdx.x; k < a.nblk; k += gridDim.x) {
        const int c = a.nblk - 1 - k;
        const int r0 = c * TRSV_B;
        const int j0 = r0 + lane, j1 = r0 + 32 + lane;
        dd_t v0 = dd_zero(), v1 = dd_zero();
        if (warp == 0) {
            if (j0 < a.n) v0 = ld_dd(a.x + j0);
            if (j1 < a.n) v1 = ld_dd(a.x + j1);
        }
        // tiles T(i, j) = L(p*64 + i, r0 + j) for p = nblk-1 down to c
        trsv_load_tile(trsv_sm, a, (a.nblk - 1) * TRSV_B, r0, tid, blockDim.x);
        __syncthreads();
        int s = 0;
        for (int p = a.nblk - 1; p > c; --p, ++s) {
            const double2 *T = trsv_sm + (s & 1) * TRSV_B * TRSV_LD;
            if (warp != 0) {
                trsv_load_tile(trsv_sm + ((s + 1) & 1) * TRSV_B * TRSV_LD, a, (p - 1) * TRSV_B, r0, tid - 32, blockDim.x - 32);
            } else if (!trsv_wait(a, p)) {
                if (lane == 0) fail = 1;
            } else {
                const int ib = min(TRSV_B, a.n - p * TRSV_B);
                if (lane < ib) {
                    const dd_t xa = ldcg_dd(a.x + p * TRSV_B + lane);
                    xs[lane] = make_double2(xa.hi, xa.lo);
                }
                if (32 + lane < ib) {
                    const dd_t xb = ldcg_dd(a.x + p * TRSV_B + 32 + lane);
                    xs[32 + lane] = make_double2(xb.hi, xb.lo);
                }
                __syncwarp();
                for (int t = ib - 1; t >= 0; --t) {
                    const dd_t xt = dd_make(xs[t].x, xs[t].y);
                    v0 = dd_sub(v0, dd_mul(tile_dd(T, t, lane), xt));
                    v1 = dd_sub(v1, dd_mul(tile_dd(T, t, 32 + lane), xt));
                }
                __syncwarp();
            }
            __syncthreads();
            if (fail) return;
        }
        if (warp == 0) {
            const double2 *T = trsv_sm + (s & 1) * TRSV_B * TRSV_LD;
            const int nb = min(TRSV_B, a.n - r0);
            for (int t = nb - 1; t >= 0; --t) {
                const int owner = t & 31;
                dd_t mine = t < 32 ? v0 : v1;
                if (lane == owner) {
                    mine = dd_div(mine, tile_dd(T, t, t));
                    if (t < 32) v0 = mine;
                    else v1 = mine;
                }
                const dd_t xt = shfl_dd(mine, owner);
                if (lane < t) v0 = dd_sub(v0, dd_mul(tile_dd(T, t, lane), xt));
                if (32 + lane < t) v1 = dd_sub(v1, dd_mul(tile_dd(T, t, 32 + lane), xt));
            }
            if (j0 < a.n) st_dd(a.x + j0, v0);
            if (j1 < a.n) st_dd(a.x + j1, v1);
            __threadfence();
            __syncwarp();
            if (lane == 0 && c != a.withhold) st_release_gpu(a.flags + c, a.epoch);
        }
        __syncthreads();
    }
}

// Co-resident CTAs of a wave kernel on the current device.
static int trsv_grid_cap(const void *kernel) {
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRSV_SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, TRSV_THREADS, TRSV_SMEM));
    if (per < 1) throw Error(ERR_CUDA, "trsv: the wave kernel does not fit on an SM");
    return per * sms;
}

void trsv_lower(cudaStream_t st, char trans, const dd_t *L, long lda, int n, dd_t *x, TrsvSync &sync, bool shared_gpu) {
    if (n <= 0) return;
    if (trans != 'N' && trans != 'T') throw Error(ERR_ARG, "trsv: trans must be 'N' or 'T'");
    const int nblk = ceil_div(n, TRSV_B);
    if (nblk > sync.capacity || !sync.flags) throw Error(ERR_ARG, "trsv: progress flags hold fewer blocks than the solve needs");
    PROF_SCOPE("trsv", st);
    if (++sync.epoch <= 0) sync.epoch = 1;
    TrsvArgs a{L, lda, n, nblk, sync.epoch, x, sync.flags, sync.flags + sync.capacity, sync.wait_ns, sync.withhold};
    const void *k = trans == 'N' ? (const void *)trsv_fwd_wave_kernel : (const void *)trsv_bwd_wave_kernel;
    static thread_local int cap[2][64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &cp = cap[trans == 'N' ? 0 : 1][dev & 63];
    if (cp == 0) cp = trsv_grid_cap(k);
    const int grid = std::min(nblk, cp);
    if (shared_gpu && nblk <= TRSV_ONE_CTA) {
        // a short solve in one CTA, which walks the blocks in order and
        // never waits on another CTA: an ordinary launch, so it runs beside
        // other streams' work (a cooperative launch waits for room for its
        // whole grid); alone on the GPU the cooperative grid is faster
        if (trans == 'N')
            trsv_fwd_wave_kernel<<<1, TRSV_THREADS, TRSV_SMEM, st>>>(a);
        else
            trsv_bwd_wave_kernel<<<1, TRSV_THREADS, TRSV_SMEM, st>>>(a);
    } else {
        void *args[] = {&a};
        CK(cudaLaunchCooperativeKernel(k, grid, TRSV_THREADS, args, TRSV_SMEM, st));
    }
    CK_LAUNCH();
}

void trsv_check(cudaStream_t st, const TrsvSync &sync) {
    if (!sync.flags) return;
    int err = 0;
    int *h = sync.h_err ? sync.h_err : &err;
    CK(cudaMemcpyAsync(h, sync.flags + sync.capacity, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (sync.wait_ev) {
        CK(cudaEventRecord(sync.wait_ev, st));
        CK(cudaEventSynchronize(sync.wait_ev));
    } else {
        CK(cudaStreamSynchronize(st));
    }
    err = *h;
    if (err != 0) {
        // clear the error word, so that the next solve starts afresh
        CK(cudaMemsetAsync(sync.flags + sync.capacity, 0, sizeof(int), st));
        CK(cudaStreamSynchronize(st));
    }
    if (err != 0)
        throw Error(ERR_CUDA, "trsv: a wait ran out of its " + std::to_string(sync.wait_ns / 1000000ull) + " ms budget for block " + std::to_string(err - 1) +
                                  " (solve abandoned)");
}

// ======================================================= triangular inverse
// X = inv(L): one CTA per column j, right-looking over k = j..n-1
// (Rtrsm "Left","Lower","N","N" on the identity).
__global__ void inv_lower_kernel(const dd_t *L, long lda, int n, dd_t *X, long ldx, long sL, long sX) {
    extern __shared__ double2 col[];
    const int j = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    L += blockIdx.y * sL;
    X += blockIdx.y * sX;
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
// The same for n <= 2 blockDim: thread t holds rows t and t + blockDim; the
// L entries of step k+1 (its rows' L(i,k+1), and L(k+1,k+1) on thread 0)
// are loaded while step k runs, so no step waits on global memory.
constexpr int INV_THREADS = 128;
__global__ void __launch_bounds__(INV_THREADS) inv_lower_small_kernel(const dd_t *L, long lda, int n, dd_t *X, long ldx, long sL, long sX) {
    extern __shared__ double2 col[];
    const int j = blockIdx.x, tid = threadIdx.x;
    L += blockIdx.y * sL;
    X += blockIdx.y * sX;
    for (int i = tid; i < n; i += INV_THREADS) col[i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    auto lik_at = [&](int k, int r) {
        const int i = tid + INV_THREADS * r;
        return (i > k && i < n) ? ld_dd(L + i + lda * (long)k) : dd_zero();
    };
    dd_t lkk = tid == 0 ? ld_dd(L + j + lda * (long)j) : dd_zero();
    dd_t lik[2] = {lik_at(j, 0), lik_at(j, 1)};
    __syncthreads();
    for (int k = j; k < n; ++k) {
        const dd_t lkk_n = (tid == 0 && k + 1 < n) ? ld_dd(L + (k + 1) + lda * (long)(k + 1)) : dd_zero();
        const dd_t lik_n[2] = {lik_at(k + 1, 0), lik_at(k + 1, 1)};
        dd_t xk = dd_make(col[k].x, col[k].y);
        if (!dd_is_zero(xk)) { // uniform across the CTA
            if (tid == 0) {
                xk = dd_div(xk, lkk);
                col[k] = make_double2(xk.hi, xk.lo);
            }
            __syncthreads();
            xk = dd_make(col[k].x, col[k].y);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int i = tid + INV_THREADS * r;
                if (i > k && i < n) {
                    dd_t v = dd_make(col[i].x, col[i].y);
                    v = dd_sub(v, dd_mul(xk, lik[r]));
                    col[i] = make_double2(v.hi, v.lo);
                }
            }
            __syncthreads();
        }
        lkk = lkk_n;
        lik[0] = lik_n[0];
        lik[1] = lik_n[1];
    }
    for (int i = tid; i < n; i += INV_THREADS) *reinterpret_cast<double2 *>(X + i + ldx * (long)j) = col[i];
}

void inv_lower(cudaStream_t st, const dd_t *L, long lda, int n, dd_t *X, long ldx, int batch, long sL, long sX) {
    if (n <= 0 || batch <= 0) return;
    if (batch > MAX_GRID_YZ) {
        for (int b0 = 0; b0 < batch; b0 += MAX_GRID_YZ) inv_lower(st, L + b0 * sL, lda, n, X + b0 * sX, ldx, std::min(MAX_GRID_YZ, batch - b0), sL, sX);
        return;
    }
    const size_t smem = sizeof(double2) * n;
    if (smem > 227 * 1024) throw Error(ERR_UNSUPPORTED, "inv_lower: block too large for one CTA");
    if (n <= 2 * INV_THREADS) {
        inv_lower_small_kernel<<<dim3(n, batch), INV_THREADS, smem, st>>>(L, lda, n, X, ldx, sL, sX);
        CK_LAUNCH();
        return;
    }
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(inv_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    inv_lower_kernel<<<dim3(n, batch), 128, smem, st>>>(L, lda, n, X, ldx, sL, sX);
    CK_LAUNCH();
}

// B = M^T M for lower M, entry by entry as Rtrmm("L","L","T","N") does in
// place: t = M(i,j) M(i,i); t += M(k,i) M(k,j), k = i+1..n-1 (terms with
// M(k,j) = 0, k < j, add exact zeros and are skipped).
__global__ void trmm_lt_kernel(const dd_t *M, long ldm, int n, dd_t *B, long ldb, long sM, long sB) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    M += blockIdx.y * sM;
    B += blockIdx.y * sB;
    int i = e % n, j = e / n;
    dd_t t = dd_mul(ld_dd(M + i + ldm * (long)j), ld_dd(M + i + ldm * (long)i));
    for (int k = max(i + 1, j); k < n; ++k) t = dd_acc(t, dd_mul(ld_dd(M + k + ldm * (long)i), ld_dd(M + k + ldm * (long)j)));
    st_dd(B + i + ldb * (long)j, t);
}
void trmm_lt(cudaStream_t st, const dd_t *M, long ldm, int n, dd_t *B, long ldb, int batch, long sM, long sB) {
    if (n <= 0 || batch <= 0) return;
    if (batch > MAX_GRID_YZ) {
        for (int b0 = 0; b0 < batch; b0 += MAX_GRID_YZ) trmm_lt(st, M + b0 * sM, ldm, n, B + b0 * sB, ldb, std::min(MAX_GRID_YZ, batch - b0), sM, sB);
        return;
    }
    trmm_lt_kernel<<<dim3(ceil_div((long)n * n, 128), batch), 128, 0, st>>>(M, ldm, n, B, ldb, sM, sB);
    CK_LAUNCH();
}

// =============================================================== symmetrize
__global__ void symmetrize_kernel(dd_t *A, int n, long sA) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    A += blockIdx.y * sA;
    int i = e % n, c = e / n;
    if (i <= c) return;
    dd_t v = dd_acc(ld_dd(A + i + (long)n * c), ld_dd(A + c + (long)n * i));
    v = dd_mul(dd_from(0.5), v);
    st_dd(A + i + (long)n * c, v);
    st_dd(A + c + (long)n * i, v);
}
void symmetrize(cudaStream_t st, dd_t *A, int n, int batch, long sA) {
    if (n <= 1 || batch <= 0) return;
    if (batch > MAX_GRID_YZ) {
        for (int b0 = 0; b0 < batch; b0 += MAX_GRID_YZ) symmetrize(st, A + b0 * sA, n, std::min(MAX_GRID_YZ, batch - b0), sA);
        return;
    }
    symmetrize_kernel<<<dim3(ceil_div((long)n * n, 256), batch), 256, 0, st>>>(A, n, sA);
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

// Chains of a batch of equal-length dot products: CTA b, x + b sx, y + b
// sy, result out[b].
__global__ void dot_seq_batch_kernel(const dd_t *x, long sx, const dd_t *y, long sy, long n, dd_t *out) {
    if (threadIdx.x != 0) return;
    x += blockIdx.x * sx;
    y += blockIdx.x * sy;
    dd_t t = dd_zero();
    for (long i = 0; i < n; ++i) t = dd_acc(t, dd_mul(ld_dd(x + i), ld_dd(y + i)));
    st_dd(out + blockIdx.x, dd_acc(dd_zero(), t));
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

void dot_batched(cudaStream_t st, const dd_t *x, long sx, const dd_t *y, long sy, long n, int batch, dd_t *out, dd_t *scratch) {
    if (batch <= 0) return;
    if (n <= DOT_SEQ) {
        dot_seq_batch_kernel<<<batch, 32, 0, st>>>(x, sx, y, sy, n, out);
        CK_LAUNCH();
        return;
    }
    for (int b = 0; b < batch; ++b) dot(st, x + b * sx, 1, y + b * sy, 1, n, out + b, scratch + 256 * (b % 8));
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
