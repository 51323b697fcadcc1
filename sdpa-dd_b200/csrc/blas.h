// Host entry points of the dd dense kernels (blas.cu).  All pointers are
// device pointers; matrices are column-major dd with a leading dimension.
#pragma once
#include "common.cuh"

namespace sddd {

struct OzakiWork;

enum GemmMode { GEMM_STORE = 0, GEMM_SUB = 1, GEMM_ACC = 2, GEMM_AB_PRE = 3, GEMM_AB_POST = 4 };
constexpr int POTRF_NB = 64;
constexpr int MAX_GRID_YZ = 65535; // largest grid.y / grid.z of one launch

// C = op(A) op(B) (STORE: sum from zero; SUB: C - p_0 - p_1 - ...;
// ACC: C + p_0 + ...), batched with strides, optionally the lower triangle
// only.  op: 'N' or 'T'.
void gemm(cudaStream_t st, char ta, char tb, int mode, int M, int N, int K, const dd_t *A, long lda, long sA, const dd_t *B, long ldb, long sB,
          dd_t *C, long ldc, long sC, int batch, bool lower);
// In-place lower Cholesky; *info_dev = 0 or the failing 1-based column.
// rdiag_dev holds POTRF_NB dd of scratch.  With tc, the trailing updates
// run as tensor-core slice products (ozaki.h) instead of dd GEMMs.
// C = alpha op(A) op(B) + beta C with MPLAPACK Rgemm's operation order
// (mplapack/Rgemm_omp.cpp and Rgemm_{NN,NT,TN,TT}_omp.cpp): C is scaled by
// beta first (zeroed for beta == 0, untouched for beta == 1); then for
// 'N' A each C(i,j) takes c += (alpha B(l,j)) A(i,l) for l ascending, for
// 'T' A c += alpha (sum_l A(l,i) B(l,j)).  op: 'N' or 'T'.
void gemm_ab(cudaStream_t st, char ta, char tb, int M, int N, int K, dd_t alpha, const dd_t *A, long lda, const dd_t *B, long ldb, dd_t beta, dd_t *C,
             long ldc);
// *info_dev = -1: a diagonal block's wait for one of its columns ran out
// (the block is left as it was); potrf_info_check turns that into an error.
void potrf(cudaStream_t st, dd_t *A, long lda, int n, int *info_dev, dd_t *rdiag_dev, OzakiWork *tc = nullptr);
// Throws ERR_CUDA for a negative info (a wait that ran out); returns info.
int potrf_info_check(int info);
void zero_upper(cudaStream_t st, dd_t *A, long lda, int n, int batch = 1, long sA = 0);
// Rpotrf("Lower") of `batch` matrices of order n <= 64, matrix b at A + b sA,
// one CTA each (the single diagonal block of potrf); any failure sets
// *info_dev to a failing column.
void potrf_batched(cudaStream_t st, dd_t *A, long lda, int n, long sA, int batch, int *info_dev);
// Progress words of the one-launch triangular solve: one flag per 64-entry
// block (the epoch of the solve that finished it), then an error word.
// The owner zeroes them once; the epoch advances with every solve.
struct TrsvSync {
    int *flags = nullptr; // capacity flags + 1 error word
    int capacity = 0;
    int epoch = 0;
    int *h_err = nullptr; // pinned host word for reading the error word (or null)
    cudaEvent_t wait_ev = nullptr; // blocking-sync event to wait on (or null: stream sync)
    unsigned long long wait_ns = 2000000000ull; // budget of one wait for a block
    int withhold = -1; // tests of the bounded waits: this block's flag is never published
};
// x = L^-1 x ('N') or L^-T x ('T'), L lower, as Rtrsv("Lower", trans, "NonUnit").
// shared_gpu: other streams keep the GPU busy (a batch worker); short
// solves then run in one CTA with an ordinary launch.
void trsv_lower(cudaStream_t st, char trans, const dd_t *L, long lda, int n, dd_t *x, TrsvSync &sync, bool shared_gpu = false);
// Throws when a solve since the flags were zeroed gave up waiting
// (synchronises st).
void trsv_check(cudaStream_t st, const TrsvSync &sync);
// W_c = L(c,c)^-1 for the 64 x 64 diagonal blocks of L (order n): W holds
// ceil(n/64) blocks of 64 x 64 (leading dimension 64), zero above the
// diagonal.
void trsv_diag_inverse(cudaStream_t st, const dd_t *L, long lda, int n, dd_t *W);
// x = L^-1 x ('N') or L^-T x ('T') by blocks, with W from
// trsv_diag_inverse: one cooperative launch; the same progress words and
// error reporting (trsv_check) as trsv_lower.  Not Rtrsv's operation order.
void trsv_blocked(cudaStream_t st, char trans, const dd_t *L, long lda, int n, const dd_t *W, dd_t *x, TrsvSync &sync);
void inv_lower(cudaStream_t st, const dd_t *L, long lda, int n, dd_t *X, long ldx, int batch = 1, long sL = 0, long sX = 0);
void trmm_lt(cudaStream_t st, const dd_t *M, long ldm, int n, dd_t *B, long ldb, int batch = 1, long sM = 0, long sB = 0);
void symmetrize(cudaStream_t st, dd_t *A, int n, int batch = 1, long sA = 0);
void fill(cudaStream_t st, dd_t *x, long n, dd_t v);
void scal(cudaStream_t st, dd_t *y, long n, dd_t a);
void copy_scal(cudaStream_t st, const dd_t *x, dd_t *y, long n, dd_t a);
void axpy(cudaStream_t st, const dd_t *x, const dd_t *y, dd_t *z, long n, dd_t a);
// out = x.y (device scalar); scratch >= 256 dd
void dot(cudaStream_t st, const dd_t *x, long incx, const dd_t *y, long incy, long n, dd_t *out, dd_t *scratch);
// out[b] = dot(x + b sx, y + b sy) for b < batch (unit strides), each with
// dot's own order.
void dot_batched(cudaStream_t st, const dd_t *x, long sx, const dd_t *y, long sy, long n, int batch, dd_t *out, dd_t *scratch);
void maxabs(cudaStream_t st, const dd_t *x, long n, dd_t *out, dd_t *scratch);

} // namespace sddd
