// Tensor-core split of the Cholesky trailing update: C(lower) -= P P^T with
// dd operands cut into signed 7-bit integer slices (an Ozaki-style
// error-free split) and multiplied on the INT8 tensor cores (tcgen05,
// kind::i8) with exact int32 accumulation, then rebuilt in dd.
#pragma once
#include "common.cuh"

namespace sddd {

constexpr int OZ_MAX_SLICES = 16;
constexpr int OZ_K = 64;        // panel width the split handles (K of the update)
constexpr int OZ_ROWS_A = 128;  // output tile rows (MMA M)
constexpr int OZ_COLS_B = 16;   // output tile columns (per B slice)

// Device workspace of the split: slices for `row_cap` rows (a multiple of
// 128), row exponents and an error word.
struct OzakiWork {
    int8_t *slices = nullptr; // OZ_MAX_SLICES x row_cap x 64 bytes, tiled, slice by slice
    int8_t *slices_b = nullptr; // the same digits by 16-row block: each block's slices contiguous
    int *exps = nullptr;      // row_cap
    int *err = nullptr;       // 0, or the code of a wait that gave up
    int *h_err = nullptr;     // pinned host word for reading err (or null)
    cudaEvent_t wait_ev = nullptr; // blocking-sync event to wait on (or null: stream sync)
    int row_cap = 0;
    int slices_used = 16;     // 7-bit slices per value (8..16)
    unsigned long long wait_ns = 2000000000ull; // budget of one mbarrier wait
    // the Cholesky's lookahead: the next diagonal block is factored on
    // `side` while the trailing update runs (ev_pre: its block is ready;
    // ev_diag: it is factored)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_pre = nullptr, ev_diag = nullptr;
};

// C(i, j) -= sum_k P(i, k) P(j, k) for rows/cols < n with i >= j; P is
// n x k (k <= 64) column-major with leading dimension ldp, C n x n with ldc.
// Rows below `skip` (the leading skip x skip block, updated elsewhere) are
// left alone; `reserve_sms` SMs are left free for concurrent kernels.
void ozaki_syrk_sub_lower(cudaStream_t st, const dd_t *P, long ldp, int n, int k, dd_t *C, long ldc, OzakiWork &w, int skip = 0,
                          int reserve_sms = 0);
// Throws when a launch since the last check gave up waiting (synchronises st).
void ozaki_check(cudaStream_t st, const OzakiWork &w);

// The split of a long product C(i,j) = sum_k W(i,k) V(j,k), i >= j (the
// Schur complement's F1 pair products): W and V n x K, row r at
// W + r * ldw (K contiguous dd); C n x n column-major, lower triangle
// stored.  K <= OG_MAX_K (every diagonal of slice products accumulates
// exactly in int32 over the whole K).
constexpr long OG_MAX_K = 32767;
struct OzakiGemmWork {
    int8_t *sw = nullptr, *sv = nullptr; // slices of W and V
    size_t slice_bytes = 0;              // bytes of each slice buffer
    int *ew = nullptr, *ev = nullptr;    // row exponents (rows_cap each)
    int rows_cap = 0;
    int *err = nullptr;
    int *h_err = nullptr;
    cudaEvent_t wait_ev = nullptr;
    int slices = 16;
    unsigned long long wait_ns = 2000000000ull;
};
// Workspace bytes of one slice buffer for n rows, K values and S slices.
inline size_t ozaki_gemm_slice_bytes(int n, long K, int slices) {
    const long rows = (long)((n + 127) / 128) * 128, kpad = (K + 63) / 64 * 64;
    return (size_t)slices * rows * kpad;
}
void ozaki_gemm_lower(cudaStream_t st, const dd_t *W, long ldw, const dd_t *V, long ldv, int n, long K, dd_t *C, long ldc, OzakiGemmWork &w);
// Throws when a launch since the last check gave up waiting (synchronises st).
void ozaki_gemm_check(cudaStream_t st, const OzakiGemmWork &w);

} // namespace sddd
