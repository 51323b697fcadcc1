// Kernels of the step-length eigenvalue (eig.cu), declared for the other
// translation units that launch them on their own buffers.
#pragma once

#include "common.cuh"

namespace sddd {

constexpr int LZ_THREADS = 512; // threads of the one-CTA-per-block Lanczos kernel
constexpr int LZ_KMAX = 128;    // bound on the Lanczos steps held in shared memory

// One CTA per block id: lambda_min(L D L^T) of block blk_ids[blockIdx.x]
// (order sizes[b], data at Lsp/Dsp + off[b]); CTAs nb .. 2 nb - 1 take the
// same nb blocks of a second space (Lsp2, Dsp2); work holds 5 n-vectors per
// CTA at stride work_stride; the result goes to out[blockIdx.x].
__global__ void __launch_bounds__(LZ_THREADS) lanczos_kernel(const int *blk_ids, int nb, const int *sizes, const long *off, const dd_t *Lsp,
                                                             const dd_t *Dsp, const dd_t *Lsp2, const dd_t *Dsp2, dd_t *work, long work_stride, dd_t *out);

// One warp per block id: smallest eigenvalue of the lower triangle of the
// symmetric M (order <= 32) at Msp + off[b]; the result goes to out[blockIdx.x].
__global__ void __launch_bounds__(32) small_min_eig_kernel(const int *blk_ids, const int *sizes, const long *off, const dd_t *Msp, dd_t *out);

} // namespace sddd
