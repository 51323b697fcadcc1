// Tensor-core split of a long dd product, C(i,j) = sum_k W(i,k) V(j,k) for
// i >= j: the Schur complement's pair products B_ij = G_i . A_j of the F1
// formula (sdpa_newton.cpp:895, calF1: the n^2-term dot of G_i = X A_i Z^-1
// with A_j), whose K = n^2 runs to thousands.
//
// Split (og_exps_kernel, og_split_kernel).  Each row of W and of V is
// scaled by 2^-e with e from the row's largest |value| over all of K, and
// peeled into S signed base-128 digits exactly as the Cholesky's split does
// (ozaki.cu): every digit lies in [-64, 64] and S = 16 digits carry 113 bits
// of the row's scale.  One scale per row over the whole K keeps every digit
// product on one grid, so the products of all K accumulate exactly in int32:
// A_d(i,j) = sum_{s+t=d} sum_k D_s(i,k) D_t(j,k), |A_d| <= 16 * 64 * 64 * K
// < 2^31 for K < 2^15.
//
// Products (ozaki_gemm_kernel).  A tile is 128 rows x 32 columns: two
// groups of 16 columns whose S slices are stacked into one MMA operand
// (stacked row 16 (t-1) + j is slice t of column j), with accumulators laid
// out by diagonal (diagonal d at columns 16 (d-2) .. +15 of the group's 256
// tensor-memory columns), as in the Cholesky's split kernel.  Per K step of
// 32 bytes and group, the MMA of A slice s against stacked slices 1..S+1-s
// (tcgen05.mma kind::i8, M = 128, N = 16 (S+1-s), K = 32) adds every product
// of that slice to its diagonals: 2 S MMAs per step.  The whole K range
// accumulates in tensor memory; the epilogue runs once per tile.
//
// Epilogue: per entry the 16 diagonal sums are combined into a 128-bit
// integer T = sum_d A_d 2^(108-7d) (exact for d <= 15, the last two
// diagonals rounded to 2^-108, below the split's own error), cut into three
// exact 42-bit doubles and summed with TwoSum/FastTwoSum into a dd, scaled
// by 2^(e_i + e_j - 108) and stored in C.
//
// Kernel layout: one persistent CTA per SM (all 512 tensor-memory columns,
// two K-step stages of 80 KB in shared memory, double-buffered: step u + 1
// loads while the MMAs of step u run) over the tiles of the lower triangle;
// warp 0 lane 0 issues the bulk copies (cp.async.bulk, no multicast) and the
// MMAs; warps 1-16 drain tensor memory.  Slice layout in global memory: per
// slice and K step of 32 bytes, 8-row groups of 256 bytes (two 128-byte core
// matrices along K: 8 rows x 16 bytes), rows in order, so the A operand of a
// 128-row block is one 4 KB copy per slice and a 16-row column group one
// 512-byte copy per slice; shared-memory descriptors: K-major, no swizzle,
// LBO 128, SBO 256.  Every mbarrier wait is bounded by the context's wait
// budget; on expiry the CTA records a code, lets its copies and MMAs land
// and frees its tensor memory.
#include "ozaki.h"

#include <algorithm>
#include <string>

#include "bulk.cuh"
#include "prof.h"

namespace sddd {

namespace {

constexpr int OG_M = 128;          // tile rows (MMA M)
constexpr int OG_G = 16;           // columns per group (per slice in the stacked operand)
constexpr int OG_GROUPS = 2;       // column groups per tile
constexpr int OG_N = OG_G * OG_GROUPS; // tile columns
constexpr int OG_KB = 32;          // K bytes per step (one MMA)
constexpr int OG_STAGES = 2;
constexpr int OG_EPI_WARPS = 16;
constexpr int OG_THREADS = 32 * (1 + OG_EPI_WARPS);
constexpr int OG_A_SLICE = OG_M * OG_KB;           // 4 KB
constexpr int OG_B_SLICE = OG_G * OG_KB;           // 512 B
constexpr int OG_A_STAGE = OZ_MAX_SLICES * OG_A_SLICE;                // 64 KB
constexpr int OG_B_STAGE = OG_GROUPS * OZ_MAX_SLICES * OG_B_SLICE;    // 16 KB
constexpr int OG_STAGE = OG_A_STAGE + OG_B_STAGE;
constexpr int OG_ACC_COLS = OZ_MAX_SLICES * OG_G; // 256 per group
static_assert(OG_GROUPS * OG_ACC_COLS <= 512, "ozaki gemm: accumulators must fit tensor memory");
constexpr size_t OG_SMEM = 1024 + (size_t)OG_STAGES * OG_STAGE;
static_assert(OG_SMEM <= 232448 - 256, "ozaki gemm: shared memory above the per-CTA limit");
constexpr int OG_EPI_COLS = OG_N / (OG_EPI_WARPS / 4); // 8 columns per epilogue thread
constexpr int OG_MAX_REGS = 96;

// kind::i8 instruction descriptor: D s32, A and B s8, both K-major, M = 128,
// N = n (a multiple of 16, 16..256).
__host__ __device__ constexpr uint32_t og_idesc(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OG_M >> 4) << 24);
}
// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128, SBO 256,
// descriptor version 1.
__device__ __forceinline__ uint64_t og_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_ld2(uint32_t taddr, int32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
}
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), "l"(da),
                 "l"(db), "r"(idesc), "r"(accumulate)
                 : "memory");
}

struct OgArgs {
    const int8_t *sw, *sv;   // slices of W and V
    long slice_stride;       // bytes between slices (both operands)
    long step_stride;        // bytes between K steps of one slice (rows_pad * 32)
    const int *ew, *ev;      // row exponents
    dd_t *C;
    long ldc;
    int n;                   // rows of W and of V (the lower triangle of n x n)
    int ns, nsteps, nI, nJ;
    long tiles;
    int *err;
    unsigned long long wait_ns;
};

//   full[st] / free_[st]  stage st landed / its MMAs completed
//   tfull / tempty        the accumulators hold a finished tile / are drained
//   fin                   every MMA the CTA issued completed (exit)
struct OgShared {
    uint64_t full[OG_STAGES], free_[OG_STAGES], tfull, tempty, fin;
    uint32_t tmem;
    int abort_flag;
};

// Bounded mbarrier wait; false when the CTA is aborting or the wait ran out
// (then the CTA aborts with `code`).
__device__ bool og_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag, const OgArgs &a, int code) {
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(b, parity)) {
        if (*abort_flag) return false;
        if (globaltimer_ns() - t0 > a.wait_ns) {
            *abort_flag = 1;
            atomicCAS(a.err, 0, code);
            return false;
        }
    }
    return true;
}
// The same wait ignoring the abort flag (still bounded), on the way out.
__device__ void og_wait_out(uint64_t *b, uint32_t parity, const OgArgs &a) {
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(b, parity))
        if (globaltimer_ns() - t0 > a.wait_ns) {
            atomicCAS(a.err, 0, 15);
            return;
        }
}

// Tiles of the lower triangle, row-block major: row block I (128 rows) has
// min(4 (I + 1), nJ) column blocks of 32.
constexpr int OG_JPI = OG_M / OG_N;
__device__ __forceinline__ void og_tile_at(long t, int nI, int nJ, int &I, int &J) {
    I = 0;
    for (; I < nI; ++I) {
        const long cnt = min((long)OG_JPI * (I + 1), (long)nJ);
        if (t < cnt) break;
        t -= cnt;
    }
    J = (int)t;
}
__device__ __forceinline__ void og_tile_next(int nJ, int &I, int &J) {
    if (++J >= min(OG_JPI * (I + 1), nJ)) {
        ++I;
        J = 0;
    }
}

// Warp 0, lane 0: the copies of every K step of the CTA's tiles (step u of
// the CTA in stage u mod 2) and their MMAs.
__device__ void og_producer(const OgArgs &a, OgShared &S, uint8_t *sm, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    const int ns = a.ns;
    const long total = (t_end - t_begin) * a.nsteps; // K steps of all tiles
    int Il, Jl;                                      // tile of the next step to load
    og_tile_at(t_begin, a.nI, a.nJ, Il, Jl);
    int kl = 0;
    auto load = [&](long u) {
        const int st = (int)(u % OG_STAGES);
        uint8_t *dst = sm + (size_t)st * OG_STAGE;
        mbar_expect_tx(&S.full[st], (uint32_t)(ns * (OG_A_SLICE + OG_GROUPS * OG_B_SLICE)));
        const long koff = (long)kl * a.step_stride;
        for (int s = 0; s < ns; ++s) {
            bulk_g2s(dst + (size_t)s * OG_A_SLICE, a.sw + s * a.slice_stride + koff + (long)Il * OG_A_SLICE, OG_A_SLICE, &S.full[st]);
            for (int g = 0; g < OG_GROUPS; ++g)
                bulk_g2s(dst + OG_A_STAGE + (size_t)(g * OZ_MAX_SLICES + s) * OG_B_SLICE,
                         a.sv + s * a.slice_stride + koff + (long)(Jl * OG_GROUPS + g) * OG_B_SLICE, OG_B_SLICE, &S.full[st]);
        }
        if (++kl == a.nsteps) {
            kl = 0;
            og_tile_next(a.nJ, Il, Jl);
        }
    };
    // double buffering: while the MMAs of step u run, step u + 1 loads
    // into the stage that step u - 1 used
    long nl = 0; // steps loaded
    if (total > 0) {
        load(0);
        nl = 1;
    }
    long nf = 0; // steps whose MMAs were issued
    bool ok = true, issued = false;
    const uint32_t sm0 = smem_u32(sm);
    long tile = 0;
    for (long u = 0; u < total && ok; ++u) {
        const int st = (int)(u % OG_STAGES);
        const int k = (int)(u % a.nsteps);
        if (k == 0 && tile > 0) {
            // the epilogue has drained the previous tile's accumulators
            ok = og_wait(&S.tempty, (uint32_t)((tile - 1) & 1), abort_flag, a, 4);
            if (!ok) break;
        }
        ok = og_wait(&S.full[st], (uint32_t)((u / OG_STAGES) & 1), abort_flag, a, 3);
        if (!ok) break;
        tc_fence_after();
        const uint32_t base = sm0 + (uint32_t)(st * OG_STAGE);
#pragma unroll 1
        for (int g = 0; g < OG_GROUPS; ++g) {
            const uint64_t db = og_desc(base + OG_A_STAGE + (uint32_t)(g * OZ_MAX_SLICES * OG_B_SLICE));
            const uint32_t dt = S.tmem + (uint32_t)(g * OG_ACC_COLS);
            for (int s = 1; s <= ns; ++s)
                tc_mma_i8(dt + (uint32_t)((s - 1) * OG_G), og_desc(base + (uint32_t)((s - 1) * OG_A_SLICE)), db, og_idesc((ns + 1 - s) * OG_G),
                          (k == 0 && s == 1) ? 0u : 1u);
        }
        issued = true;
        nf = u + 1;
        tc_commit(&S.free_[st]);
        if (k == a.nsteps - 1) {
            tc_commit(&S.tfull);
            ++tile;
        }
        if (nl < total) {
            // stage of step u + 1 = stage of step u - 1: its MMAs must be done
            if (u >= 1) {
                ok = og_wait(&S.free_[(u + 1) % OG_STAGES], (uint32_t)(((u - 1) / OG_STAGES) & 1), abort_flag, a, 1);
                if (!ok) break;
            }
            load(nl);
            ++nl;
        }
    }
    // every issued copy lands and every issued MMA completes before exit
    for (long v = nf; v < nl; ++v) og_wait_out(&S.full[v % OG_STAGES], (uint32_t)((v / OG_STAGES) & 1), a);
    if (issued) {
        tc_commit(&S.fin);
        og_wait_out(&S.fin, 0, a);
    }
}

// The entry's value / 2^(e_i + e_j) as a dd: T = sum_d A_d 2^(108 - 7d)
// (diagonal d at v[d-2]), then T 2^-108.
__device__ __forceinline__ void og_entry_dd(const int32_t (*v)[2], int c, int nd, double &hi, double &lo) {
    __int128 T = 0;
#pragma unroll
    for (int u = 0; u < OZ_MAX_SLICES; ++u) {
        if (u >= nd) break;
        const int d = u + 2;
        const int sh = 108 - 7 * d;
        const __int128 x = (__int128)v[u][c];
        if (sh >= 0)
            T += x << sh;
        else
            T += (x + ((__int128)1 << (-sh - 1))) >> (-sh); // round to the 2^-108 grid
    }
    // three exact 42-bit pieces: T = t2 2^84 + t1 2^42 + t0
    const long long t0 = (long long)(T & (((__int128)1 << 42) - 1));
    const long long t1 = (long long)((T >> 42) & (((__int128)1 << 42) - 1));
    const long long t2 = (long long)(T >> 84);
    const double d2 = ldexp((double)t2, 84 - 108), d1 = ldexp((double)t1, 42 - 108), d0 = ldexp((double)t0, -108);
    double e, s = ddm::two_sum(d2, d1, e);
    hi = ddm::fast_two_sum(s, e + d0, lo);
}

// Epilogue warps 1-16: warp w reads tensor-memory lanes 32 (w mod 4) .. +31
// (rows of the tile) and 8 columns: group h / 2, columns 8 (h mod 2) ..
// +7 of it, h = (w - 1) / 4; two columns per tensor-memory round trip.
template <int NSC>
__device__ void og_epilogue(const OgArgs &a, OgShared &S, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, h = (warp - 1) >> 2;
    const int g = h >> 1, c0 = 8 * (h & 1);
    const int row = 32 * q + lane;
    const uint32_t lane_base = S.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(g * OG_ACC_COLS + c0);
    const int nd = NSC > 0 ? NSC : a.ns;
    int I, J;
    og_tile_at(t_begin, a.nI, a.nJ, I, J);
    for (long n = 0; n < t_end - t_begin; ++n) {
        int okw = 1;
        if (lane == 0) okw = og_wait(&S.tfull, (uint32_t)(n & 1), abort_flag, a, 6) ? 1 : 0;
        if (__shfl_sync(0xffffffffu, okw, 0) == 0) break;
        tc_fence_after();
        const int i = I * OG_M + row;
        const int jb = J * OG_N + g * OG_G + c0;
        const int ei = i < a.n ? a.ew[i] : 0;
        dd_t out[OG_EPI_COLS];
#pragma unroll
        for (int ch = 0; ch < OG_EPI_COLS / 2; ++ch) {
            int32_t v[OZ_MAX_SLICES][2];
#pragma unroll
            for (int u = 0; u < OZ_MAX_SLICES; ++u) {
                if (u < nd) {
                    tc_ld2(lane_base + (uint32_t)(u * OG_G + 2 * ch), v[u]);
                } else {
                    v[u][0] = 0;
                    v[u][1] = 0;
                }
            }
            tc_wait_ld();
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                double phi, plo;
                og_entry_dd(v, c, nd, phi, plo);
                const int j = jb + 2 * ch + c;
                const int sc = ei + (j < a.n ? a.ev[j] : 0);
                out[2 * ch + c] = dd_make(ldexp(phi, sc), ldexp(plo, sc));
            }
        }
        // the accumulators are drained: the next tile may overwrite them
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.tempty);
        if (i < a.n) {
#pragma unroll
            for (int c = 0; c < OG_EPI_COLS; ++c) {
                const int j = jb + c;
                if (j <= i && j < a.n) st_dd(a.C + i + a.ldc * (long)j, out[c]);
            }
        }
        og_tile_next(a.nJ, I, J);
    }
}

__global__ void __maxnreg__(OG_MAX_REGS) ozaki_gemm_kernel(OgArgs a) {
    extern __shared__ uint8_t og_raw[];
    __shared__ OgShared S;
    uint8_t *sm = reinterpret_cast<uint8_t *>(((uintptr_t)og_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5;
    const long t_begin = a.tiles * blockIdx.x / gridDim.x, t_end = a.tiles * (blockIdx.x + 1) / gridDim.x;
    if (t_begin >= t_end) return;
    if (tid == 0) {
        S.abort_flag = *(volatile int *)a.err != 0;
        for (int st = 0; st < OG_STAGES; ++st) {
            mbar_init(&S.full[st], 1);
            mbar_init(&S.free_[st], 1);
        }
        mbar_init(&S.tfull, 1);
        mbar_init(&S.tempty, OG_EPI_WARPS);
        mbar_init(&S.fin, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (S.abort_flag) return;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)), "r"(512) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        if ((tid & 31) == 0) og_producer(a, S, sm, t_begin, t_end);
        __syncwarp();
    } else {
        if (a.ns == OZ_MAX_SLICES)
            og_epilogue<OZ_MAX_SLICES>(a, S, t_begin, t_end);
        else
            og_epilogue<0>(a, S, t_begin, t_end);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(512) : "memory");
    }
}

// e_r for each row of an n x K operand (row r at X + r * ldr, K contiguous
// dd): |X(r,:)| 2^-e_r <= 1/2 (0 for a zero row).  One warp per row.
__global__ void og_exps_kernel(const dd_t *X, long ldr, int n, long K, int rows_pad, int *exps) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= rows_pad) return;
    double m = 0.0;
    if (r < n)
        for (long k = lane; k < K; k += 32) m = fmax(m, fabs(X[r * ldr + k].hi));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
        int e = 0;
        if (m > 0.0) {
            int E;
            frexp(m, &E); // m < 2^E, so |X| 2^-(E+1) <= 1/2
            e = E + 1;
        }
        exps[r] = e;
    }
}

// Digits of 32 rows x 64 K values per CTA (warp c: K values 16c..16c+15 of
// the CTA's 64): ns slices, each 16 bytes of one row into its core matrix.
__global__ void __launch_bounds__(128) og_split_kernel(const dd_t *X, long ldr, int n, long K, int ns, const int *exps, int8_t *slices,
                                                        long slice_stride, long step_stride) {
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    const int r = blockIdx.x * 32 + lane;
    const long k0 = (long)blockIdx.y * 64 + 16 * c;
    const int e = exps[r];
    dd_t x[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const long k = k0 + u;
        const dd_t v = (r < n && k < K) ? ld_dd(X + r * ldr + k) : dd_zero();
        x[u] = dd_make(ldexp(v.hi, 7 - e), ldexp(v.lo, 7 - e));
    }
    // step k0 / 32, core matrix (k0 / 16) mod 2 of row group r / 8
    int8_t *dst = slices + (k0 / OG_KB) * step_stride + (long)(r >> 3) * 256 + ((k0 / 16) & 1) * 128 + (r & 7) * 16;
    for (int s = 0; s < ns; ++s) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const double d = rint(x[u].hi);
            w[u >> 2] |= ((uint32_t)((int)d) & 0xffu) << (8 * (u & 3));
            double err, sum = ddm::two_sum(x[u].hi - d, x[u].lo, err);
            x[u] = dd_make(sum * 128.0, err * 128.0);
        }
        *reinterpret_cast<uint4 *>(dst + (long)s * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

} // namespace

void ozaki_gemm_lower(cudaStream_t st, const dd_t *W, long ldw, const dd_t *V, long ldv, int n, long K, dd_t *C, long ldc, OzakiGemmWork &w) {
    if (n <= 0) return;
    if (K <= 0 || K > OG_MAX_K) throw Error(ERR_ARG, "ozaki gemm: K must lie in 1..32767 (exact int32 accumulation)");
    if (w.slices < 8 || w.slices > OZ_MAX_SLICES) throw Error(ERR_ARG, "ozaki gemm: slice count must be 8..16");
    const int rows_pad = (int)(ceil_div(n, OG_M) * OG_M);
    const long kpad = (long)ceil_div(K, 64) * 64;
    const long step_stride = (long)rows_pad * OG_KB;
    const long slice_stride = step_stride * (kpad / OG_KB);
    const size_t need = (size_t)w.slices * slice_stride;
    if (!w.sw || !w.sv || !w.ew || !w.ev || !w.err || need > w.slice_bytes || rows_pad > w.rows_cap)
        throw Error(ERR_ARG, "ozaki gemm: workspace smaller than the operands");
    PROF_SCOPE("schur_pairs_tc", st);
    og_exps_kernel<<<rows_pad / 8, 256, 0, st>>>(W, ldw, n, K, rows_pad, w.ew);
    CK_LAUNCH();
    og_exps_kernel<<<rows_pad / 8, 256, 0, st>>>(V, ldv, n, K, rows_pad, w.ev);
    CK_LAUNCH();
    dim3 sg(rows_pad / 32, (unsigned)(kpad / 64));
    og_split_kernel<<<sg, 128, 0, st>>>(W, ldw, n, K, w.slices, w.ew, w.sw, slice_stride, step_stride);
    CK_LAUNCH();
    og_split_kernel<<<sg, 128, 0, st>>>(V, ldv, n, K, w.slices, w.ev, w.sv, slice_stride, step_stride);
    CK_LAUNCH();
    OgArgs a;
    a.sw = w.sw;
    a.sv = w.sv;
    a.slice_stride = slice_stride;
    a.step_stride = step_stride;
    a.ew = w.ew;
    a.ev = w.ev;
    a.C = C;
    a.ldc = ldc;
    a.n = n;
    a.ns = w.slices;
    a.nsteps = (int)(kpad / OG_KB);
    a.nI = rows_pad / OG_M;
    a.nJ = (int)ceil_div(n, OG_N);
    a.err = w.err;
    a.wait_ns = w.wait_ns;
    long tiles = 0;
    for (int I = 0; I < a.nI; ++I) tiles += std::min((long)OG_JPI * (I + 1), (long)a.nJ);
    a.tiles = tiles;
    static thread_local int sms[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &sm = sms[dev & 63];
    if (sm == 0) {
        CK(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)OG_SMEM));
    }
    const int grid = (int)std::min<long>(sm, tiles);
    ozaki_gemm_kernel<<<grid, OG_THREADS, OG_SMEM, st>>>(a);
    CK_LAUNCH();
}

void ozaki_gemm_check(cudaStream_t st, const OzakiGemmWork &w) {
    if (!w.err) return;
    int err = 0;
    int *h = w.h_err ? w.h_err : &err;
    CK(cudaMemcpyAsync(h, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (w.wait_ev) {
        CK(cudaEventRecord(w.wait_ev, st));
        CK(cudaEventSynchronize(w.wait_ev));
    } else {
        CK(cudaStreamSynchronize(st));
    }
    err = *h;
    if (err != 0) {
        // clear the error word, so that the next launch starts afresh
        CK(cudaMemsetAsync(w.err, 0, sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        throw Error(ERR_CUDA, "ozaki gemm: a tensor-core split product gave up waiting (code " + std::to_string(err) + ")");
    }
}

} // namespace sddd
