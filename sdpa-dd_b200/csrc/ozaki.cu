// Tensor-core split of the Cholesky trailing update, C(lower) -= P P^T.
//
// Split (ozaki_split_kernel).  Row r of the panel is scaled by 2^-e_r, with
// e_r chosen so that every |P(r,k)| 2^-e_r <= 1/2, and then peeled into
// signed base-128 digits: u = P(r,k) 2^(7-e_r); for s = 1..S:
// D_s = rint(u.hi), u = (u - D_s) * 128.  Each step is exact in dd (the
// integer is subtracted from the high part, the remainder renormalised with
// TwoSum), every digit lies in [-64, 64], and after S digits the value is
// known to 2^-(7S+1) of its row's scale: S = 16 gives 113 bits.
//   P(r,k) = 2^e_r sum_s D_s(r,k) 2^-7s  (+ remainder)
//
// Products (ozaki_syrk_kernel).  C(i,j) -= 2^(e_i+e_j) sum_d 2^-7d A_d(i,j),
// A_d = sum_{s+t=d} D_s(i,:) . D_t(j,:), for d = 2..S+1 (the S(S+1)/2 slice
// pairs that reach 7(S+1) bits).  Every A_d is an exact int32 (|A_d| <=
// 16 * 64 * 64 * 64 = 2^22), accumulated by tcgen05.mma kind::i8 in tensor
// memory.
//
// One tcgen05.mma costs about the same time for any N up to 128 (on B200 a
// kind::i8 M=128 K=32 instruction occupies the issuing thread ~97 cycles
// for N = 32..128 and ~170 for N = 256), so the kernel issues few, wide
// MMAs: a tile is 128 rows x 16 columns, its B operand the tile's S slices
// stacked (row 16 (t-1) + j is slice t of column j), and its accumulators
// are laid out by diagonal (diagonal d in columns 16 (d-2) .. 16 (d-2) + 15).
// The MMA of A slice s against stacked B slices 1 .. S+1-s (N = 16 (S+1-s))
// then writes diagonals s+1 .. S+1 in one instruction: S x 2 K steps = 32
// MMAs per tile for 16 slices.
//
// Epilogue: four consecutive diagonals combine exactly into a double
// (2^21 A_d + 2^14 A_d+1 + 2^7 A_d+2 + A_d+3 < 2^44: two int32 pairs and one
// FMA), the four groups (2^-28 apart) sum to a dd through two TwoSums, and
// the dd is scaled by 2^(e_i+e_j-35) and subtracted from C.
//
// Kernel layout: one persistent CTA per SM over the tiles of the lower
// triangle (row-block major, so a CTA keeps its 128-row A slices in shared
// memory while it walks the columns).  Warp 0 lane 0 stages operands with
// bulk copies (cp.async.bulk, no multicast; B four tiles deep) and issues
// the MMAs; warps 1-16 drain tensor memory, which holds two accumulator
// buffers of 16 x 16 columns, so one tile multiplies while the last drains.
// Operand layout in global and shared memory: per slice, 8-row groups of
// 512 bytes, each four 128-byte core matrices (8 rows x 16 K-bytes): the
// K-major, non-swizzled canonical layout of the MMA's shared-memory
// descriptors (LBO 128 bytes between the two K chunks of one MMA, SBO 512
// bytes between row groups), so a tile's stacked B slices are contiguous.
// Every mbarrier wait is bounded (the context's wait budget, 2 s by
// default); on expiry the CTA records a code in
// the error word, stops issuing, waits (bounded) for what it issued and
// frees its tensor memory.
#include "ozaki.h"

#include <algorithm>
#include <string>

#include "bulk.cuh"
#include "prof.h"

namespace sddd {

namespace {

constexpr int OZ_EPI_WARPS = 16; // epilogue warps: four per tensor-memory lane quadrant
constexpr int OZ_EPI_COLS = OZ_COLS_B / (OZ_EPI_WARPS / 4); // tile columns per epilogue thread
constexpr int OZ_THREADS = 32 * (1 + OZ_EPI_WARPS); // warp 0: copies + MMA; the rest: epilogue
// 17 warps put five on one SM sub-partition: 5 x 32 x 96 registers fit its 16384
constexpr int OZ_MAX_REGS = 96;
constexpr int OZ_A_BYTES = OZ_ROWS_A * OZ_K; // one slice of a 128-row block
constexpr int OZ_B_BYTES = OZ_COLS_B * OZ_K; // one slice of a 16-row block
constexpr int OZ_TILE_B = OZ_MAX_SLICES * OZ_B_BYTES; // the stacked B slices of a tile
constexpr int OZ_STAGES = 4;                 // B tiles in shared memory
constexpr int OZ_ACC_COLS = OZ_MAX_SLICES * OZ_COLS_B; // tensor-memory columns of one accumulator buffer
static_assert(2 * OZ_ACC_COLS <= 512, "split kernel: two accumulator buffers must fit tensor memory");
static_assert(OZ_ACC_COLS <= 256, "split kernel: the widest MMA has N = 16 S <= 256");
// the 16 A slices of a row block and OZ_STAGES stacked B tiles
constexpr size_t OZ_SMEM = 1024 + (size_t)OZ_MAX_SLICES * OZ_A_BYTES + (size_t)OZ_STAGES * OZ_TILE_B;
static_assert(OZ_SMEM <= 232448 - 256, "split kernel: shared memory above the per-CTA limit");
// kind::i8 instruction descriptor: D s32, A and B s8, both K-major, M = 128,
// N = n (a multiple of 16, 16..256).
__host__ __device__ constexpr uint32_t oz_idesc(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OZ_ROWS_A >> 4) << 24);
}

__device__ __forceinline__ unsigned long long oz_ns() { return globaltimer_ns(); }
// Waits for the phase with the given parity to complete; false when the CTA
// is aborting or the wait ran out (then the CTA aborts with `code`).
__device__ bool oz_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag, int *err, int code, unsigned long long wait_ns) {
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = oz_ns();
    while (!mbar_try_wait(b, parity)) {
        if (*abort_flag) return false;
        if (oz_ns() - t0 > wait_ns) {
            *abort_flag = 1;
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128, SBO 512,
// descriptor version 1.
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

struct OzArgs {
    const int8_t *slices;   // slice by slice (A operands: a row block of one slice is contiguous)
    const int8_t *slices_b; // by 16-row block (B operands: a tile's slices are contiguous)
    long slice_stride; // bytes between slices
    const int *exps;
    dd_t *C;
    long ldc;
    int n, ns, nI, nJ;
    int skip; // rows below skip are not written (their block is updated elsewhere)
    long tiles;
    int *err;
    unsigned long long wait_ns; // budget of one mbarrier wait
};

// Tiles of the lower triangle, row-block major: row block I (128 rows) has
// min(8 (I + 1), nJ) column blocks of 16.
constexpr int OZ_JPI = OZ_ROWS_A / OZ_COLS_B;
__device__ __forceinline__ void oz_tile_at(long t, int nI, int nJ, int &I, int &J) {
    I = 0;
    for (; I < nI; ++I) {
        const long cnt = min((long)OZ_JPI * (I + 1), (long)nJ);
        if (t < cnt) break;
        t -= cnt;
    }
    J = (int)t;
}
__device__ __forceinline__ void oz_tile_next(int nJ, int &I, int &J) {
    if (++J >= min(OZ_JPI * (I + 1), nJ)) {
        ++I;
        J = 0;
    }
}

// Shared state of one CTA.
//   barA          A slices of the current row block landed
//   barB[st]      the B slices of the tile in stage st landed
//   bfree[st]     every MMA of the tile in stage st completed (the stage,
//                 and at a row-block change A, may be reloaded)
//   tfull/tempty  accumulator buffer b holds a finished tile / is drained
//   fin           every MMA the CTA issued completed (exit)
struct OzShared {
    uint64_t barA, barB[OZ_STAGES], bfree[OZ_STAGES], tfull[2], tempty[2], fin;
    uint32_t tmem;
    int abort_flag;
};

__device__ __forceinline__ void tc_mma_i8_n(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), "l"(da),
                 "l"(db), "r"(idesc), "r"(accumulate)
                 : "memory");
}

// The MMAs of one tile into the accumulator buffer at dbuf: for A slice s
// and K step kk, one MMA against the stacked B slices t = 1 .. S+1-s
// (N = 16 (S+1-s)) writes the columns of diagonals s+1 .. S+1.  The first
// (s = 1, N = 16 S) covers every column and overwrites; the rest accumulate.
template <int NS>
__device__ __forceinline__ void oz_issue_tile(uint32_t dbuf, uint64_t descA, uint64_t descB) {
#pragma unroll
    for (int s = 1; s <= NS; ++s) {
#pragma unroll
        for (int kk = 0; kk < 2; ++kk)
            tc_mma_i8_n(dbuf + (uint32_t)((s - 1) * OZ_COLS_B), descA + (uint64_t)(((s - 1) * OZ_A_BYTES + kk * 256) >> 4),
                        descB + (uint64_t)((kk * 256) >> 4), oz_idesc((NS + 1 - s) * OZ_COLS_B), (s == 1 && kk == 0) ? 0u : 1u);
    }
}
__device__ __forceinline__ void oz_issue_tile_rt(int ns, uint32_t dbuf, uint64_t descA, uint64_t descB) {
    for (int s = 1; s <= ns; ++s)
        for (int kk = 0; kk < 2; ++kk)
            tc_mma_i8_n(dbuf + (uint32_t)((s - 1) * OZ_COLS_B), descA + (uint64_t)(((s - 1) * OZ_A_BYTES + kk * 256) >> 4),
                        descB + (uint64_t)((kk * 256) >> 4), oz_idesc((ns + 1 - s) * OZ_COLS_B), (s == 1 && kk == 0) ? 0u : 1u);
}

// A wait that ignores the abort flag (still bounded): used on the way out,
// where copies and MMAs already issued must finish before the CTA releases
// its shared and tensor memory.
__device__ void oz_wait_out(uint64_t *b, uint32_t parity, int *err, unsigned long long wait_ns) {
    const unsigned long long t0 = oz_ns();
    while (!mbar_try_wait(b, parity)) {
        if (oz_ns() - t0 > wait_ns) {
            atomicCAS(err, 0, 5);
            return;
        }
    }
}

// Warp 0, lane 0: bulk copies of the operands and the MMAs.  The A slices
// of a row block stay in shared memory while the CTA walks its columns; the
// B slices of the next OZ_STAGES - 1 tiles are in flight while a tile
// multiplies (tile n in stage n mod OZ_STAGES, accumulators in buffer
// n mod 2).
__device__ void oz_producer(const OzArgs &a, OzShared &S, uint8_t *smA, uint8_t *smB, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    const int ns = a.ns;
    const long ntile = t_end - t_begin;
    // one bulk copy per tile: the block's ns slices lie back to back
    auto load_B = [&](int jb, int st) {
        mbar_expect_tx(&S.barB[st], (uint32_t)(ns * OZ_B_BYTES));
        bulk_g2s(smB + (size_t)st * OZ_TILE_B, a.slices_b + (long)jb * ns * OZ_B_BYTES, (uint32_t)(ns * OZ_B_BYTES), &S.barB[st]);
    };
    const uint64_t descA = oz_desc(smem_u32(smA));
    const uint64_t descB0 = oz_desc(smem_u32(smB));
    int Ip, Jp; // the next tile to prefetch (np)
    oz_tile_at(t_begin, a.nI, a.nJ, Ip, Jp);
    long np = 0;
    for (; np < ntile && np < OZ_STAGES - 1; ++np) {
        load_B(Jp, (int)(np % OZ_STAGES));
        oz_tile_next(a.nJ, Ip, Jp);
    }
    int I, J;
    oz_tile_at(t_begin, a.nI, a.nJ, I, J);
    uint32_t phA = 0;
    bool pendA = false, issued = false;
    int curA = -1;
    long nb = 0; // tiles whose B copy has been waited for
    bool ok = true;
    for (long n = 0; n < ntile && ok; ++n) {
        const int st = (int)(n % OZ_STAGES), b = (int)(n & 1);
        if (I != curA) {
            // every MMA of the previous tile reads A
            if (n > 0) {
                ok = oz_wait(&S.bfree[(n - 1) % OZ_STAGES], (uint32_t)(((n - 1) / OZ_STAGES) & 1), abort_flag, a.err, 1, a.wait_ns);
                if (!ok) break;
            }
            mbar_expect_tx(&S.barA, (uint32_t)(ns * OZ_A_BYTES));
            for (int s = 0; s < ns; ++s)
                bulk_g2s(smA + (size_t)s * OZ_A_BYTES, a.slices + s * a.slice_stride + (long)I * OZ_A_BYTES, OZ_A_BYTES, &S.barA);
            pendA = true;
            ok = oz_wait(&S.barA, phA, abort_flag, a.err, 2, a.wait_ns);
            if (!ok) break;
            phA ^= 1u;
            pendA = false;
            curA = I;
        }
        ok = oz_wait(&S.barB[st], (uint32_t)((n / OZ_STAGES) & 1), abort_flag, a.err, 3, a.wait_ns);
        if (!ok) break;
        nb = n + 1;
        ok = oz_wait(&S.tempty[b], (uint32_t)(((n >> 1) & 1) ^ 1), abort_flag, a.err, 4, a.wait_ns);
        if (!ok) break;
        tc_fence_after();
        const uint64_t descB = descB0 + (uint64_t)(((size_t)st * OZ_TILE_B) >> 4);
        if (ns == OZ_MAX_SLICES)
            oz_issue_tile<OZ_MAX_SLICES>(S.tmem + (uint32_t)(b * OZ_ACC_COLS), descA, descB);
        else
            oz_issue_tile_rt(ns, S.tmem + (uint32_t)(b * OZ_ACC_COLS), descA, descB);
        issued = true;
        tc_commit(&S.tfull[b]);
        tc_commit(&S.bfree[st]);
        // prefetch tile np (= n + OZ_STAGES - 1) once tile np - OZ_STAGES
        // (= n - 1), the last user of its stage, has completed
        if (np < ntile) {
            const int sp = (int)(np % OZ_STAGES);
            if (np >= OZ_STAGES) {
                ok = oz_wait(&S.bfree[sp], (uint32_t)(((np - OZ_STAGES) / OZ_STAGES) & 1), abort_flag, a.err, 1, a.wait_ns);
                if (!ok) break;
            }
            load_B(Jp, sp);
            oz_tile_next(a.nJ, Ip, Jp);
            ++np;
        }
        oz_tile_next(a.nJ, I, J);
    }
    // On the way out every issued copy lands and every issued MMA completes
    // (bounded waits) before the CTA frees its memory.
    if (pendA) oz_wait_out(&S.barA, phA, a.err, a.wait_ns);
    for (long k = nb; k < np; ++k) oz_wait_out(&S.barB[k % OZ_STAGES], (uint32_t)((k / OZ_STAGES) & 1), a.err, a.wait_ns);
    if (issued) {
        tc_commit(&S.fin);
        oz_wait_out(&S.fin, 0, a.err, a.wait_ns);
    }
}

// 2^e as a double for -1022 <= e <= 1023 (built from its bits)
__device__ __forceinline__ double oz_pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

__device__ __forceinline__ void tc_ld2(uint32_t taddr, int32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
}

// Sum of the diagonals of one entry as a dd, from its diagonal values
// v[0..15] (diagonal d at v[d-2]; those beyond S+1 are zero), in units of
// 2^(e_i + e_j): value = sum_d A_d 2^-7d.  Pairs P_k = 2^7 A_2k+2 + A_2k+3
// are exact in int32 (|P| < 2^30) and in a double; groups G_j = 2^14 P_2j +
// P_2j+1 are exact doubles (|G| < 2^44, one FMA each), so value = 2^-35
// (G0 + G1 2^-28 + G2 2^-56 + G3 2^-84).  Two TwoSums leave only the
// rounding of the two smallest parts' sum and of the final low part:
// within 2^-106 of the value plus 2^-140 absolute.  The result comes back
// without its factor 2^-35, which the caller folds into the entry's scale.
__device__ __forceinline__ void oz_entry_dd(const int32_t (*v)[2], int c, double &hi, double &lo) {
    double G[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int32_t p0 = v[4 * j][c] * 128 + v[4 * j + 1][c], p1 = v[4 * j + 2][c] * 128 + v[4 * j + 3][c];
        G[j] = __fma_rn((double)p0, 16384.0, (double)p1);
    }
    const double a = G[0], b = G[1] * 0x1p-28, cc = G[2] * 0x1p-56, d = G[3] * 0x1p-84;
    double e1, s1 = ddm::two_sum(a, b, e1);
    double e2, s2 = ddm::two_sum(e1, cc, e2);
    double l, h = ddm::two_sum(s1, s2, l);
    h = ddm::fast_two_sum(h, l + (e2 + d), l);
    hi = h;
    lo = l;
}

// Epilogue warps 1-16: warp w reads tensor-memory lanes 32 (w mod 4) .. +31
// (its rows of the tile) and columns 4 h .. 4 h + 3 of every diagonal,
// h = (w - 1) / 4, two columns at a time with all diagonals in one round
// trip; each entry's dd (oz_entry_dd) is scaled by 2^(e_i + e_j) and
// subtracted from C, whose entries were requested before the wait for the
// accumulators.  NSC: the slice count when known at compile time, else 0.
template <int NSC>
__device__ void oz_epilogue(const OzArgs &a, OzShared &S, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, h = (warp - 1) >> 2;
    const int row = 32 * q + lane;
    const uint32_t lane_base = S.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(OZ_EPI_COLS * h);
    const int nd = NSC > 0 ? NSC : a.ns; // diagonals 2 .. S+1
    int I, J;
    oz_tile_at(t_begin, a.nI, a.nJ, I, J);
    // lane 0 waits; the warp follows its outcome (the tensor-memory loads
    // are warp-collective)
    auto wait_full = [&](int b, uint32_t parity) {
        int okw = 1;
        if (lane == 0) okw = oz_wait(&S.tfull[b], parity, abort_flag, a.err, 6, a.wait_ns) ? 1 : 0;
        return __shfl_sync(0xffffffffu, okw, 0) != 0;
    };
    for (long n = 0; n < t_end - t_begin; ++n) {
        const int i = I * OZ_ROWS_A + row;
        const int jb = J * OZ_COLS_B + OZ_EPI_COLS * h;
        const int b = (int)(n & 1);
        dd_t *cp = a.C + i + a.ldc * (long)jb;
        // entries of the lower triangle of C: columns jb .. jb + ncol - 1
        const int ncol = (i < a.n && i >= a.skip) ? max(0, min(OZ_EPI_COLS, min(a.n, i + 1) - jb)) : 0;
        double2 cv[OZ_EPI_COLS];
#pragma unroll
        for (int c = 0; c < OZ_EPI_COLS; ++c)
            cv[c] = c < ncol ? __ldcs(reinterpret_cast<const double2 *>(cp + a.ldc * (long)c)) : make_double2(0.0, 0.0);
        if (!wait_full(b, (uint32_t)((n >> 1) & 1))) break;
        tc_fence_after();
        const uint32_t tb = lane_base + (uint32_t)(b * OZ_ACC_COLS);
        const int ei = a.exps[i]; // scale exponent of the row (padded rows hold 0)
        const int4 e4 = *reinterpret_cast<const int4 *>(a.exps + jb);
        const int ej[4] = {e4.x, e4.y, e4.z, e4.w};
        // Drain first: every entry's dd from tensor memory, then the
        // buffer goes back to the MMA warp; only then the entries meet C,
        // so the accumulators are never held while C is in flight.
        double phi[OZ_EPI_COLS], plo[OZ_EPI_COLS];
#pragma unroll
        for (int ch = 0; ch < OZ_EPI_COLS / 2; ++ch) {
            int32_t v[OZ_MAX_SLICES][2];
#pragma unroll
            for (int u = 0; u < OZ_MAX_SLICES; ++u) {
                if (u < nd) {
                    tc_ld2(tb + (uint32_t)(u * OZ_COLS_B + 2 * ch), v[u]);
                } else {
                    v[u][0] = 0;
                    v[u][1] = 0;
                }
            }
            tc_wait_ld();
            if (ch == OZ_EPI_COLS / 2 - 1) { // the buffer is drained
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&S.tempty[b]);
            }
#pragma unroll
            for (int c = 0; c < 2; ++c) oz_entry_dd(v, c, phi[2 * ch + c], plo[2 * ch + c]);
        }
#pragma unroll
        for (int cc = 0; cc < OZ_EPI_COLS; ++cc) {
            if (cc < ncol) {
                const int sc = ei + ej[cc] - 35;
                dd_t p;
                if (sc >= -1022 && sc <= 1023) {
                    const double pw = oz_pow2(sc);
                    p = dd_make(phi[cc] * pw, plo[cc] * pw);
                } else {
                    p = dd_make(ldexp(phi[cc], sc), ldexp(plo[cc], sc));
                }
                const dd_t res = dd_sub(dd_make(cv[cc].x, cv[cc].y), p);
                __stcs(reinterpret_cast<double2 *>(cp + a.ldc * (long)cc), make_double2(res.hi, res.lo));
            }
        }
        oz_tile_next(a.nJ, I, J);
    }
}

__global__ void __maxnreg__(OZ_MAX_REGS) ozaki_syrk_kernel(OzArgs a) {
    extern __shared__ uint8_t oz_raw[];
    __shared__ OzShared S;
    uint8_t *smA = reinterpret_cast<uint8_t *>(((uintptr_t)oz_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *smB = smA + (size_t)OZ_MAX_SLICES * OZ_A_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const long t_begin = a.tiles * blockIdx.x / gridDim.x, t_end = a.tiles * (blockIdx.x + 1) / gridDim.x;
    if (t_begin >= t_end) return;
    if (tid == 0) {
        S.abort_flag = *(volatile int *)a.err != 0;
        mbar_init(&S.barA, 1);
        mbar_init(&S.fin, 1);
        for (int st = 0; st < OZ_STAGES; ++st) {
            mbar_init(&S.barB[st], 1);
            mbar_init(&S.bfree[st], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.tfull[b], 1);
            mbar_init(&S.tempty[b], OZ_EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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
        if ((tid & 31) == 0) oz_producer(a, S, smA, smB, t_begin, t_end);
        __syncwarp();
    } else {
        if (a.ns == OZ_MAX_SLICES)
            oz_epilogue<OZ_MAX_SLICES>(a, S, t_begin, t_end);
        else
            oz_epilogue<0>(a, S, t_begin, t_end);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(512) : "memory");
    }
}

// Digits of 32 rows per CTA; warp c takes K bytes 16c..16c+15.  Each
// 16-byte group goes to both layouts: slice by slice (slices) and by
// 16-row block, the block's ns slices back to back (slices_b).
__global__ void __launch_bounds__(128) ozaki_split_kernel(const dd_t *P, long ldp, int n, int k, int ns, int8_t *slices, int8_t *slices_b, long slice_stride,
                                                          int *exps) {
    __shared__ double rmax[4][32];
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    const int r = blockIdx.x * 32 + lane;
    dd_t x[16];
    double m = 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int kk = 16 * c + q;
        x[q] = (r < n && kk < k) ? ld_dd(P + r + ldp * (long)kk) : dd_zero();
        m = fmax(m, fabs(x[q].hi));
    }
    rmax[c][lane] = m;
    __syncthreads();
    m = fmax(fmax(rmax[0][lane], rmax[1][lane]), fmax(rmax[2][lane], rmax[3][lane]));
    int e = 0;
    if (m > 0.0) {
        int E;
        frexp(m, &E); // m < 2^E, so |P| 2^-(E+1) <= 1/2
        e = E + 1;
    }
    if (c == 0) exps[r] = e;
#pragma unroll
    for (int q = 0; q < 16; ++q) x[q] = dd_make(ldexp(x[q].hi, 7 - e), ldexp(x[q].lo, 7 - e));
    const int within = ((r >> 3) & 1) * 512 + c * 128 + (r & 7) * 16; // offset inside a 16-row block of one slice
    int8_t *dst = slices + (long)(r >> 4) * 1024 + within;
    int8_t *dstb = slices_b + (long)(r >> 4) * ns * 1024 + within;
    for (int s = 0; s < ns; ++s) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const double d = rint(x[q].hi);
            w[q >> 2] |= ((uint32_t)((int)d) & 0xffu) << (8 * (q & 3));
            double err, sum = ddm::two_sum(x[q].hi - d, x[q].lo, err);
            x[q] = dd_make(sum * 128.0, err * 128.0);
        }
        const uint4 v = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4 *>(dst + (long)s * slice_stride) = v;
        *reinterpret_cast<uint4 *>(dstb + (long)s * 1024) = v;
    }
}

} // namespace

void ozaki_syrk_sub_lower(cudaStream_t st, const dd_t *P, long ldp, int n, int k, dd_t *C, long ldc, OzakiWork &w, int skip, int reserve_sms) {
    if (n <= 0 || k <= 0) return;
    if (k > OZ_K) throw Error(ERR_ARG, "ozaki: panel wider than 64 columns");
    if (w.slices_used < 8 || w.slices_used > OZ_MAX_SLICES) throw Error(ERR_ARG, "ozaki: slice count must be 8..16");
    const int rows = (int)(ceil_div(n, OZ_ROWS_A) * OZ_ROWS_A);
    if (rows > w.row_cap || !w.slices || !w.slices_b || !w.exps || !w.err) throw Error(ERR_ARG, "ozaki: workspace smaller than the panel");
    const long stride = (long)w.row_cap * OZ_K;
    ozaki_split_kernel<<<rows / 32, 128, 0, st>>>(P, ldp, n, k, w.slices_used, w.slices, w.slices_b, stride, w.exps);
    CK_LAUNCH();
    OzArgs a;
    a.slices = w.slices;
    a.slices_b = w.slices_b;
    a.slice_stride = stride;
    a.exps = w.exps;
    a.C = C;
    a.ldc = ldc;
    a.n = n;
    a.ns = w.slices_used;
    a.nI = rows / OZ_ROWS_A;
    a.nJ = (int)ceil_div(n, OZ_COLS_B);
    a.skip = skip;
    a.err = w.err;
    a.wait_ns = w.wait_ns;
    long tiles = 0;
    for (int I = 0; I < a.nI; ++I) tiles += std::min((long)(OZ_ROWS_A / OZ_COLS_B) * (I + 1), (long)a.nJ);
    a.tiles = tiles;
    static thread_local int sms[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &sm = sms[dev & 63];
    if (sm == 0) {
        CK(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(ozaki_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)OZ_SMEM));
    }
    const int grid = (int)std::min<long>(std::max(1, sm - reserve_sms), tiles);
    ozaki_syrk_kernel<<<grid, OZ_THREADS, OZ_SMEM, st>>>(a);
    CK_LAUNCH();
}

void ozaki_check(cudaStream_t st, const OzakiWork &w) {
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
        throw Error(ERR_CUDA, "ozaki: a tensor-core split update gave up waiting (code " + std::to_string(err) + ")");
    }
}

} // namespace sddd
