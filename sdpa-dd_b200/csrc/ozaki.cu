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
// 16 * 64 * 64 * 64 = 2^22): it is accumulated by tcgen05.mma kind::i8 in
// tensor memory.  Four consecutive diagonals combine exactly in int64
// (2^21 A_d + 2^14 A_d+1 + 2^7 A_d+2 + A_d+3 < 2^44) and convert exactly to
// double; the four group values become one dd (TwoSum, exact, then one dd
// addition) that is scaled by 2^(e_i+e_j) and subtracted from C.
//
// Kernel layout: one persistent CTA per SM over 128 x 32 output tiles of the
// lower triangle (row-block major, so a CTA keeps its 128-row A slices while
// it walks the columns).  Warp 0 lane 0 stages operands with bulk copies
// (cp.async.bulk, no multicast) and issues the MMAs; warps 1-8 drain tensor
// memory.  Tensor memory holds two rounds of eight diagonal accumulators
// (8 x 32 columns each): round 0 (d = 10..17) of the next tile is issued
// while round 1 (d = 2..9) of the current one is being drained.
// Operand layout in global and shared memory: per slice, 8-row groups of
// 512 bytes, each four 128-byte core matrices (8 rows x 16 K-bytes): the
// K-major, non-swizzled canonical layout of the MMA's shared-memory
// descriptors (LBO 128 bytes between the two K chunks of one MMA, SBO 512
// bytes between row groups).
// Every mbarrier wait is bounded (2 s); on expiry the CTA records a code in
// the error word, stops issuing, waits (bounded) for what it issued and
// frees its tensor memory.
#include "ozaki.h"

#include <algorithm>
#include <string>

#include "prof.h"

namespace sddd {

namespace {

constexpr int OZ_THREADS = 288; // warp 0: copies + MMA; warps 1-8: epilogue
constexpr int OZ_A_BYTES = OZ_ROWS_A * OZ_K; // one slice of a 128-row block
constexpr int OZ_B_BYTES = OZ_COLS_B * OZ_K; // one slice of a 32-row block
constexpr size_t OZ_SMEM = 1024 + (size_t)OZ_MAX_SLICES * OZ_A_BYTES + 2 * (size_t)OZ_MAX_SLICES * OZ_B_BYTES;
// kind::i8 instruction descriptor: D s32, A and B s8, both K-major,
// N = 32, M = 128.
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_COLS_B >> 3) << 17) | ((uint32_t)(OZ_ROWS_A >> 4) << 24);
constexpr unsigned long long OZ_WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long oz_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) { asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity to complete; false when the CTA
// is aborting or the wait ran out (then the CTA aborts with `code`).
__device__ bool oz_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag, int *err, int code) {
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = oz_ns();
    while (!mbar_try_wait(b, parity)) {
        if (*abort_flag) return false;
        if (oz_ns() - t0 > OZ_WAIT_NS) {
            *abort_flag = 1;
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), "l"(da),
                 "l"(db), "r"(OZ_IDESC), "r"(accumulate)
                 : "memory");
}
__device__ __forceinline__ void tc_ld8(uint32_t taddr, int32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128, SBO 512,
// descriptor version 1.
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

// First diagonal of round r.  Round 0 takes the small diagonals 10..17 (200
// of the 272 MMAs of a 16-slice tile), round 1 the large ones 2..9: the
// epilogue's C update then overlaps the long round 0 of the next tile.
__host__ __device__ constexpr int oz_round_d0(int r) { return r == 0 ? 10 : 2; }

struct OzArgs {
    const int8_t *slices;
    long slice_stride; // bytes between slices
    const int *exps;
    dd_t *C;
    long ldc;
    int n, ns, nI, nJ;
    long tiles;
    int *err;
};

// Tiles of the lower triangle, row-block major: row block I has
// min(4 (I + 1), nJ) column blocks.
__device__ __forceinline__ void oz_tile_at(long t, int nI, int nJ, int &I, int &J) {
    I = 0;
    for (; I < nI; ++I) {
        const long cnt = min(4L * (I + 1), (long)nJ);
        if (t < cnt) break;
        t -= cnt;
    }
    J = (int)t;
}
__device__ __forceinline__ void oz_tile_next(int nJ, int &I, int &J) {
    if (++J >= min(4 * (I + 1), nJ)) {
        ++I;
        J = 0;
    }
}

// Shared state of one CTA.
struct OzShared {
    uint64_t barA, barB[2], bfree[2], tfull[2], tempty[2];
    uint32_t tmem;
    int abort_flag;
};

// MMAs of round R into its tensor-memory buffer: for each diagonal d of the
// round, the slice pairs (s, d - s) over the two 32-byte K steps; the first
// MMA of a diagonal overwrites, the others accumulate.  descA/descB address
// slice 1 of the A and B operands; slices are OZ_A_BYTES / OZ_B_BYTES apart.
template <int R, int NS>
__device__ __forceinline__ void oz_issue_round(uint32_t tmem, uint64_t descA, uint64_t descB) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int d = oz_round_d0(R) + u;
        if (d <= NS + 1) {
            const uint32_t dcol = tmem + (uint32_t)(R * 256 + u * 32);
#pragma unroll
            for (int s = 1; s <= NS; ++s) {
                const int t = d - s;
                if (t >= 1 && t <= NS) {
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const uint64_t da = descA + (uint64_t)(((s - 1) * OZ_A_BYTES + kk * 256) >> 4);
                        const uint64_t db = descB + (uint64_t)(((t - 1) * OZ_B_BYTES + kk * 256) >> 4);
                        const int s_first = d - NS > 1 ? d - NS : 1;
                        tc_mma_i8(dcol, da, db, (s == s_first && kk == 0) ? 0u : 1u);
                    }
                }
            }
        }
    }
}

// The same for a slice count known only at run time.
__device__ __forceinline__ void oz_issue_round_rt(int r, int ns, uint32_t tmem, uint64_t descA, uint64_t descB) {
    for (int u = 0; u < 8; ++u) {
        const int d = oz_round_d0(r) + u;
        if (d > ns + 1) break;
        const uint32_t dcol = tmem + (uint32_t)(r * 256 + u * 32);
        uint32_t acc = 0;
        const int s_lo = max(1, d - ns), s_hi = min(ns, d - 1);
        for (int s = s_lo; s <= s_hi; ++s) {
            const int t = d - s;
            for (int kk = 0; kk < 2; ++kk) {
                tc_mma_i8(dcol, descA + (uint64_t)(((s - 1) * OZ_A_BYTES + kk * 256) >> 4), descB + (uint64_t)(((t - 1) * OZ_B_BYTES + kk * 256) >> 4),
                          acc);
                acc = 1;
            }
        }
    }
}

__device__ void oz_producer(const OzArgs &a, OzShared &S, uint8_t *smA, uint8_t *smB, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    int I, J;
    oz_tile_at(t_begin, a.nI, a.nJ, I, J);
    auto issue_B = [&](int jb, int buf) {
        mbar_expect_tx(&S.barB[buf], (uint32_t)(a.ns * OZ_B_BYTES));
        for (int s = 0; s < a.ns; ++s)
            bulk_g2s(smB + (size_t)buf * OZ_MAX_SLICES * OZ_B_BYTES + (size_t)s * OZ_B_BYTES, a.slices + s * a.slice_stride + (long)jb * OZ_B_BYTES,
                     OZ_B_BYTES, &S.barB[buf]);
    };
    const uint64_t descA = oz_desc(smem_u32(smA));
    const uint64_t descB0 = oz_desc(smem_u32(smB)), descB1 = oz_desc(smem_u32(smB + (size_t)OZ_MAX_SLICES * OZ_B_BYTES));
    // phase parities, one bit per barrier of a pair; pending copies likewise
    uint32_t phA = 0, phB = 0, phFree = 0, phEmpty = 0, pendB = 0;
    int curA = -1;
    bool pendA = false;
    issue_B(J, 0);
    pendB = 1u;
    long n = 0;
    bool ok = true;
    for (long t = t_begin; t < t_end && ok; ++t, ++n) {
        const int b = (int)(n & 1);
        bool prev_done = n == 0; // tile n-1 complete (its B buffer and A free)
        if (I != curA) {
            if (!prev_done) {
                ok = oz_wait(&S.bfree[b ^ 1], (phFree >> (b ^ 1)) & 1u, abort_flag, a.err, 1);
                phFree ^= 1u << (b ^ 1);
                if (!ok) break;
                prev_done = true;
            }
            mbar_expect_tx(&S.barA, (uint32_t)(a.ns * OZ_A_BYTES));
            for (int s = 0; s < a.ns; ++s)
                bulk_g2s(smA + (size_t)s * OZ_A_BYTES, a.slices + s * a.slice_stride + (long)I * OZ_A_BYTES, OZ_A_BYTES, &S.barA);
            pendA = true;
            ok = oz_wait(&S.barA, phA, abort_flag, a.err, 2);
            phA ^= 1u;
            if (!ok) break;
            pendA = false;
            curA = I;
        }
        ok = oz_wait(&S.barB[b], (phB >> b) & 1u, abort_flag, a.err, 3);
        phB ^= 1u << b;
        if (!ok) break;
        pendB &= ~(1u << b);
        const uint64_t descB = b ? descB1 : descB0;
        for (int r = 0; r < 2 && ok; ++r) {
            ok = oz_wait(&S.tempty[r], ((phEmpty >> r) & 1u) ^ 1u, abort_flag, a.err, 4);
            phEmpty ^= 1u << r;
            if (!ok) break;
            tc_fence_after();
            if (a.ns == OZ_MAX_SLICES) {
                if (r == 0)
                    oz_issue_round<0, OZ_MAX_SLICES>(S.tmem, descA, descB);
                else
                    oz_issue_round<1, OZ_MAX_SLICES>(S.tmem, descA, descB);
            } else {
                oz_issue_round_rt(r, a.ns, S.tmem, descA, descB);
            }
            tc_commit(&S.tfull[r]);
        }
        if (!ok) break;
        tc_commit(&S.bfree[b]);
        // next tile's B into the other buffer, once tile n-1 has released it
        int In = I, Jn = J;
        oz_tile_next(a.nJ, In, Jn);
        if (t + 1 < t_end) {
            if (!prev_done) {
                ok = oz_wait(&S.bfree[b ^ 1], (phFree >> (b ^ 1)) & 1u, abort_flag, a.err, 1);
                phFree ^= 1u << (b ^ 1);
                if (!ok) break;
            }
            issue_B(Jn, b ^ 1);
            pendB |= 1u << (b ^ 1);
        }
        I = In;
        J = Jn;
    }
    // Before the CTA frees its tensor memory: every issued copy has landed
    // (bounded waits; an aborted CTA gives up after 2 s each).
    if (pendA) oz_wait(&S.barA, phA, abort_flag, a.err, 5);
    for (int b2 = 0; b2 < 2; ++b2)
        if ((pendB >> b2) & 1u) oz_wait(&S.barB[b2], (phB >> b2) & 1u, abort_flag, a.err, 5);
}

__device__ __forceinline__ double oz_combine(const int32_t *a0, const int32_t *a1, const int32_t *a2, const int32_t *a3, int c, double scale) {
    const long long v = ((long long)a0[c] << 21) + ((long long)a1[c] << 14) + ((long long)a2[c] << 7) + (long long)a3[c];
    return __ll2double_rn(v) * scale;
}

// 2^e as a double for -1022 <= e <= 1023 (built from its bits)
__device__ __forceinline__ double oz_pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Drains round R (its 8 diagonals from oz_round_d0(R)) for this thread's 16 columns
// into the dd accumulator (R = 0 sets it, R = 1 adds to it).
template <int R>
__device__ __forceinline__ void oz_drain(const OzArgs &a, uint32_t lane_base, double *acc_hi, double *acc_lo) {
    constexpr int D0 = oz_round_d0(R);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        double g[2][8];
#pragma unroll
        for (int gi = 0; gi < 2; ++gi) {
            int32_t v[4][8];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int slot = 4 * gi + u;
                if (D0 + slot <= a.ns + 1) {
                    tc_ld8(lane_base + (uint32_t)(R * 256 + slot * 32 + 8 * half), v[u]);
                } else {
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[u][c] = 0;
                }
            }
            tc_wait_ld();
            // group value (2^21 A_d + 2^14 A_d+1 + 2^7 A_d+2 + A_d+3) 2^-7(d+3)
            const double sc = oz_pow2(-7 * (D0 + 4 * gi + 3));
#pragma unroll
            for (int c = 0; c < 8; ++c) g[gi][c] = oz_combine(v[0], v[1], v[2], v[3], c, sc);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cc = 8 * half + c;
            double e, s = ddm::two_sum(g[0][c], g[1][c], e); // exact: 72 bits at most
            if (R == 0) {
                acc_hi[cc] = s;
                acc_lo[cc] = e;
            } else { // accurate dd addition of (s, e)
                double t1, t2, s2;
                double s1 = ddm::two_sum(acc_hi[cc], s, s2);
                t1 = ddm::two_sum(acc_lo[cc], e, t2);
                s2 += t1;
                s1 = ddm::fast_two_sum(s1, s2, s2);
                s2 += t2;
                acc_hi[cc] = ddm::fast_two_sum(s1, s2, acc_lo[cc]);
            }
        }
    }
}

// C(i, jb + c) -= 2^(e_i + e_j) acc[c] for c in [c0, c0 + 8) (cv: C prefetched)
__device__ __forceinline__ void oz_update8(const OzArgs &a, int i, int jb, int c0, int ei, const double *acc_hi, const double *acc_lo,
                                           const double2 *cv) {
    const int4 e0 = *reinterpret_cast<const int4 *>(a.exps + jb + c0), e1 = *reinterpret_cast<const int4 *>(a.exps + jb + c0 + 4);
    const int ej[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int j = jb + c0 + c;
        if (i < a.n && j < a.n && j <= i) {
            const int sc = ei + ej[c];
            dd_t p;
            if (sc >= -1022 && sc <= 1023) {
                const double pw = oz_pow2(sc);
                p = dd_make(acc_hi[c0 + c] * pw, acc_lo[c0 + c] * pw);
            } else {
                p = dd_make(ldexp(acc_hi[c0 + c], sc), ldexp(acc_lo[c0 + c], sc));
            }
            const dd_t r = dd_sub(dd_make(cv[c].x, cv[c].y), p);
            __stcs(reinterpret_cast<double2 *>(a.C + i + a.ldc * (long)j), make_double2(r.hi, r.lo));
        }
    }
}

__device__ __forceinline__ void oz_load8(const OzArgs &a, int i, int jb, int c0, double2 *cv) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int j = jb + c0 + c;
        cv[c] = (i < a.n && j < a.n && j <= i) ? __ldcs(reinterpret_cast<const double2 *>(a.C + i + a.ldc * (long)j)) : make_double2(0.0, 0.0);
    }
}

__device__ void oz_epilogue(const OzArgs &a, OzShared &S, long t_begin, long t_end) {
    volatile int *abort_flag = &S.abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, h = (warp - 1) >> 2;
    const int row = 32 * q + lane;
    const uint32_t lane_base = S.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(16 * h);
    int I, J;
    oz_tile_at(t_begin, a.nI, a.nJ, I, J);
    uint32_t ph = 0; // parity of tfull[0] and tfull[1] (they complete in step)
    // lane 0 waits; the warp follows its outcome (the tensor-memory loads
    // are warp-collective)
    auto wait_full = [&](int r) {
        int okw = 1;
        if (lane == 0) okw = oz_wait(&S.tfull[r], ph, abort_flag, a.err, 6) ? 1 : 0;
        return __shfl_sync(0xffffffffu, okw, 0) != 0;
    };
    auto release = [&](int r) {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.tempty[r]);
    };
    for (long t = t_begin; t < t_end; ++t) {
        const int i = I * OZ_ROWS_A + row;
        const int jb = J * OZ_COLS_B + 16 * h;
        const int ei = a.exps[i]; // scale exponent of the row (padded rows hold 0)
        double acc_hi[16], acc_lo[16];
        double2 cv[8];
        if (!wait_full(0)) break;
        tc_fence_after();
        oz_drain<0>(a, lane_base, acc_hi, acc_lo);
        release(0);
        if (!wait_full(1)) break;
        tc_fence_after();
        oz_drain<1>(a, lane_base, acc_hi, acc_lo);
        release(1);
        ph ^= 1u;
        // the next tile's MMAs run while C is read and written
        oz_load8(a, i, jb, 0, cv);
        oz_update8(a, i, jb, 0, ei, acc_hi, acc_lo, cv);
        oz_load8(a, i, jb, 8, cv);
        oz_update8(a, i, jb, 8, ei, acc_hi, acc_lo, cv);
        oz_tile_next(a.nJ, I, J);
    }
}

__global__ void __launch_bounds__(OZ_THREADS, 1) ozaki_syrk_kernel(OzArgs a) {
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
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.barB[b], 1);
            mbar_init(&S.bfree[b], 1);
            mbar_init(&S.tfull[b], 1);
            mbar_init(&S.tempty[b], 8);
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
        oz_epilogue(a, S, t_begin, t_end);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(512) : "memory");
    }
}

// Digits of 32 rows per CTA; warp c takes K bytes 16c..16c+15.
__global__ void __launch_bounds__(128) ozaki_split_kernel(const dd_t *P, long ldp, int n, int k, int ns, int8_t *slices, long slice_stride, int *exps) {
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
    int8_t *dst = slices + (long)(r >> 3) * 512 + c * 128 + (r & 7) * 16;
    for (int s = 0; s < ns; ++s) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const double d = rint(x[q].hi);
            w[q >> 2] |= ((uint32_t)((int)d) & 0xffu) << (8 * (q & 3));
            double err, sum = ddm::two_sum(x[q].hi - d, x[q].lo, err);
            x[q] = dd_make(sum * 128.0, err * 128.0);
        }
        *reinterpret_cast<uint4 *>(dst + (long)s * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

} // namespace

void ozaki_syrk_sub_lower(cudaStream_t st, const dd_t *P, long ldp, int n, int k, dd_t *C, long ldc, OzakiWork &w) {
    if (n <= 0 || k <= 0) return;
    if (k > OZ_K) throw Error(ERR_ARG, "ozaki: panel wider than 64 columns");
    if (w.slices_used < 8 || w.slices_used > OZ_MAX_SLICES) throw Error(ERR_ARG, "ozaki: slice count must be 8..16");
    const int rows = (int)(ceil_div(n, OZ_ROWS_A) * OZ_ROWS_A);
    if (rows > w.row_cap || !w.slices || !w.exps || !w.err) throw Error(ERR_ARG, "ozaki: workspace smaller than the panel");
    const long stride = (long)w.row_cap * OZ_K;
    ozaki_split_kernel<<<rows / 32, 128, 0, st>>>(P, ldp, n, k, w.slices_used, w.slices, stride, w.exps);
    CK_LAUNCH();
    OzArgs a;
    a.slices = w.slices;
    a.slice_stride = stride;
    a.exps = w.exps;
    a.C = C;
    a.ldc = ldc;
    a.n = n;
    a.ns = w.slices_used;
    a.nI = rows / OZ_ROWS_A;
    a.nJ = (int)ceil_div(n, OZ_COLS_B);
    a.err = w.err;
    long tiles = 0;
    for (int I = 0; I < a.nI; ++I) tiles += std::min(4L * (I + 1), (long)a.nJ);
    a.tiles = tiles;
    static thread_local int sms[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &sm = sms[dev & 63];
    if (sm == 0) {
        CK(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(ozaki_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)OZ_SMEM));
    }
    const int grid = (int)std::min<long>(sm, tiles);
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
    if (err != 0) throw Error(ERR_CUDA, "ozaki: a tensor-core split update gave up waiting (code " + std::to_string(err) + ")");
}

} // namespace sddd
