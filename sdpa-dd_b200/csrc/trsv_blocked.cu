// Blocked dd triangular solves for the tensor-core split form.
//
// The split form's Cholesky factor of B is not the reference's bit pattern
// (its trailing updates round once per panel), so its solves need not keep
// Rtrsv's per-entry chain either.  Here the 64 x 64 diagonal blocks of L
// are inverted once per factorisation (trsv_diag_inverse, one CTA per
// block, all blocks at once), and a solve is a wavefront of 64-entry
// blocks in which no step divides or waits on a single entry:
//   'N'  v_c = b_c - sum_{p<c} L(c,p) x_p,   x_c = W_c v_c
//   'T'  v_c = b_c - sum_{p>c} L(p,c)^T x_p, x_c = W_c^T v_c   (W_c = L(c,c)^-1)
// followed by one step of iterative refinement against L(c,c) itself,
// x_c += W_c (v_c - L(c,c) x_c) (transposed for 'T'), which brings the
// block's solve to the accuracy of a substitution even where L(c,c) is far
// from orthogonal (the Schur matrix near the optimum).
// One cooperative launch per solve: CTA k owns blocks k, k + G, ... (in
// solve order).  For each of its blocks it streams the tiles L(c,p) (or
// L(p,c)) and finally W_c into shared memory with bulk copies (one copy per
// tile column of up to 1 KB, three tiles in flight, completion on an
// mbarrier), waits for block p's flag (release/acquire, bounded), and all
// 256 threads multiply: thread (r, q) sums the 16 products of row r (or
// column r) in quarter q of the tile into its own running dd sum, so a tile
// costs a 16-step chain and the critical path per block is one tile and
// three 64 x 64 products (W_c, L(c,c), W_c), each a 16-step chain and a
// 4-way combination.  L is read once per solve.
//
// Every wait is bounded (the solve's wait budget, 2 s by default); a CTA
// that gives up records the awaited block in the error word (read by
// trsv_check), waits (bounded) for its copies in flight and returns.
#include "blas.h"
#include "bulk.cuh"
#include "devops.cuh"
#include "prof.h"

namespace sddd {

namespace {

constexpr int TB = 64;           // block order
constexpr int TB_LD = 65;        // padded leading dimension of a tile in shared memory
constexpr int TB_STAGES = 3;     // tiles in flight per CTA
constexpr int TB_THREADS = 256;  // (row, quarter) pairs of a tile
constexpr int TB_TILE = TB * TB_LD; // double2 per stage

struct TbShared {
    uint64_t bar[TB_STAGES];
    int fail;
    long fail_at; // the first tile not consumed when the CTA gave up
};
constexpr size_t TB_SMEM = sizeof(double2) * ((size_t)TB_STAGES * TB_TILE + 3 * TB + 4 * TB) + 128;
static_assert(TB_SMEM <= 232448, "blocked solve: shared memory above the per-CTA limit");

struct TbArgs {
    const dd_t *L;
    long lda;
    const dd_t *W; // nblk tiles of TB x TB (leading dimension TB): L(c,c)^-1, lower
    int n, nblk, epoch, trans; // trans: 0 'N', 1 'T'
    dd_t *x;
    int *flags, *err;
    unsigned long long wait_ns;
    int withhold; // a block whose flag is never published (-1: none)
};

// The k-th tile block c reads: 'N' L(c, k) for k < c, 'T' L(nblk-1-k, c)
// for k < nblk-1-c; then L(c,c) and W_c (ntiles = 'N' c + 2, 'T' nblk-c+1).  Column j of the tile (rows
// r0 .. r0+rows-1 of column c0 + j) goes to T + j * TB_LD.
struct TileSrc {
    const dd_t *base; // column 0, row 0
    long ld;          // between columns
    int rows, cols;
};

__device__ __forceinline__ TileSrc tb_tile(const TbArgs &a, int c, int k, int ntiles) {
    const int nbc = min(TB, a.n - c * TB);
    TileSrc s;
    if (k == ntiles - 1) {
        s.base = a.W + (long)c * TB * TB;
        s.ld = TB;
        s.rows = nbc;
        s.cols = nbc;
    } else if (k == ntiles - 2) {
        s.base = a.L + (long)c * TB + a.lda * (long)(c * TB);
        s.ld = a.lda;
        s.rows = nbc;
        s.cols = nbc;
    } else if (a.trans == 0) {
        s.base = a.L + (long)c * TB + a.lda * (long)(k * TB);
        s.ld = a.lda;
        s.rows = nbc;
        s.cols = TB; // p = k < c: a full block
    } else {
        const int p = a.nblk - 1 - k;
        s.base = a.L + (long)p * TB + a.lda * (long)(c * TB);
        s.ld = a.lda;
        s.rows = min(TB, a.n - p * TB);
        s.cols = nbc;
    }
    return s;
}

// Warp 0: the copies of one tile into stage buffer T (lane l copies
// columns l and l + 32).
__device__ __forceinline__ void tb_issue(const TileSrc &s, double2 *T, uint64_t *bar, int lane) {
    if (lane == 0) mbar_expect_tx(bar, (uint32_t)(s.rows * s.cols * (int)sizeof(double2)));
    __syncwarp();
    for (int j = lane; j < s.cols; j += 32) bulk_g2s(T + j * TB_LD, s.base + s.ld * (long)j, (uint32_t)(s.rows * sizeof(double2)), bar);
}

// Bounded wait on a stage's mbarrier (thread 0 only).
__device__ bool tb_wait_bar(uint64_t *bar, uint32_t parity, unsigned long long wait_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > wait_ns) return false;
    return true;
}

__device__ __forceinline__ int tb_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void tb_st_release(int *p, int v) { asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }

// Bounded wait for block p's flag (thread 0 only).
__device__ bool tb_wait_flag(const TbArgs &a, int p) {
    const unsigned long long t0 = globaltimer_ns();
    while (tb_ld_acquire(a.flags + p) != a.epoch) {
        if (tb_ld_acquire(a.err) != 0 || globaltimer_ns() - t0 > a.wait_ns) return false;
        __nanosleep(20);
    }
    return true;
}

__device__ __forceinline__ dd_t sm_dd(const double2 *T, int i) {
    const double2 v = T[i];
    return dd_make(v.x, v.y);
}

__device__ __forceinline__ double2 tb_pack(dd_t v) { return make_double2(v.hi, v.lo); }

// The four quarters' partial sums of entry i: (p0 + p1) + (p2 + p3).
__device__ __forceinline__ dd_t tb_sum4(const double2 *part, int i) {
    return dd_add(dd_add(sm_dd(part, i), sm_dd(part, TB + i)), dd_add(sm_dd(part, 2 * TB + i), sm_dd(part, 3 * TB + i)));
}

// Thread (r, q)'s part of row r of M y ('N') or of column r of M^T y ('T')
// over the terms t2 of quarter q (t2 < nb); with lower, only M(i,j), i >= j.
__device__ __forceinline__ double2 tb_matvec(const double2 *M, const double2 *y, int r, int q, int nb, int trans, bool lower) {
    dd_t w = dd_zero();
    if (r < nb) {
        int lo = q * 16, hi = min(lo + 16, nb);
        if (trans == 0) {
            if (lower) hi = min(hi, r + 1);
            for (int t2 = lo; t2 < hi; ++t2) w = dd_add(w, dd_mul(sm_dd(M, r + t2 * TB_LD), sm_dd(y, t2)));
        } else {
            if (lower) lo = max(lo, r);
            for (int t2 = lo; t2 < hi; ++t2) w = dd_add(w, dd_mul(sm_dd(M, t2 + r * TB_LD), sm_dd(y, t2)));
        }
    }
    return tb_pack(w);
}

__global__ void __launch_bounds__(TB_THREADS, 1) trsv_blocked_kernel(TbArgs a) {
    extern __shared__ __align__(128) double2 tb_sm[];
    double2 *tiles = tb_sm;                      // TB_STAGES x TB_TILE
    double2 *xs = tiles + TB_STAGES * TB_TILE;   // TB: x of block p, then the residual v of block c
    double2 *x0 = xs + TB;                       // TB: W_c v
    double2 *rs = x0 + TB;                       // TB: v - L(c,c) x0
    double2 *part = rs + TB;                     // 4 x TB partial sums
    TbShared &S = *reinterpret_cast<TbShared *>(part + 4 * TB);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r = tid & (TB - 1), q = tid >> 6; // row (or column) of the tile, quarter of its other index
    if (tid == 0) {
        for (int s = 0; s < TB_STAGES; ++s) mbar_init(&S.bar[s], 1);
        S.fail = 0;
        mbar_init_fence();
    }
    __syncthreads();
    long g = 0;        // tiles consumed by this CTA (stage and parity)
    long issued = 0;   // tiles whose copies this CTA issued
    for (int k = blockIdx.x; k < a.nblk; k += gridDim.x) {
        const int c = a.trans == 0 ? k : a.nblk - 1 - k;
        const int nbc = min(TB, a.n - c * TB);
        const int ntiles = a.trans == 0 ? c + 2 : a.nblk - c + 1;
        if (warp == 0)
            for (int t = 0; t < TB_STAGES && t < ntiles; ++t) {
                const int st = (int)((g + t) % TB_STAGES);
                tb_issue(tb_tile(a, c, t, ntiles), tiles + st * TB_TILE, &S.bar[st], lane);
            }
        issued = g + min(TB_STAGES, ntiles);
        dd_t acc = dd_zero();
        for (int t = 0; t < ntiles; ++t) {
            const long gt = g + t;
            const int st = (int)(gt % TB_STAGES);
            const double2 *T = tiles + st * TB_TILE;
            const bool last = t == ntiles - 1;
            const int p = a.trans == 0 ? t : a.nblk - 1 - t; // block whose x this tile multiplies
            if (tid == 0) {
                bool ok = t >= ntiles - 2 || tb_wait_flag(a, p);
                int code = p + 1; // the block waited for
                if (ok) {
                    ok = tb_wait_bar(&S.bar[st], (uint32_t)((gt / TB_STAGES) & 1), a.wait_ns);
                    code = c + 1; // a tile of this block never landed
                }
                if (!ok) {
                    S.fail = 1;
                    S.fail_at = gt;
                    atomicCAS(a.err, 0, code);
                }
            }
            __syncthreads();
            if (S.fail) break;
            if (t < ntiles - 2) {
                const int nbp = min(TB, a.n - p * TB);
                if (tid < TB) xs[tid] = tid < nbp ? __ldcg(reinterpret_cast<const double2 *>(a.x) + (long)p * TB + tid) : make_double2(0.0, 0.0);
                __syncthreads();
                // rows (or columns) r of block c, terms t2 of quarter q
                const int kn = a.trans == 0 ? TB : nbp;
                if (r < nbc) {
                    const int lo = q * 16, hi = min(lo + 16, kn);
                    if (a.trans == 0) {
                        for (int t2 = lo; t2 < hi; ++t2) acc = dd_add(acc, dd_mul(sm_dd(T, r + t2 * TB_LD), sm_dd(xs, t2)));
                    } else {
                        for (int t2 = lo; t2 < hi; ++t2) acc = dd_add(acc, dd_mul(sm_dd(T, t2 + r * TB_LD), sm_dd(xs, t2)));
                    }
                }
            } else if (last) {
                // T = W_c; the previous stage holds L(c,c)
                const double2 *Lc = tiles + (int)((gt - 1) % TB_STAGES) * TB_TILE;
                // residual of block c: v = b_c - (sum of the four partial sums)
                part[q * TB + r] = make_double2(acc.hi, acc.lo);
                __syncthreads();
                if (tid < TB) {
                    dd_t v = dd_zero();
                    if (tid < nbc) v = dd_sub(ld_dd(a.x + (long)c * TB + tid), tb_sum4(part, tid));
                    xs[tid] = make_double2(v.hi, v.lo);
                }
                __syncthreads();
                // x0 = W_c v ('N') or W_c^T v ('T')
                part[q * TB + r] = tb_matvec(T, xs, r, q, nbc, a.trans, false);
                __syncthreads();
                if (tid < TB) x0[tid] = tid < nbc ? tb_pack(tb_sum4(part, tid)) : make_double2(0.0, 0.0);
                __syncthreads();
                // rs = v - L(c,c) x0 (lower triangle only: the strict upper
                // part of the tile holds the Schur matrix's own entries)
                part[q * TB + r] = tb_matvec(Lc, x0, r, q, nbc, a.trans, true);
                __syncthreads();
                if (tid < TB) rs[tid] = tid < nbc ? tb_pack(dd_sub(sm_dd(xs, tid), tb_sum4(part, tid))) : make_double2(0.0, 0.0);
                __syncthreads();
                // x = x0 + W_c rs
                part[q * TB + r] = tb_matvec(T, rs, r, q, nbc, a.trans, false);
                __syncthreads();
                if (tid < nbc) st_dd(a.x + (long)c * TB + tid, dd_add(sm_dd(x0, tid), tb_sum4(part, tid)));
                __threadfence();
            }
            __syncthreads(); // stage st and xs are free again
            if (warp == 0 && t + TB_STAGES < ntiles) {
                const int sn = (int)((gt + TB_STAGES) % TB_STAGES);
                tb_issue(tb_tile(a, c, t + TB_STAGES, ntiles), tiles + sn * TB_TILE, &S.bar[sn], lane);
            }
            if (t + TB_STAGES < ntiles) issued = gt + TB_STAGES + 1;
        }
        if (S.fail) {
            // the copies issued but not consumed land (bounded waits)
            // before the CTA exits and its shared memory is reused
            if (tid == 0)
                for (long u = S.fail_at; u < issued; ++u) tb_wait_bar(&S.bar[u % TB_STAGES], (uint32_t)((u / TB_STAGES) & 1), a.wait_ns);
            __syncthreads();
            return;
        }
        if (tid == 0 && c != a.withhold) tb_st_release(a.flags + c, a.epoch);
        g += ntiles;
    }
}

// W_c = L(c,c)^-1 for every diagonal block: one CTA per block; thread j
// solves L(c,c) w = e_j for column j (rows j..nb-1, in order, into shared
// memory), with the reciprocals of the pivots computed once.
constexpr size_t TB_INV_SMEM = sizeof(double2) * (2 * (size_t)TB_TILE + TB);

__global__ void __launch_bounds__(TB) trsv_diag_inverse_kernel(const dd_t *L, long lda, int n, dd_t *W) {
    extern __shared__ __align__(16) double2 inv_sm[];
    double2 *T = inv_sm;             // L(c,c), lower part
    double2 *Wt = inv_sm + TB_TILE;  // column j of the inverse at Wt + j * TB_LD
    double2 *rp = Wt + TB_TILE;      // 1 / L(i,i)
    const int c = blockIdx.x, j = threadIdx.x;
    const int nb = min(TB, n - c * TB);
    const dd_t *D = L + (long)c * TB + lda * (long)(c * TB);
    for (int col = 0; col < nb; ++col)
        if (j < nb && j >= col) T[j + col * TB_LD] = *reinterpret_cast<const double2 *>(D + j + lda * (long)col);
    __syncthreads();
    if (j < nb) {
        const dd_t rj = dd_div(dd_make(1.0, 0.0), sm_dd(T, j + j * TB_LD));
        rp[j] = make_double2(rj.hi, rj.lo);
    }
    __syncthreads();
    double2 *w = Wt + j * TB_LD;
    if (j < nb) {
        w[j] = rp[j];
        for (int i = j + 1; i < nb; ++i) {
            dd_t s = dd_zero();
            for (int k = j; k < i; ++k) s = dd_add(s, dd_mul(sm_dd(T, i + k * TB_LD), sm_dd(w, k)));
            const dd_t v = dd_mul(dd_neg(s), sm_dd(rp, i)); // w_i = -s / L(i,i)
            w[i] = make_double2(v.hi, v.lo);
        }
    }
    __syncthreads();
    // W_c column-major, leading dimension TB, zero above the diagonal and
    // outside the block; row-coalesced stores
    dd_t *Wc = W + (long)c * TB * TB;
    for (int col = 0; col < TB; ++col) {
        const dd_t v = (col < nb && j < nb && j >= col) ? sm_dd(Wt, j + col * TB_LD) : dd_zero();
        st_dd(Wc + j + (long)TB * col, v);
    }
}

} // namespace

void trsv_diag_inverse(cudaStream_t st, const dd_t *L, long lda, int n, dd_t *W) {
    if (n <= 0) return;
    PROF_SCOPE("trsv_diag_inverse", st);
    static thread_local bool attr[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (!attr[dev & 63]) {
        CK(cudaFuncSetAttribute(trsv_diag_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TB_INV_SMEM));
        attr[dev & 63] = true;
    }
    trsv_diag_inverse_kernel<<<ceil_div(n, TB), TB, TB_INV_SMEM, st>>>(L, lda, n, W);
    CK_LAUNCH();
}

void trsv_blocked(cudaStream_t st, char trans, const dd_t *L, long lda, int n, const dd_t *W, dd_t *x, TrsvSync &sync) {
    if (n <= 0) return;
    if (trans != 'N' && trans != 'T') throw Error(ERR_ARG, "trsv_blocked: trans must be 'N' or 'T'");
    const int nblk = ceil_div(n, TB);
    if (nblk > sync.capacity || !sync.flags) throw Error(ERR_ARG, "trsv_blocked: progress flags hold fewer blocks than the solve needs");
    PROF_SCOPE("trsv", st);
    if (++sync.epoch <= 0) sync.epoch = 1;
    TbArgs a{L, lda, W, n, nblk, sync.epoch, trans == 'N' ? 0 : 1, x, sync.flags, sync.flags + sync.capacity, sync.wait_ns, sync.withhold};
    static thread_local int cap[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &cp = cap[dev & 63];
    if (cp == 0) {
        int sms = 0, per = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(trsv_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TB_SMEM));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trsv_blocked_kernel, TB_THREADS, TB_SMEM));
        if (per < 1) throw Error(ERR_CUDA, "trsv_blocked: the kernel does not fit on an SM");
        cp = per * sms;
    }
    const int grid = std::min(nblk, cp);
    void *args[] = {&a};
    CK(cudaLaunchCooperativeKernel((const void *)trsv_blocked_kernel, grid, TB_THREADS, args, TB_SMEM, st));
    CK_LAUNCH();
}

} // namespace sddd
