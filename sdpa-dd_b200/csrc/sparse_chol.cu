// Sparse Schur complement on the device (see sparse_chol.h).
//
// Storage.  The factor of the reordered B lives in the 64 x 64 tiles of its
// lower triangle that hold an entry of the symbolic factor; entry (a, b),
// a >= b, is the reference's sparse_bMat entry of row b, column a
// (Newton::initialize_sparse_bMat, sdpa_newton.cpp:225-340).  Each tile
// carries 64 structure words (word j: the rows of column j that belong to
// the symbolic factor), so that every kernel applies exactly the updates the
// reference applies and no other.
//
// Factor (Lal::getCholesky(SparseMatrix&, int*), sdpa_linear.cpp:353-395).
// Per pivot b in ascending order the reference sets d_b = 1 / sqrt(B(b,b))
// (0 when B(b,b) < 0), scales column b by it ("*="), then for every pair
// r <= a of struct(b) subtracts L(r,b) * L(a,b) from entry (a, r).  Each
// entry thus sees its updates in ascending pivot order, one dd multiply and
// one dd subtract each, and is scaled once, when its column becomes the
// pivot.  Here, per panel J of 64 pivots:
//   sp_panel_kernel   one CTA per tile of column block J (the diagonal
//                     tile first): every CTA factors the diagonal tile in
//                     shared memory (pivots in order, the next column's
//                     pivot chain beside the other columns' updates), and
//                     CTA k > 0 carries its own tile below with the same
//                     pivots;
//   sp_update_kernel  every tile (I, K), K > J, that some column of J
//                     reaches in both I and K: entry (a, r) -= L(r,b) L(a,b)
//                     for the columns b of J ascending, where both are in
//                     the structure.
// Every entry keeps the reference's chain of operations, so the factor is
// the reference's bit for bit.
//
// Solves (Lal::solveSystems(Vector&, SparseMatrix&, Vector&),
// sdpa_linear.cpp:654-810, the loop that is compiled): forward over the
// entries in storage order, x(b) *= d_b at the diagonal and x(a) -= L(a,b)
// x(b) below it; backward in reverse storage order, x(b) -= L(a,b) x(a) for
// a descending, then x(b) *= d_b.  One cooperative launch per direction:
// CTA c owns row block c (forward) or the mirror order (backward), walks
// only the tiles of its row (column) block, and waits for the blocks it
// reads through per-block flags with a bounded wait, as the dense
// triangular solves do.
#include "sparse_chol.h"

#include <algorithm>

#include "prof.h"

namespace sddd {

constexpr int SPL = SP_T + 1; // padded leading dimension in shared memory
constexpr int SP_THREADS = 256;
constexpr int SP_UPD_SPLIT = 4; // CTAs per trailing-update tile (16 columns each)
constexpr size_t SP_TILE_SMEM = sizeof(double2) * SP_T * SPL;
constexpr size_t SP_TWO_TILES = 2 * SP_TILE_SMEM;
constexpr size_t SP_SOLVE_SMEM = 2 * SP_TILE_SMEM + sizeof(double2) * SP_T;

__device__ __forceinline__ bool bit64(unsigned long long w, int i) { return (w >> i) & 1ull; }
__device__ __forceinline__ dd_t sm_dd(const double2 *S, int i, int j) {
    const double2 v = S[i + SPL * j];
    return dd_make(v.x, v.y);
}
__device__ __forceinline__ void sm_st(double2 *S, int i, int j, dd_t v) { S[i + SPL * j] = make_double2(v.hi, v.lo); }

// Tile (contiguous 64 x 64, column-major) into shared memory with leading
// dimension 65: threads [t0, t0 + nt) put their 16-byte copies in flight
// and wait for them; the caller's barrier publishes the tile.
__device__ __forceinline__ void sp_load_tile(double2 *S, const dd_t *T, int t0, int nt) {
    for (int e = t0; e < SP_T * SP_T; e += nt) {
        const int i = e & (SP_T - 1), j = e >> 6;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(S + i + SPL * j)), "l"(T + e) : "memory");
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void sp_store_tile(dd_t *T, const double2 *S, int t0, int nt) {
    for (int e = t0; e < SP_T * SP_T; e += nt) {
        const int i = e & (SP_T - 1), j = e >> 6;
        *reinterpret_cast<double2 *>(T + e) = S[i + SPL * j];
    }
}

// ------------------------------------------------------------ entries
// Tile entries from B through the order: (a, b) -> B(order[a], order[b])
// for the entries of the structure, zero elsewhere.
__global__ void sp_gather_B_kernel(const dd_t *B, int m, const int *order, const int *tIJ, const unsigned long long *mask, dd_t *tiles) {
    const int t = blockIdx.x;
    const int I = tIJ[2 * t], J = tIJ[2 * t + 1];
    for (int e = threadIdx.x; e < SP_T * SP_T; e += blockDim.x) {
        const int i = e & (SP_T - 1), j = e >> 6;
        const int a = I * SP_T + i, b = J * SP_T + j;
        dd_t v = dd_zero();
        if (a < m && b < m && bit64(mask[(long)t * SP_T + j], i)) v = ld_dd(B + order[a] + (long)m * order[b]);
        st_dd(tiles + (long)t * SP_T * SP_T + e, v);
    }
}

// Entries of the reference layout into the (zeroed) tiles, and back.
__global__ void sp_scatter_kernel(const dd_t *vals, const int *ent_b, const int *ent_a, long nnz, const int *tile_of, int nblk, dd_t *tiles) {
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= nnz) return;
    const int b = ent_b[q], a = ent_a[q];
    const int t = tile_of[a / SP_T + (long)nblk * (b / SP_T)];
    st_dd(tiles + (long)t * SP_T * SP_T + (a % SP_T) + SP_T * (b % SP_T), ld_dd(vals + q));
}
__global__ void sp_gather_kernel(const dd_t *tiles, const int *ent_b, const int *ent_a, long nnz, const int *tile_of, int nblk, dd_t *vals) {
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= nnz) return;
    const int b = ent_b[q], a = ent_a[q];
    const int t = tile_of[a / SP_T + (long)nblk * (b / SP_T)];
    st_dd(vals + q, ld_dd(tiles + (long)t * SP_T * SP_T + (a % SP_T) + SP_T * (b % SP_T)));
}

// ------------------------------------------------------------ panel
// CTA 0: the diagonal tile of panel J; CTA k > 0: the diagonal tile again
// (identical arithmetic) and below-diagonal tile col_tiles[k - 1].  Every
// CTA reads the unfactored diagonal tile at its start, so the factored one
// is written back by the CTA that finishes last (counted in done[J], which
// it resets for the next factorisation).
// Step k (one barrier): warp 0 takes column k+1 through pivot k's update,
// its own pivot (1/sqrt) and its scaling, while warps 1.. apply pivot k's
// update to columns k+2.. (one column per warp at a time, rows over the
// lanes); so the chain of pivots runs beside the bulk of the updates and
// every entry still sees pivot k's update before pivot k+1's.
constexpr int SP_PANEL_THREADS = 512;
__global__ void __launch_bounds__(SP_PANEL_THREADS) sp_panel_kernel(dd_t *tiles, const unsigned long long *mask, int m, int J, int diag_t,
                                                                    const int *col_tiles, int *done) {
    extern __shared__ double2 sp_sm[];
    double2 *D = sp_sm;
    double2 *U = sp_sm + SP_T * SPL; // used only when the CTA has a tile below (ut >= 0, mu != 0)
    __shared__ unsigned long long md[SP_T], mu[SP_T];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int nb = min(SP_T, m - J * SP_T);
    const int ut = blockIdx.x > 0 ? col_tiles[blockIdx.x - 1] : -1;
    sp_load_tile(D, tiles + (long)diag_t * SP_T * SP_T, tid, blockDim.x);
    if (ut >= 0) sp_load_tile(U, tiles + (long)ut * SP_T * SP_T, tid, blockDim.x);
    if (tid < SP_T) {
        md[tid] = mask[(long)diag_t * SP_T + tid];
        mu[tid] = ut >= 0 ? mask[(long)ut * SP_T + tid] : 0ull;
    }
    __syncthreads();
    // warp 0: column c's pivot d_c = 1/sqrt(B(c,c)) (0 for a negative
    // pivot) and the scaling of column c by it
    auto pivot = [&](int c) {
        double ih = 0.0, il = 0.0;
        if (lane == 0) {
            const dd_t d = sm_dd(D, c, c);
            const dd_t inv = dd_lt_d(d, 0.0) ? dd_zero() : dd_div(dd_from(1.0), dd_sqrt(d));
            sm_st(D, c, c, inv);
            ih = inv.hi;
            il = inv.lo;
        }
        const dd_t inv = dd_make(__shfl_sync(0xffffffffu, ih, 0), __shfl_sync(0xffffffffu, il, 0));
        const unsigned long long cc = md[c], uc = mu[c];
        for (int i = lane; i < SP_T; i += 32) {
            if (i > c && bit64(cc, i)) sm_st(D, i, c, dd_muleq(sm_dd(D, i, c), inv));
            if (bit64(uc, i)) sm_st(U, i, c, dd_muleq(sm_dd(U, i, c), inv));
        }
        __syncwarp();
    };
    // pivot k's update of column r (r in struct(k)): entry (i, r) -= L(r,k) L(i,k)
    auto apply = [&](int k, int r, unsigned long long ck, unsigned long long uk) {
        const dd_t lrk = sm_dd(D, r, k);
        for (int i = lane; i < SP_T; i += 32) {
            if (i >= r && bit64(ck, i)) sm_st(D, i, r, dd_sub(sm_dd(D, i, r), dd_mul(lrk, sm_dd(D, i, k))));
            if (bit64(uk, i)) sm_st(U, i, r, dd_sub(sm_dd(U, i, r), dd_mul(lrk, sm_dd(U, i, k))));
        }
    };
    if (warp == 0 && nb > 0) pivot(0);
    __syncthreads();
    for (int k = 0; k + 1 < nb; ++k) {
        const unsigned long long ck = md[k], uk = mu[k];
        if (warp == 0) {
            if (bit64(ck, k + 1)) apply(k, k + 1, ck, uk);
            __syncwarp();
            pivot(k + 1);
        } else {
            for (int r = k + 1 + warp; r < nb; r += nw - 1)
                if (bit64(ck, r)) apply(k, r, ck, uk);
        }
        __syncthreads();
    }
    if (ut >= 0) sp_store_tile(tiles + (long)ut * SP_T * SP_T, U, tid, blockDim.x);
    __shared__ int last;
    if (tid == 0) last = atomicAdd(done + J, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (last) {
        sp_store_tile(tiles + (long)diag_t * SP_T * SP_T, D, tid, blockDim.x);
        if (tid == 0) done[J] = 0;
    }
}

// ------------------------------------------------------------ update
// upd: (target, source (I, J), source (K, J)) per target; CTA q * 4 + p
// updates the 16 columns [16p, 16p + 16) of target q.
__global__ void __launch_bounds__(SP_THREADS) sp_update_kernel(dd_t *tiles, const unsigned long long *mask, const int *upd, int nbJ) {
    extern __shared__ double2 sp_sm[];
    double2 *SI = sp_sm;
    double2 *SK = sp_sm + SP_T * SPL;
    __shared__ unsigned long long mI[SP_T], mK[SP_T];
    const int tid = threadIdx.x;
    const int q = blockIdx.x / SP_UPD_SPLIT, part = blockIdx.x % SP_UPD_SPLIT;
    const int tt = upd[3 * q], sI = upd[3 * q + 1], sK = upd[3 * q + 2];
    const bool diag_target = sI == sK;
    sp_load_tile(SI, tiles + (long)sI * SP_T * SP_T, tid, blockDim.x);
    if (!diag_target) sp_load_tile(SK, tiles + (long)sK * SP_T * SP_T, tid, blockDim.x);
    if (tid < SP_T) {
        mI[tid] = mask[(long)sI * SP_T + tid];
        mK[tid] = mask[(long)sK * SP_T + tid];
    }
    __syncthreads();
    const double2 *SKp = diag_target ? SI : SK;
    dd_t *T = tiles + (long)tt * SP_T * SP_T;
    constexpr int COLS = SP_T / SP_UPD_SPLIT;
    for (int e = tid; e < SP_T * COLS; e += blockDim.x) {
        const int i = e & (SP_T - 1), k = part * COLS + (e >> 6);
        if (diag_target && i < k) continue;
        dd_t v = ld_dd(T + i + SP_T * k);
        for (int j = 0; j < nbJ; ++j)
            if (bit64(mI[j], i) && bit64(mK[j], k)) v = dd_sub(v, dd_mul(sm_dd(SKp, k, j), sm_dd(SI, i, j)));
        st_dd(T + i + SP_T * k, v);
    }
}

// ------------------------------------------------------------ solves
struct SpSolveArgs {
    const dd_t *tiles;
    const unsigned long long *mask;
    const int *tIJ, *row_ptr, *row_tiles, *col_ptr, *col_tiles, *diag;
    int m, nblk, epoch;
    dd_t *x;
    int *flags, *err;
    unsigned long long wait_ns;
    int withhold;
};

__device__ __forceinline__ int sp_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void sp_st_release(int *p, int v) { asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
__device__ __forceinline__ unsigned long long sp_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Lane 0 waits (bounded) for block blk's flag; every lane gets the outcome.
__device__ bool sp_wait(const SpSolveArgs &a, int blk) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long t0 = sp_ns();
        unsigned iter = 0;
        while (sp_ld_acquire(a.flags + blk) != a.epoch) {
            if (sp_ld_acquire(a.err) != 0 || ++iter > (1u << 26) || sp_ns() - t0 > a.wait_ns) {
                atomicCAS(a.err, 0, blk + 1);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
    }
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
__device__ __forceinline__ dd_t sp_shfl(dd_t v, int src) {
    return dd_make(__shfl_sync(0xffffffffu, v.hi, src), __shfl_sync(0xffffffffu, v.lo, src));
}
__device__ __forceinline__ dd_t sp_ldcg(const dd_t *p) {
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return dd_make(v.x, v.y);
}

__global__ void __launch_bounds__(SP_THREADS) sp_fwd_kernel(SpSolveArgs a) {
    extern __shared__ double2 sp_sm[];
    double2 *xs = sp_sm + 2 * SP_T * SPL;
    __shared__ unsigned long long msk[2][SP_T];
    __shared__ int fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    for (int c = blockIdx.x; c < a.nblk; c += gridDim.x) {
        const int r0 = c * SP_T;
        const int q0 = a.row_ptr[c], noff = a.row_ptr[c + 1] - q0;
        dd_t v0 = dd_zero(), v1 = dd_zero();
        if (warp == 0) {
            if (r0 + lane < a.m) v0 = ld_dd(a.x + r0 + lane);
            if (r0 + 32 + lane < a.m) v1 = ld_dd(a.x + r0 + 32 + lane);
        }
        int t = noff > 0 ? a.row_tiles[q0] : a.diag[c];
        sp_load_tile(sp_sm, a.tiles + (long)t * SP_T * SP_T, tid, blockDim.x);
        if (tid < SP_T) msk[0][tid] = a.mask[(long)t * SP_T + tid];
        __syncthreads();
        for (int s = 0; s < noff; ++s) {
            const int buf = s & 1;
            const double2 *T = sp_sm + buf * SP_T * SPL;
            const int J = a.tIJ[2 * t + 1];
            const int tn = s + 1 < noff ? a.row_tiles[q0 + s + 1] : a.diag[c];
            if (warp != 0) {
                sp_load_tile(sp_sm + (buf ^ 1) * SP_T * SPL, a.tiles + (long)tn * SP_T * SP_T, tid - 32, blockDim.x - 32);
                if (tid >= 32 && tid < 32 + SP_T) msk[buf ^ 1][tid - 32] = a.mask[(long)tn * SP_T + tid - 32];
            } else if (!sp_wait(a, J)) {
                if (lane == 0) fail = 1;
            } else {
                const int jb = min(SP_T, a.m - J * SP_T);
                if (lane < jb) {
                    const dd_t xa = sp_ldcg(a.x + J * SP_T + lane);
                    xs[lane] = make_double2(xa.hi, xa.lo);
                }
                if (32 + lane < jb) {
                    const dd_t xb = sp_ldcg(a.x + J * SP_T + 32 + lane);
                    xs[32 + lane] = make_double2(xb.hi, xb.lo);
                }
                __syncwarp();
                for (int j = 0; j < jb; ++j) {
                    const unsigned long long w = msk[buf][j];
                    if (!w) continue;
                    const dd_t xt = dd_make(xs[j].x, xs[j].y);
                    if (bit64(w, lane)) v0 = dd_sub(v0, dd_mul(sm_dd(T, lane, j), xt));
                    if (bit64(w, 32 + lane)) v1 = dd_sub(v1, dd_mul(sm_dd(T, 32 + lane, j), xt));
                }
                __syncwarp();
            }
            __syncthreads();
            if (fail) return;
            t = tn;
        }
        if (warp == 0) {
            const int buf = noff & 1;
            const double2 *T = sp_sm + buf * SP_T * SPL;
            const int nb = min(SP_T, a.m - r0);
            for (int j = 0; j < nb; ++j) {
                const int owner = j & 31;
                dd_t mine = j < 32 ? v0 : v1;
                if (lane == owner) {
                    mine = dd_muleq(mine, sm_dd(T, j, j));
                    if (j < 32) v0 = mine;
                    else v1 = mine;
                }
                const dd_t xt = sp_shfl(mine, owner);
                const unsigned long long w = msk[buf][j];
                if (lane > j && bit64(w, lane)) v0 = dd_sub(v0, dd_mul(sm_dd(T, lane, j), xt));
                if (32 + lane > j && bit64(w, 32 + lane)) v1 = dd_sub(v1, dd_mul(sm_dd(T, 32 + lane, j), xt));
            }
            if (r0 + lane < a.m) st_dd(a.x + r0 + lane, v0);
            if (r0 + 32 + lane < a.m) st_dd(a.x + r0 + 32 + lane, v1);
            __threadfence();
            __syncwarp();
            if (lane == 0 && c != a.withhold) sp_st_release(a.flags + c, a.epoch);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SP_THREADS) sp_bwd_kernel(SpSolveArgs a) {
    extern __shared__ double2 sp_sm[];
    double2 *xs = sp_sm + 2 * SP_T * SPL;
    __shared__ unsigned long long msk[2][SP_T];
    __shared__ int fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    for (int k = blockIdx.x; k < a.nblk; k += gridDim.x) {
        const int c = a.nblk - 1 - k;
        const int r0 = c * SP_T;
        // tiles (I, c), I > c, in descending I, then the diagonal tile
        const int q1 = a.col_ptr[c + 1], noff = q1 - a.col_ptr[c];
        dd_t v0 = dd_zero(), v1 = dd_zero();
        if (warp == 0) {
            if (r0 + lane < a.m) v0 = ld_dd(a.x + r0 + lane);
            if (r0 + 32 + lane < a.m) v1 = ld_dd(a.x + r0 + 32 + lane);
        }
        int t = noff > 0 ? a.col_tiles[q1 - 1] : a.diag[c];
        sp_load_tile(sp_sm, a.tiles + (long)t * SP_T * SP_T, tid, blockDim.x);
        if (tid < SP_T) msk[0][tid] = a.mask[(long)t * SP_T + tid];
        __syncthreads();
        for (int s = 0; s < noff; ++s) {
            const int buf = s & 1;
            const double2 *T = sp_sm + buf * SP_T * SPL;
            const int I = a.tIJ[2 * t];
            const int tn = s + 1 < noff ? a.col_tiles[q1 - 2 - s] : a.diag[c];
            if (warp != 0) {
                sp_load_tile(sp_sm + (buf ^ 1) * SP_T * SPL, a.tiles + (long)tn * SP_T * SP_T, tid - 32, blockDim.x - 32);
                if (tid >= 32 && tid < 32 + SP_T) msk[buf ^ 1][tid - 32] = a.mask[(long)tn * SP_T + tid - 32];
            } else if (!sp_wait(a, I)) {
                if (lane == 0) fail = 1;
            } else {
                const int ib = min(SP_T, a.m - I * SP_T);
                if (lane < ib) {
                    const dd_t xa = sp_ldcg(a.x + I * SP_T + lane);
                    xs[lane] = make_double2(xa.hi, xa.lo);
                }
                if (32 + lane < ib) {
                    const dd_t xb = sp_ldcg(a.x + I * SP_T + 32 + lane);
                    xs[32 + lane] = make_double2(xb.hi, xb.lo);
                }
                __syncwarp();
                const unsigned long long w0 = msk[buf][lane], w1 = msk[buf][32 + lane];
                for (int i = ib - 1; i >= 0; --i) {
                    const dd_t xt = dd_make(xs[i].x, xs[i].y);
                    if (bit64(w0, i)) v0 = dd_sub(v0, dd_mul(sm_dd(T, i, lane), xt));
                    if (bit64(w1, i)) v1 = dd_sub(v1, dd_mul(sm_dd(T, i, 32 + lane), xt));
                }
                __syncwarp();
            }
            __syncthreads();
            if (fail) return;
            t = tn;
        }
        if (warp == 0) {
            const int buf = noff & 1;
            const double2 *T = sp_sm + buf * SP_T * SPL;
            const int nb = min(SP_T, a.m - r0);
            const unsigned long long w0 = msk[buf][lane], w1 = msk[buf][32 + lane];
            for (int j = nb - 1; j >= 0; --j) {
                const int owner = j & 31;
                dd_t mine = j < 32 ? v0 : v1;
                if (lane == owner) {
                    mine = dd_muleq(mine, sm_dd(T, j, j));
                    if (j < 32) v0 = mine;
                    else v1 = mine;
                }
                const dd_t xt = sp_shfl(mine, owner);
                // x(b) -= L(j, b) x(j) for the columns b < j that hold row j
                if (lane < j && bit64(w0, j)) v0 = dd_sub(v0, dd_mul(sm_dd(T, j, lane), xt));
                if (32 + lane < j && bit64(w1, j)) v1 = dd_sub(v1, dd_mul(sm_dd(T, j, 32 + lane), xt));
            }
            if (r0 + lane < a.m) st_dd(a.x + r0 + lane, v0);
            if (r0 + 32 + lane < a.m) st_dd(a.x + r0 + 32 + lane, v1);
            __threadfence();
            __syncwarp();
            if (lane == 0 && c != a.withhold) sp_st_release(a.flags + c, a.epoch);
        }
        __syncthreads();
    }
}

__global__ void sp_permute_kernel(const dd_t *x, const int *order, int m, dd_t *xp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) st_dd(xp + k, ld_dd(x + order[k]));
}
__global__ void sp_unpermute_kernel(const dd_t *xp, const int *order, int m, dd_t *x) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) st_dd(x + order[k], ld_dd(xp + k));
}

// ============================================================== host side
static void upload_schedule(Context &c, SparseDev &s) {
    const TileSchedule &t = s.sched;
    cudaStream_t st = c.stream;
    std::vector<int> tij(2 * (size_t)t.ntiles), diag(t.nblk);
    for (int k = 0; k < t.ntiles; ++k) {
        tij[2 * k] = t.tI[k];
        tij[2 * k + 1] = t.tJ[k];
    }
    for (int J = 0; J < t.nblk; ++J) diag[J] = t.tile_of[J + (size_t)t.nblk * J];
    s.tIJ.upload(tij, st);
    s.diag.upload(diag, st);
    s.tile_of.upload(t.tile_of, st);
    std::vector<unsigned long long> mk(t.mask.begin(), t.mask.end());
    s.mask.upload(mk, st);
    s.col_ptr.upload(t.col_ptr, st);
    s.col_tiles.upload(t.col_tiles.empty() ? std::vector<int>{0} : t.col_tiles, st);
    s.row_ptr.upload(t.row_ptr, st);
    s.row_tiles.upload(t.row_tiles.empty() ? std::vector<int>{0} : t.row_tiles, st);
    s.upd.upload(t.upd.empty() ? std::vector<int>{0} : t.upd, st);
    s.tiles.alloc((size_t)t.ntiles * SP_T * SP_T);
    s.xp.alloc(std::max(1, t.m));
    s.panel_done.alloc(std::max(1, t.nblk));
    CK(cudaMemsetAsync(s.panel_done.p, 0, sizeof(int) * std::max(1, t.nblk), st));
    s.drop_graph();
    // per entry of the reference layout: its column b and row a
    const SparseStructure &ss = s.plan.s;
    std::vector<int> eb(ss.nnz()), ea(ss.nnz());
    for (int b = 0; b < ss.m; ++b)
        for (int q = ss.rowptr[b]; q < ss.rowptr[b + 1]; ++q) {
            eb[q] = b;
            ea[q] = ss.col[q];
        }
    s.ent_b.upload(eb, st);
    s.ent_a.upload(ea, st);
    CK(cudaStreamSynchronize(st));
}

void sparse_setup(Context &c) {
    if (!c.sp) c.sp = new SparseDev();
    SparseDev &s = *c.sp;
    s.plan = plan_schur(c.prob, c.schur_mode);
    s.active = s.plan.sparse;
    if (!s.active) return;
    s.sched = make_tile_schedule(s.plan.s);
    s.order.upload(s.plan.order, c.stream);
    upload_schedule(c, s);
}

void sparse_setup_structure(Context &c, const SparseStructure &ss) {
    const std::string bad = check_structure(ss);
    if (!bad.empty()) throw Error(ERR_ARG, "sparse factor structure: " + bad);
    if (!c.sp) c.sp = new SparseDev();
    SparseDev &s = *c.sp;
    s.plan = SparsePlan();
    s.plan.sparse = true;
    s.plan.s = ss;
    s.plan.order.resize(ss.m);
    for (int i = 0; i < ss.m; ++i) s.plan.order[i] = i;
    s.plan.extended = 2 * ss.nnz() - ss.m;
    s.active = true;
    s.sched = make_tile_schedule(ss);
    s.order.upload(s.plan.order, c.stream);
    upload_schedule(c, s);
}

// The launches of one factorisation.  Panel J waits for every update that
// writes into its column block; the update of panel J waits for panel J and
// for the previous update of each tile it writes (updates of one tile stay
// in pivot order).  Panels of independent subtrees of the elimination run
// side by side.
static void sparse_launches(Context &c, cudaGraph_t g) {
    SparseDev &s = *c.sp;
    const TileSchedule &t = s.sched;
    CK(cudaFuncSetAttribute(sp_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SP_TWO_TILES));
    CK(cudaFuncSetAttribute(sp_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SP_TWO_TILES));
    std::vector<cudaGraphNode_t> last_writer(t.ntiles, nullptr);
    std::vector<std::vector<cudaGraphNode_t>> into(t.nblk);
    auto uniq = [](std::vector<cudaGraphNode_t> v) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        return v;
    };
    dd_t *tiles = s.tiles.p;
    const unsigned long long *mask = s.mask.p;
    int m = t.m;
    int *done = s.panel_done.p;
    for (int J = 0; J < t.nblk; ++J) {
        const int ncol = t.col_ptr[J + 1] - t.col_ptr[J];
        int diag = t.tile_of[J + (size_t)t.nblk * J];
        const size_t smem = ncol > 0 ? SP_TWO_TILES : SP_TILE_SMEM;
        const int *col = s.col_tiles.p + t.col_ptr[J];
        int Jv = J;
        cudaGraphNode_t pnode = nullptr;
        {
            void *args[] = {&tiles, &mask, &m, &Jv, &diag, &col, &done};
            cudaKernelNodeParams kp{};
            kp.func = (void *)sp_panel_kernel;
            kp.gridDim = dim3(1 + ncol);
            kp.blockDim = dim3(SP_PANEL_THREADS);
            kp.sharedMemBytes = (unsigned)smem;
            kp.kernelParams = args;
            const std::vector<cudaGraphNode_t> deps = uniq(into[J]);
            CK(cudaGraphAddKernelNode(&pnode, g, deps.data(), deps.size(), &kp));
        }
        // the update of panel J in two nodes: the targets in column block
        // J + 1 (listed first: the schedule sorts targets by column block),
        // which panel J + 1 waits for, and the rest, which run beside it
        int nbJ = std::min(SP_T, t.m - J * SP_T);
        const int q0 = t.upd_ptr[J], q1 = t.upd_ptr[J + 1];
        int qs = q0;
        while (qs < q1 && t.tJ[t.upd[3 * qs]] == J + 1) ++qs;
        for (int part = 0; part < 2; ++part) {
            const int a = part == 0 ? q0 : qs, b = part == 0 ? qs : q1;
            if (a == b) continue;
            const int *upd = s.upd.p + 3 * (size_t)a;
            void *args[] = {&tiles, &mask, &upd, &nbJ};
            cudaKernelNodeParams kp{};
            kp.func = (void *)sp_update_kernel;
            kp.gridDim = dim3((b - a) * SP_UPD_SPLIT);
            kp.blockDim = dim3(SP_THREADS);
            kp.sharedMemBytes = (unsigned)SP_TWO_TILES;
            kp.kernelParams = args;
            std::vector<cudaGraphNode_t> deps{pnode};
            for (int q = a; q < b; ++q)
                if (last_writer[t.upd[3 * q]]) deps.push_back(last_writer[t.upd[3 * q]]);
            deps = uniq(deps);
            cudaGraphNode_t unode;
            CK(cudaGraphAddKernelNode(&unode, g, deps.data(), deps.size(), &kp));
            for (int q = a; q < b; ++q) {
                const int target = t.upd[3 * q];
                last_writer[target] = unode;
                into[t.tJ[target]].push_back(unode);
            }
        }
    }
}

static void sparse_panels(Context &c) {
    SparseDev &s = *c.sp;
    if (!s.graph) {
        cudaGraph_t g;
        CK(cudaGraphCreate(&g, 0));
        try {
            sparse_launches(c, g);
            CK(cudaGraphInstantiate(&s.graph, g, 0));
        } catch (...) {
            cudaGraphDestroy(g);
            throw;
        }
        CK(cudaGraphDestroy(g));
    }
    CK(cudaGraphLaunch(s.graph, c.stream));
}

void sparse_factor_B(Context &c) {
    SparseDev &s = *c.sp;
    PROF_SCOPE("sparse_factor", c.stream);
    if (s.sched.ntiles == 0) return;
    sp_gather_B_kernel<<<s.sched.ntiles, SP_THREADS, 0, c.stream>>>(c.B.p, c.m, s.order.p, s.tIJ.p, s.mask.p, s.tiles.p);
    CK_LAUNCH();
    sparse_panels(c);
}

void sparse_load_values(Context &c, const dd_t *vals) {
    SparseDev &s = *c.sp;
    const long nnz = s.plan.s.nnz();
    if (s.sched.ntiles == 0) return;
    CK(cudaMemsetAsync(s.tiles.p, 0, sizeof(dd_t) * (size_t)s.sched.ntiles * SP_T * SP_T, c.stream));
    sp_scatter_kernel<<<ceil_div(nnz, 256), 256, 0, c.stream>>>(vals, s.ent_b.p, s.ent_a.p, nnz, s.tile_of.p, s.sched.nblk, s.tiles.p);
    CK_LAUNCH();
}

void sparse_factor_values(Context &c, const dd_t *vals) {
    PROF_SCOPE("sparse_factor", c.stream);
    sparse_load_values(c, vals);
    if (c.sp->sched.ntiles > 0) sparse_panels(c);
}

void sparse_values(Context &c, dd_t *vals) {
    SparseDev &s = *c.sp;
    const long nnz = s.plan.s.nnz();
    if (nnz == 0) return;
    sp_gather_kernel<<<ceil_div(nnz, 256), 256, 0, c.stream>>>(s.tiles.p, s.ent_b.p, s.ent_a.p, nnz, s.tile_of.p, s.sched.nblk, vals);
    CK_LAUNCH();
}

static int sp_grid_cap(const void *kernel) {
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SP_SOLVE_SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, SP_THREADS, SP_SOLVE_SMEM));
    if (per < 1) throw Error(ERR_CUDA, "sparse solve: the wave kernel does not fit on an SM");
    return per * sms;
}

static void sp_solve_dir(Context &c, char dir, dd_t *x) {
    SparseDev &s = *c.sp;
    const TileSchedule &t = s.sched;
    TrsvSync &sync = trsv_sync(c, t.m);
    if (++sync.epoch <= 0) sync.epoch = 1;
    SpSolveArgs a{s.tiles.p, s.mask.p, s.tIJ.p, s.row_ptr.p, s.row_tiles.p, s.col_ptr.p, s.col_tiles.p, s.diag.p, t.m, t.nblk, sync.epoch, x,
                  sync.flags, sync.flags + sync.capacity, sync.wait_ns, sync.withhold};
    const void *k = dir == 'N' ? (const void *)sp_fwd_kernel : (const void *)sp_bwd_kernel;
    static thread_local int cap[2][64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int &cp = cap[dir == 'N' ? 0 : 1][dev & 63];
    if (cp == 0) cp = sp_grid_cap(k);
    const int grid = std::min(t.nblk, cp);
    void *args[] = {&a};
    CK(cudaLaunchCooperativeKernel(k, grid, SP_THREADS, args, SP_SOLVE_SMEM, c.stream));
    CK_LAUNCH();
}

void sparse_solve_raw(Context &c, dd_t *x) {
    if (c.sp->sched.m == 0) return;
    PROF_SCOPE("sparse_solve", c.stream);
    sp_solve_dir(c, 'N', x);
    sp_solve_dir(c, 'T', x);
    trsv_check(c.stream, c.trsv);
}

void sparse_solve(Context &c, dd_t *x) {
    SparseDev &s = *c.sp;
    const int m = s.sched.m;
    if (m == 0) return;
    PROF_SCOPE("sparse_solve", c.stream);
    sp_permute_kernel<<<ceil_div(m, 256), 256, 0, c.stream>>>(x, s.order.p, m, s.xp.p);
    CK_LAUNCH();
    sp_solve_dir(c, 'N', s.xp.p);
    sp_solve_dir(c, 'T', s.xp.p);
    sp_unpermute_kernel<<<ceil_div(m, 256), 256, 0, c.stream>>>(s.xp.p, s.order.p, m, x);
    CK_LAUNCH();
    trsv_check(c.stream, c.trsv);
}

double sparse_chol_terms(const Context &c) { return c.sp ? (double)c.sp->sched.exact_terms : 0.0; }

} // namespace sddd
