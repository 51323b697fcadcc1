// Schur complement B_ij = (X A_i Z^-1) . A_j on the device
// (Newton::Make_bMat / compute_bMat_dense_SDP, sdpa_newton.cpp:979-1068,
// 1223-1244).
//
// Per SDP block the reference visits every pair (i, j) of constraints once,
// from the owner i with (NonZeroEffect_i, i) >= (NonZeroEffect_j, j), using
// the owner's formula:
//   F1  G = X (A_i Z^-1) once per owner, value = A_j . G (calF1, :895)
//   F2  F = A_i Z^-1, value from rows of X and columns of F per nonzero of
//       A_j (calF2, :897-935); for dense A_j it switches to G = X F
//   F3  double loop over the nonzeros of A_i and A_j (calF3, :937-977)
// and adds value to B(i,j) and B(j,i) ("+=", blocks in order).
//
// On the B200 the pairs are regrouped by kind - never reordering the work on
// one entry:
//   - dense partners of F1/F2 owners: one TN GEMM  W^T V  over
//     W = [vec G_owner] and V = [vec A_dense] (k = n^2, each entry a
//     sequential dot), lower-triangle tiles only, scattered into B;
//   - sparse partners of F1/F2 owners and all F3 pairs: one thread (F1, F3)
//     or one warp (F2) per pair.
#include "context.h"
#include "ozaki.h"
#include "blas.h"
#include "newton.h"
#include "devops.cuh"
#include "prof.h"

#include <algorithm>
#include <unordered_map>

namespace sddd {

static BlockView view(const BlockDev &b) { return b.view(); }

// B(i,j) += v; B(j,i) += v for i != j (the reference's "+=").
__device__ __forceinline__ void b_add(dd_t *B, int m, int i, int j, dd_t v) {
    dd_t *p = B + i + (long)m * j;
    st_dd(p, dd_acc(ld_dd(p), v));
    if (i != j) {
        dd_t *q = B + j + (long)m * i;
        st_dd(q, dd_acc(ld_dd(q), v));
    }
}

// Where a block's pair value goes: into B directly (blocks one after the
// other), or, with stage != null, into the block's own staging square at
// (owner position, partner position), from which schur_accumulate_kernel
// adds the blocks' values to B in block order (blocks side by side).
__device__ __forceinline__ void pair_out(dd_t *B, int m, dd_t *stage, int nc, int s_own, int s_par, int i, int j, dd_t v) {
    if (stage)
        st_dd(stage + (long)s_own * nc + s_par, v);
    else
        b_add(B, m, i, j, v);
}

// ------------------------------------------------- F = A Z^-1, sparse A
// Row i of F is the ordered sum over the row list of v * (row src of Z^-1).
__global__ void f_sparse_kernel(int n, const int *ownFG, const int *rl_off, const int *rl_ptr, const int *rl_src, const dd_t *rl_val, const dd_t *invZ,
                                dd_t *F, int nfg) {
    const int r = blockIdx.y;
    const int off = rl_off[r];
    if (off < 0) return;
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    const int i = e % n, c = e / n;
    const int *ptr = rl_ptr + off;
    dd_t acc = dd_zero();
    for (int q = ptr[i]; q < ptr[i + 1]; ++q) acc = dd_acc(acc, dd_mul(rl_val[q], ld_dd(invZ + rl_src[q] + (long)n * c)));
    st_dd(F + (long)r * n * n + e, acc);
}

// --------------------------------------------- dense partners: W^T V GEMM
// C(r, d) = sum_k G_r[k] A_d[k] (Rdot over n^2 entries, calF1 / calF2 dense
// branch), for dense partner d with sorted position nsparse + d <= s(owner r).
template <int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    schur_dense_pairs_kernel(BlockView bv, const int *ownFG, int nfg, int ndense, const dd_t *__restrict__ W, const dd_t *__restrict__ V, dd_t *B, int m,
                             dd_t *stage) {
    constexpr int TX = BN / TN, TY = BM / TM, NT = TX * TY;
    __shared__ double2 As[BK][BM + 1];
    __shared__ double2 Bs[BK][BN + 1];
    __shared__ int s_row[BM];
    const long K = (long)bv.n * bv.n;
    const int r0 = blockIdx.y * BM, d0 = blockIdx.x * BN;
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    for (int e = tid; e < BM; e += NT) s_row[e] = (r0 + e < nfg) ? ownFG[r0 + e] : -1;
    __syncthreads();
    const int rlast = min(r0 + BM, nfg) - 1;
    if (bv.nsparse + d0 > s_row[rlast - r0]) return; // no valid pair in the tile
    dd_t acc[TM][TN];
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[r][c] = dd_zero();
    for (long k0 = 0; k0 < K; k0 += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            int kk = e % BK, ii = e / BK;
            long gk = k0 + kk;
            int gi = r0 + ii;
            double2 v = make_double2(0.0, 0.0);
            if (gi < nfg && gk < K) v = *reinterpret_cast<const double2 *>(W + gk + K * gi);
            As[kk][ii] = v;
        }
        for (int e = tid; e < BN * BK; e += NT) {
            int kk = e % BK, jj = e / BK;
            long gk = k0 + kk;
            int gj = d0 + jj;
            double2 v = make_double2(0.0, 0.0);
            if (gj < ndense && gk < K) v = *reinterpret_cast<const double2 *>(V + gk + K * gj);
            Bs[kk][jj] = v;
        }
        __syncthreads();
        const int kmax = (int)min((long)BK, K - k0);
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
                for (int c = 0; c < TN; ++c) acc[r][c] = dd_acc(acc[r][c], dd_mul(b[c], a[r]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < TM; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) {
            int gi = r0 + ty + TY * r, gd = d0 + tx + TX * c;
            if (gi >= nfg || gd >= ndense) continue;
            int s_own = s_row[ty + TY * r];
            int s_par = bv.nsparse + gd;
            if (s_par > s_own) continue;
            int i = bv.con[bv.perm[s_own]], j = bv.con[bv.perm[s_par]];
            // acc holds the Rdot partial (templ); Rdot returns 0 + templ
            pair_out(B, m, stage, bv.nc, s_own, s_par, i, j, dd_acc(dd_zero(), acc[r][c]));
        }
}

// ------------------------------------------ sparse partners of F1 owners
// value = A_j . G (calF1 with a sparse A_j)
__global__ void schur_f1_sparse_kernel(BlockView bv, const int *ownFG, int nfg, const dd_t *G, dd_t *B, int m, dd_t *stage) {
    const int r = blockIdx.y;
    const int s_own = ownFG[r];
    const int t_own = bv.perm[s_own];
    if (bv.formula[t_own] != F1) return;
    const int sp = blockIdx.x * blockDim.x + threadIdx.x; // sparse partner position
    if (sp >= bv.nsparse || sp > s_own) return;
    const int tj = bv.perm[sp];
    const int off = bv.coo_off[tj];
    dd_t v = sparse_dot_dense(bv.n, bv.nnz[tj], bv.row + off, bv.col + off, bv.val + off, G + (long)r * bv.n * bv.n);
    pair_out(B, m, stage, bv.nc, s_own, sp, bv.con[t_own], bv.con[tj], v);
}

// ------------------------------------------ sparse partners of F2 owners
// calF2 SPARSE (sdpa_newton.cpp:903-922): value = sum over nonzeros of A_j
// of v * Rdot(n, X(alpha, :), F(:, beta)) (+ the swapped term).  One warp per
// pair: lanes compute the dots, lane 0 accumulates in order.
constexpr int F2_WARPS = 4;
__global__ void schur_f2_sparse_kernel(BlockView bv, const int *ownFG, int nfg, const dd_t *X, const dd_t *F, dd_t *B, int m, dd_t *stage) {
    __shared__ double2 dots[F2_WARPS][64];
    const int r = blockIdx.y;
    const int s_own = ownFG[r];
    const int t_own = bv.perm[s_own];
    if (bv.formula[t_own] != F2) return;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int sp = blockIdx.x * F2_WARPS + warp;
    const bool active = sp < bv.nsparse && sp <= s_own;
    const int n = bv.n;
    const dd_t *Fr = F + (long)r * n * n;
    dd_t ret = dd_zero();
    int tj = 0;
    if (active) {
        tj = bv.perm[sp];
        const int off = bv.coo_off[tj], nnz = bv.nnz[tj];
        const int *row = bv.row + off, *col = bv.col + off;
        const dd_t *val = bv.val + off;
        for (int q0 = 0; q0 < nnz; q0 += 32) {
            const int q = q0 + lane;
            dd_t d1 = dd_zero(), d2 = dd_zero();
            if (q < nnz) {
                const int al = row[q], be = col[q];
                for (int k = 0; k < n; ++k) d1 = dd_acc(d1, dd_mul(ld_dd(X + al + (long)n * k), ld_dd(Fr + k + (long)n * be)));
                if (al != be)
                    for (int k = 0; k < n; ++k) d2 = dd_acc(d2, dd_mul(ld_dd(X + be + (long)n * k), ld_dd(Fr + k + (long)n * al)));
            }
            dots[warp][2 * lane] = make_double2(d1.hi, d1.lo);
            dots[warp][2 * lane + 1] = make_double2(d2.hi, d2.lo);
            __syncwarp();
            if (lane == 0) {
                const int cnt = min(32, nnz - q0);
                for (int u = 0; u < cnt; ++u) {
                    dd_t v1 = val[q0 + u];
                    ret = dd_acc(ret, dd_mul(v1, dd_make(dots[warp][2 * u].x, dots[warp][2 * u].y)));
                    if (row[q0 + u] != col[q0 + u]) ret = dd_acc(ret, dd_mul(v1, dd_make(dots[warp][2 * u + 1].x, dots[warp][2 * u + 1].y)));
                }
            }
            __syncwarp();
        }
        if (lane == 0) pair_out(B, m, stage, bv.nc, s_own, sp, bv.con[t_own], bv.con[tj], ret);
    }
}

// --------------------------------- dense partners from the split products
// pairs[r + nfg d] = G_r . A_d (d <= r) of a block whose constraints are all
// dense F1/F2 owners (sorted position = owner index = dense index): added to
// B(i,j) and B(j,i) as the reference adds each pair's value.
__global__ void schur_scatter_pairs_kernel(BlockView bv, int nfg, const dd_t *pairs, dd_t *B, int m) {
    const int r = blockIdx.y;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d > r) return;
    const int i = bv.con[bv.perm[r]], j = bv.con[bv.perm[d]];
    b_add(B, m, i, j, ld_dd(pairs + r + (long)nfg * d));
}

// ----------------------------------------------------------- F3 owners
// calF3 (sdpa_newton.cpp:937-977), one thread per pair.
__global__ void schur_f3_kernel(BlockView bv, const int *ownF3, int nf3, const dd_t *X, const dd_t *invZ, dd_t *B, int m, dd_t *stage) {
    const int r = blockIdx.y;
    const int s_own = ownF3[r];
    const int sp = blockIdx.x * blockDim.x + threadIdx.x;
    if (sp > s_own) return;
    const int n = bv.n;
    const int ti = bv.perm[s_own], tj = bv.perm[sp];
    const int oi = bv.coo_off[ti], ni = bv.nnz[ti], oj = bv.coo_off[tj], nj = bv.nnz[tj];
    const int *ri = bv.row + oi, *ci = bv.col + oi, *rj = bv.row + oj, *cj = bv.col + oj;
    const dd_t *vi = bv.val + oi, *vj = bv.val + oj;
    dd_t ret = dd_zero();
    for (int q1 = 0; q1 < nj; ++q1) {
        const int al = rj[q1], be = cj[q1];
        const dd_t v1 = vj[q1];
        dd_t sum = dd_zero();
        for (int q2 = 0; q2 < ni; ++q2) {
            const int ga = ri[q2], de = ci[q2];
            const dd_t v2 = vi[q2];
            sum = dd_acc(sum, dd_mul(dd_mul(v2, ld_dd(invZ + de + (long)n * be)), ld_dd(X + al + (long)n * ga)));
            if (ga != de) sum = dd_acc(sum, dd_mul(dd_mul(v2, ld_dd(invZ + ga + (long)n * be)), ld_dd(X + al + (long)n * de)));
        }
        ret = dd_acc(ret, dd_mul(v1, sum));
        if (al == be) continue;
        sum = dd_zero();
        for (int q2 = 0; q2 < ni; ++q2) {
            const int ga = ri[q2], de = ci[q2];
            const dd_t v2 = vi[q2];
            sum = dd_acc(sum, dd_mul(dd_mul(v2, ld_dd(invZ + de + (long)n * al)), ld_dd(X + be + (long)n * ga)));
            if (ga != de) sum = dd_acc(sum, dd_mul(dd_mul(v2, ld_dd(invZ + ga + (long)n * al)), ld_dd(X + be + (long)n * de)));
        }
        ret = dd_acc(ret, dd_mul(v1, sum));
    }
    pair_out(B, m, stage, bv.nc, s_own, sp, bv.con[ti], bv.con[tj], ret);
}

// One block's pairs, all on stream st, with F and G scratch of its own and
// its pair values into B (stage null) or into its staging square.
static void schur_block(Context &c, int l, cudaStream_t st, dd_t *Fb, dd_t *Gb, dd_t *stage) {
    const int m = c.m;
    BlockDev &bd = *c.blocks[l];
    const BlockView bv = view(bd);
    const int n = bd.n;
    const long nn = (long)n * n;
    const dd_t *X = c.X.blk(c.off, l), *Zi = c.invZ.blk(c.off, l);
    const int nfg = bd.nFG();
    if (nfg > 0) {
        // F_r = A_r Z^-1
        bool any_sparse = false;
        for (int v : bd.h_rl_off) any_sparse |= v >= 0;
        if (any_sparse) {
            dim3 grid(ceil_div(nn, 128), nfg);
            f_sparse_kernel<<<grid, 128, 0, st>>>(n, bd.ownFG.p, bd.rl_off.p, bd.rl_ptr.p, bd.rl_src.p, bd.rl_val.p, Zi, Fb, nfg);
            CK_LAUNCH();
        }
        if (bd.fg_dense_contig) {
            // the FG owners' dense matrices are consecutive in bd.dense
            const long o0 = bd.h_dense_off[bd.h_perm[bd.h_ownFG[0]]];
            gemm(st, 'N', 'N', GEMM_STORE, n, n, n, bd.dense.p + o0, n, nn, Zi, n, 0, Fb, n, nn, nfg, false);
        } else {
            for (int r = 0; r < nfg; ++r) {
                long o = bd.h_dense_off[bd.h_perm[bd.h_ownFG[r]]];
                if (o >= 0) gemm(st, 'N', 'N', GEMM_STORE, n, n, n, bd.dense.p + o, n, 0, Zi, n, 0, Fb + r * nn, n, 0, 1, false);
            }
        }
        // G_r = X F_r
        gemm(st, 'N', 'N', GEMM_STORE, n, n, n, X, n, 0, Fb, n, nn, Gb, n, nn, nfg, false);
        // dense partners
        const int ndense = bd.nc - bd.nsparse;
        if (!stage && c.tc_slices > 0 && bd.nsparse == 0 && nfg == bd.nc && bd.fg_dense_contig && nn <= OG_MAX_K) {
            // every pair of the block is one n^2-term product G_r . A_d:
            // the INT8 tensor-core split of W^T V, W = [vec G_r],
            // V = [vec A_d], then the pairs into B
            OzakiGemmWork &w = tcg_work(c, nfg, nn, c.tc_slices);
            c.tcg_pairs.alloc((size_t)nfg * nfg);
            const long o0 = bd.h_dense_off[bd.h_perm[0]];
            ozaki_gemm_lower(st, Gb, nn, bd.dense.p + o0, nn, nfg, nn, c.tcg_pairs.p, nfg, w);
            dim3 grid(ceil_div(nfg, 128), nfg);
            schur_scatter_pairs_kernel<<<grid, 128, 0, st>>>(bv, nfg, c.tcg_pairs.p, c.B.p, m);
            CK_LAUNCH();
        } else if (ndense > 0) {
            // Every pair is one sequential dot over the n^2 entries.  With
            // few pairs (small m) 64 x 64 tiles of 16 pairs per thread
            // leave the GPU nearly idle on long chains; one pair per
            // thread in 16 x 16 tiles spreads them over many more CTAs.
            if ((long)ceil_div(ndense, 64) * ceil_div(nfg, 64) >= 2L * 148) {
                constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4;
                dim3 grid(ceil_div(ndense, BN), ceil_div(nfg, BM));
                schur_dense_pairs_kernel<BM, BN, BK, TM, TN>
                    <<<grid, (BM / TM) * (BN / TN), 0, st>>>(bv, bd.ownFG.p, nfg, ndense, Gb, bd.dense.p, c.B.p, m, stage);
            } else {
                constexpr int BM = 16, BN = 16, BK = 32, TM = 1, TN = 1;
                dim3 grid(ceil_div(ndense, BN), ceil_div(nfg, BM));
                schur_dense_pairs_kernel<BM, BN, BK, TM, TN>
                    <<<grid, (BM / TM) * (BN / TN), 0, st>>>(bv, bd.ownFG.p, nfg, ndense, Gb, bd.dense.p, c.B.p, m, stage);
            }
            CK_LAUNCH();
        }
        // sparse partners
        if (bd.nsparse > 0) {
            dim3 g1(ceil_div(bd.nsparse, 128), nfg);
            schur_f1_sparse_kernel<<<g1, 128, 0, st>>>(bv, bd.ownFG.p, nfg, Gb, c.B.p, m, stage);
            CK_LAUNCH();
            dim3 g2(ceil_div(bd.nsparse, F2_WARPS), nfg);
            schur_f2_sparse_kernel<<<g2, 32 * F2_WARPS, 0, st>>>(bv, bd.ownFG.p, nfg, X, Fb, c.B.p, m, stage);
            CK_LAUNCH();
        }
    }
    const int nf3 = bd.nF3();
    if (nf3 > 0) {
        dim3 grid(ceil_div(bd.nsparse, 128), nf3);
        schur_f3_kernel<<<grid, 128, 0, st>>>(bv, bd.ownF3.p, nf3, X, Zi, c.B.p, m, stage);
        CK_LAUNCH();
    }
}

// ------------------------------------------------ many blocks: one graph
// B(i,j) = 0 + v_l1 + v_l2 + ... over the blocks holding both constraints,
// in block order (bMat.setZero, then each block's "+="), from the blocks'
// staging squares; both triangles.
__global__ void schur_accumulate_kernel(const int *ent, const int *ptr, const long *src, int nent, const dd_t *stage, dd_t *B, int m) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    const int i = ent[2 * e], j = ent[2 * e + 1];
    dd_t acc = dd_zero();
    for (int q = ptr[e]; q < ptr[e + 1]; ++q) acc = dd_acc(acc, ld_dd(stage + src[q]));
    st_dd(B + i + (long)m * j, acc);
    if (i != j) st_dd(B + j + (long)m * i, acc);
}

constexpr int SG_MIN_BLOCKS = 4;         // fewer blocks: the blocks one after the other
constexpr int SG_BRANCHES = 8;           // parallel branches of the graph
constexpr long SG_MAX_STAGE = 1L << 24;  // staging entries (256 MB)
constexpr long SG_MAX_FG = 1L << 22;     // F (and G) scratch entries per branch

static void schur_block(Context &c, int l, cudaStream_t st, dd_t *Fb, dd_t *Gb, dd_t *stage);

// Builds (once per upload) and launches the many-block graph; false when the
// problem takes the sequential path (few blocks, the tensor-core split of
// the pair products, or scratch above the caps).
static bool schur_graph_launch(Context &c) {
    if (c.nSDP < SG_MIN_BLOCKS || c.tc_slices > 0) return false;
    if (!c.sg) c.sg = new SchurGraph();
    SchurGraph &g = *c.sg;
    if (g.gen != c.upload_gen) {
        g.gen = c.upload_gen;
        g.eligible = false;
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        std::vector<long> soff(c.nSDP + 1, 0);
        long maxfg = 1;
        for (int l = 0; l < c.nSDP; ++l) {
            const BlockDev &bd = *c.blocks[l];
            soff[l + 1] = soff[l] + (long)bd.nc * bd.nc;
            maxfg = std::max(maxfg, (long)bd.nFG() * bd.n * bd.n);
        }
        if (soff[c.nSDP] > SG_MAX_STAGE || maxfg > SG_MAX_FG) return false;
        // the B entries and their contributions, blocks in order
        std::unordered_map<long, int> index;
        std::vector<std::pair<long, std::vector<long>>> entries;
        for (int l = 0; l < c.nSDP; ++l) {
            const BlockDev &bd = *c.blocks[l];
            const std::vector<int> &con = c.prob.cons[l];
            for (int so = 0; so < bd.nc; ++so)
                for (int sp = 0; sp <= so; ++sp) {
                    const int a = con[bd.h_perm[so]], b = con[bd.h_perm[sp]];
                    const long key = (long)std::max(a, b) * c.m + std::min(a, b);
                    auto it = index.find(key);
                    int e;
                    if (it == index.end()) {
                        e = (int)entries.size();
                        index.emplace(key, e);
                        entries.push_back({key, {}});
                    } else {
                        e = it->second;
                    }
                    entries[e].second.push_back(soff[l] + (long)so * bd.nc + sp);
                }
        }
        std::sort(entries.begin(), entries.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        std::vector<int> ent, ptr(1, 0);
        std::vector<long> src;
        for (const auto &e : entries) {
            ent.push_back((int)(e.first / c.m));
            ent.push_back((int)(e.first % c.m));
            src.insert(src.end(), e.second.begin(), e.second.end());
            ptr.push_back((int)src.size());
        }
        g.nent = (int)entries.size();
        g.ent.upload(ent, c.stream);
        g.ptr.upload(ptr, c.stream);
        g.src.upload(src, c.stream);
        g.stage.alloc((size_t)std::max(1L, soff[c.nSDP]));
        g.F.alloc((size_t)SG_BRANCHES * maxfg);
        g.G.alloc((size_t)SG_BRANCHES * maxfg);
        if (g.branch.empty()) {
            g.branch.resize(SG_BRANCHES);
            g.joined.resize(SG_BRANCHES);
            for (int k = 0; k < SG_BRANCHES; ++k) {
                CK(cudaStreamCreateWithFlags(&g.branch[k], cudaStreamNonBlocking));
                CK(cudaEventCreateWithFlags(&g.joined[k], cudaEventDisableTiming));
            }
            CK(cudaEventCreateWithFlags(&g.forked, cudaEventDisableTiming));
        }
        CK(cudaStreamSynchronize(c.stream));
        cudaStream_t st = c.stream;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            CK(cudaMemsetAsync(c.B.p, 0, sizeof(dd_t) * (size_t)c.m * c.m, st)); // bMat.setZero()
            CK(cudaEventRecord(g.forked, st));
            const int nbr = std::min(SG_BRANCHES, c.nSDP);
            for (int k = 0; k < nbr; ++k) CK(cudaStreamWaitEvent(g.branch[k], g.forked, 0));
            for (int l = 0; l < c.nSDP; ++l) {
                const int k = l % nbr;
                schur_block(c, l, g.branch[k], g.F.p + k * maxfg, g.G.p + k * maxfg, g.stage.p + soff[l]);
            }
            for (int k = 0; k < nbr; ++k) {
                CK(cudaEventRecord(g.joined[k], g.branch[k]));
                CK(cudaStreamWaitEvent(st, g.joined[k], 0));
            }
            if (g.nent > 0) {
                schur_accumulate_kernel<<<ceil_div(g.nent, 128), 128, 0, st>>>(g.ent.p, g.ptr.p, g.src.p, g.nent, g.stage.p, c.B.p, c.m);
                CK_LAUNCH();
            }
        } catch (...) {
            cudaGraph_t dropped;
            cudaStreamEndCapture(st, &dropped);
            if (dropped) cudaGraphDestroy(dropped);
            throw;
        }
        CK(cudaStreamEndCapture(st, &graph));
        CK(cudaGraphInstantiate(&g.exec, graph, 0));
        CK(cudaGraphDestroy(graph));
        g.eligible = true;
    }
    if (!g.eligible) return false;
    CK(cudaGraphLaunch(g.exec, c.stream));
    return true;
}

void schur_build(Context &c) {
    cudaStream_t st = c.stream;
    PROF_SCOPE("schur_build", st);
    if (schur_graph_launch(c)) return;
    const int m = c.m;
    CK(cudaMemsetAsync(c.B.p, 0, sizeof(dd_t) * (size_t)m * m, st)); // bMat.setZero()
    for (int l = 0; l < c.nSDP; ++l) schur_block(c, l, st, c.Fbuf.p, c.Gbuf.p, nullptr);
    if (c.tcg.err) ozaki_gemm_check(st, c.tcg);
}

} // namespace sddd
