// Batched Newton core for batches of small SDPs (sddd_batch_*; no
// counterpart in the reference, which solves one problem per process).
//
// The workers of a batch each run the ordinary solver on their own context.
// At the Schur build and Cholesky of B (Newton::Make_bMat +
// Lal::choleskyFactorWithAdjust, sdpa_newton.cpp:1223-1299) a worker whose
// problem qualifies (one SDP block, every constraint a dense F1/F2 owner:
// the dense random configuration) hands its context to the engine and
// waits; the engine gathers the contexts that arrive (all active workers,
// or those waiting when the oldest has waited CORE_WAIT_US) and runs the
// core of all of them as one captured CUDA graph of persistent launches:
//   zero B                          (bMat.setZero)
//   F_r = A_r Z^-1, G_r = X F_r     (calF1's two products, one CTA per
//                                    (problem, constraint, 32 x 32 tile),
//                                    grid-stride)
//   B_ij += G_i . A_j, j <= i       (one tiled launch per tile shape, each
//                                    over the problems assigned to it)
//   L L^T = B                       (one CTA per problem, right-looking)
// Each entry sees the same operations in the same order as the single-
// problem kernels (gemm_kernel STORE, schur_dense_pairs_kernel, potrf), so
// every problem's result stays bit for bit that of a single solve.
//
// The graph reads a descriptor block (per problem: pointers and sizes; per
// tile shape: the prefix of its tiles) that the engine copies from pinned
// memory as the graph's first node, so one instantiated graph serves every
// batch whatever its problems.
//
// Tile shapes of the pair products are picked per size class of m by a
// small autotuner: the first batches of a class time each candidate shape
// (event nodes around each pairs launch inside the graph) on that class's
// problems, normalised per pair-term, and the fastest is kept for the rest.
#include "batched.h"

#include <algorithm>
#include <chrono>
#include <cstring>

#include "blas.h"
#include "devops.cuh"
#include "newton.h"

namespace sddd {

namespace {

constexpr int CORE_CAP = 256;      // problems per batch
constexpr int CORE_SHAPES = 3;     // candidate tile shapes of the pair products
constexpr int CORE_MAX_M = 1024;
constexpr int CORE_MAX_N = 128;
constexpr int CORE_WAIT_US = 1500; // longest wait for more problems

struct CoreItem {
    int m, n;
    const dd_t *A;          // m dense n x n matrices, sorted (= storage) order
    const int *con, *perm;  // constraint of a sorted position
    const dd_t *X, *Zi;
    dd_t *F, *G;            // m n^2 each
    dd_t *B;                // m x m
    int *info;
};

struct CoreBatch {
    int count;
    int total_fg;                          // work units of the F and G products
    int fg_off[CORE_CAP + 1];              // prefix of m * (32 x 32 tiles of n x n)
    int shape[CORE_CAP];                   // tile shape of each problem
    long tile_off[CORE_SHAPES][CORE_CAP + 1]; // per shape: prefix of its problems' tiles (0 for others)
    CoreItem it[CORE_CAP];
};

// Problem holding flat index u of a prefix array off[0..count] (off[0] = 0).
template <class T>
__device__ __forceinline__ int core_find(const T *off, int count, T u) {
    int lo = 0, hi = count; // off[lo] <= u < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= u)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// bMat.setZero() of every problem: blockIdx.y = problem.
__global__ void core_zero_kernel(const CoreBatch *bt) {
    const int q = blockIdx.y;
    if (q >= bt->count) return;
    const CoreItem &it = bt->it[q];
    const long mm = (long)it.m * it.m;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < mm; e += (long)gridDim.x * blockDim.x) st_dd(it.B + e, dd_zero());
}

// F_r = A_r Z^-1 (stage 0) or G_r = X F_r (stage 1) for every (problem,
// r): one CTA per 32 x 32 output tile of one product (work units u =
// fg_off[q] + r * tiles + tile), k in chunks of 16 staged in shared memory,
// 2 x 2 outputs per thread; every output keeps gemm_kernel's STORE form,
// acc += Q(k,j) * P(i,k) for k ascending from zero.
constexpr int FG_T = 32, FG_K = 16;
__global__ void __launch_bounds__(256) core_fg_kernel(const CoreBatch *bt, int stage) {
    __shared__ double2 Ps[FG_K][FG_T + 1];
    __shared__ double2 Qs[FG_K][FG_T + 1];
    const int total = bt->total_fg;
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int q = core_find(bt->fg_off, bt->count, u);
        const CoreItem &it = bt->it[q];
        const int n = it.n, nt = (n + FG_T - 1) / FG_T;
        const int w = u - bt->fg_off[q], r = w / (nt * nt), tile = w % (nt * nt);
        const int i0 = (tile % nt) * FG_T, j0 = (tile / nt) * FG_T;
        const long nn = (long)n * n;
        const dd_t *P = stage == 0 ? it.A + r * nn : it.X;
        const dd_t *Q = stage == 0 ? it.Zi : it.F + r * nn;
        dd_t *out = stage == 0 ? it.F + r * nn : it.G + r * nn;
        dd_t acc[2][2] = {{dd_zero(), dd_zero()}, {dd_zero(), dd_zero()}};
        for (int k0 = 0; k0 < n; k0 += FG_K) {
            for (int e = tid; e < FG_T * FG_K; e += 256) {
                const int ii = e % FG_T, kk = e / FG_T;
                const int gi = i0 + ii, gk = k0 + kk;
                Ps[kk][ii] = (gi < n && gk < n) ? *reinterpret_cast<const double2 *>(P + gi + (long)n * gk) : make_double2(0.0, 0.0);
            }
            for (int e = tid; e < FG_T * FG_K; e += 256) {
                const int kk = e % FG_K, jj = e / FG_K;
                const int gj = j0 + jj, gk = k0 + kk;
                Qs[kk][jj] = (gj < n && gk < n) ? *reinterpret_cast<const double2 *>(Q + gk + (long)n * gj) : make_double2(0.0, 0.0);
            }
            __syncthreads();
            const int kmax = min(FG_K, n - k0);
            for (int kk = 0; kk < kmax; ++kk) {
                dd_t a[2], b[2];
#pragma unroll
                for (int x = 0; x < 2; ++x) a[x] = dd_make(Ps[kk][ty + 16 * x].x, Ps[kk][ty + 16 * x].y);
#pragma unroll
                for (int y = 0; y < 2; ++y) b[y] = dd_make(Qs[kk][tx + 16 * y].x, Qs[kk][tx + 16 * y].y);
#pragma unroll
                for (int x = 0; x < 2; ++x)
#pragma unroll
                    for (int y = 0; y < 2; ++y) acc[x][y] = dd_acc(acc[x][y], dd_mul(b[y], a[x]));
            }
            __syncthreads();
        }
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                const int i = i0 + ty + 16 * x, j = j0 + tx + 16 * y;
                if (i < n && j < n) st_dd(out + i + (long)n * j, acc[x][y]);
            }
    }
}

// B(i,j) += v; B(j,i) += v for i != j (the reference's "+=").
__device__ __forceinline__ void core_badd(dd_t *B, int m, int i, int j, dd_t v) {
    dd_t *p = B + i + (long)m * j;
    st_dd(p, dd_acc(ld_dd(p), v));
    if (i != j) {
        dd_t *q = B + j + (long)m * i;
        st_dd(q, dd_acc(ld_dd(q), v));
    }
}

// Pair products of the problems assigned to tile shape S: tiles of BM owner
// rows x BN partner columns of every such problem (the full square grid of
// its pairs, tiles above the diagonal skipped), each entry the sequential
// n^2-term dot of schur_dense_pairs_kernel.
template <int S, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) core_pairs_kernel(const CoreBatch *bt) {
    constexpr int TX = BN / TN, TY = BM / TM, NT = TX * TY;
    __shared__ double2 As[BK][BM + 1];
    __shared__ double2 Bs[BK][BN + 1];
    const long total = bt->tile_off[S][bt->count];
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    for (long u = blockIdx.x; u < total; u += gridDim.x) {
        const int q = core_find(bt->tile_off[S], bt->count, u);
        const CoreItem &it = bt->it[q];
        const int m = it.m;
        const int ntc = (m + BN - 1) / BN;
        const long t = u - bt->tile_off[S][q];
        const int r0 = (int)(t / ntc) * BM, d0 = (int)(t % ntc) * BN;
        if (d0 > r0 + BM - 1) continue; // above the diagonal (uniform in the CTA)
        const long K = (long)it.n * it.n;
        dd_t acc[TM][TN];
#pragma unroll
        for (int a = 0; a < TM; ++a)
#pragma unroll
            for (int b = 0; b < TN; ++b) acc[a][b] = dd_zero();
        for (long k0 = 0; k0 < K; k0 += BK) {
            for (int e = tid; e < BM * BK; e += NT) {
                const int kk = e % BK, ii = e / BK;
                const long gk = k0 + kk;
                const int gi = r0 + ii;
                As[kk][ii] = (gi < m && gk < K) ? *reinterpret_cast<const double2 *>(it.G + gk + K * gi) : make_double2(0.0, 0.0);
            }
            for (int e = tid; e < BN * BK; e += NT) {
                const int kk = e % BK, jj = e / BK;
                const long gk = k0 + kk;
                const int gj = d0 + jj;
                Bs[kk][jj] = (gj < m && gk < K) ? *reinterpret_cast<const double2 *>(it.A + gk + K * gj) : make_double2(0.0, 0.0);
            }
            __syncthreads();
            const int kmax = (int)min((long)BK, K - k0);
            for (int kk = 0; kk < kmax; ++kk) {
                dd_t a[TM], b[TN];
#pragma unroll
                for (int x = 0; x < TM; ++x) a[x] = dd_make(As[kk][ty + TY * x].x, As[kk][ty + TY * x].y);
#pragma unroll
                for (int y = 0; y < TN; ++y) b[y] = dd_make(Bs[kk][tx + TX * y].x, Bs[kk][tx + TX * y].y);
#pragma unroll
                for (int x = 0; x < TM; ++x)
#pragma unroll
                    for (int y = 0; y < TN; ++y) acc[x][y] = dd_acc(acc[x][y], dd_mul(b[y], a[x]));
            }
            __syncthreads();
        }
#pragma unroll
        for (int x = 0; x < TM; ++x)
#pragma unroll
            for (int y = 0; y < TN; ++y) {
                const int r = r0 + ty + TY * x, d = d0 + tx + TX * y;
                if (r >= m || d > r) continue;
                core_badd(it.B, m, it.con[it.perm[r]], it.con[it.perm[d]], dd_acc(dd_zero(), acc[x][y]));
            }
    }
}

// In-place lower Cholesky of every problem's B, one CTA per problem,
// right-looking column by column: pivot (sqrt, then the reciprocal
// 1/L(j,j)), scaling of the column by it, then the update of the trailing
// lower triangle; every entry takes x - L(j,k) L(i,k) for k ascending and
// then its sqrt or scaling, as potrf's kernels do.  *info: the 1-based
// failing column.
constexpr int CORE_POTRF_THREADS = 1024;
__global__ void __launch_bounds__(CORE_POTRF_THREADS) core_potrf_kernel(const CoreBatch *bt) {
    const int q = blockIdx.x;
    if (q >= bt->count) return;
    const CoreItem &it = bt->it[q];
    const int m = it.m;
    dd_t *A = it.B;
    __shared__ double2 rj;
    __shared__ int fail;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) fail = 0;
    __syncthreads();
    for (int j = 0; j < m; ++j) {
        if (tid == 0) {
            const dd_t d = ld_dd(A + j + (long)m * j);
            if (dd_le_d(d, 0.0) || dd_isnan(d)) {
                fail = 1;
                *it.info = j + 1;
            } else {
                const dd_t l = dd_sqrt(d);
                st_dd(A + j + (long)m * j, l);
                const dd_t r = dd_div(dd_from(1.0), l);
                rj = make_double2(r.hi, r.lo);
            }
        }
        __syncthreads();
        if (fail) return;
        const dd_t r = dd_make(rj.x, rj.y);
        for (int i = j + 1 + tid; i < m; i += nt) st_dd(A + i + (long)m * j, dd_mul(r, ld_dd(A + i + (long)m * j)));
        __syncthreads();
        // trailing lower triangle: entries (i, k), j < k <= i
        const int w = m - j - 1;
        const long cnt = (long)w * (w + 1) / 2;
        for (long e = tid; e < cnt; e += nt) {
            // e -> (k, i): column k = j+1+c, rows i = k..m-1; column-major packing
            const int c = (int)((2.0 * w + 1.0 - sqrt((2.0 * w + 1.0) * (2.0 * w + 1.0) - 8.0 * (double)e)) / 2.0);
            int cc = c;
            long base = (long)cc * w - (long)cc * (cc - 1) / 2;
            while (base > e) { // guard the floating estimate
                --cc;
                base = (long)cc * w - (long)cc * (cc - 1) / 2;
            }
            while (base + (w - cc) <= e) {
                base += w - cc;
                ++cc;
            }
            const int k = j + 1 + cc, i = k + (int)(e - base);
            dd_t *p = A + i + (long)m * k;
            st_dd(p, dd_sub(ld_dd(p), dd_mul(ld_dd(A + k + (long)m * j), ld_dd(A + i + (long)m * j))));
        }
        __syncthreads();
    }
}

struct Shape {
    int bm, bn;
};
constexpr Shape SHAPES[CORE_SHAPES] = {{16, 16}, {32, 32}, {64, 64}};

int size_class(int m) { return m <= 64 ? 0 : m <= 128 ? 1 : m <= 256 ? 2 : 3; }

} // namespace

struct CoreEngine::Impl {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t ev_shape[CORE_SHAPES][2] = {};
    CoreBatch *hb = nullptr, *db = nullptr;
    cudaGraphExec_t exec = nullptr;
    int sms = 148;
    // autotuner: per size class, the chosen shape (-1: still measuring) and
    // the measured ms per pair-term of each candidate (< 0: not yet)
    int chosen[4] = {-1, -1, -1, -1};
    double per_term[4][CORE_SHAPES];
    int trial[4] = {0, 0, 0, 0};
    std::vector<Context *> pending;
    std::chrono::steady_clock::time_point first_wait;
};

bool core_eligible(const Context &c) {
    if (c.nSDP != 1 || c.tc_slices > 0 || c.m > CORE_MAX_M || c.sparse_active()) return false;
    const BlockDev &bd = *c.blocks[0];
    return bd.n <= CORE_MAX_N && bd.nsparse == 0 && bd.nFG() == bd.nc && bd.fg_dense_contig && bd.nc == c.m;
}

CoreEngine::CoreEngine(int device) : p(new Impl) {
    p->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming));
    for (auto &e : p->ev_shape) {
        CK(cudaEventCreate(&e[0]));
        CK(cudaEventCreate(&e[1]));
    }
    CK(cudaMallocHost(&p->hb, sizeof(CoreBatch)));
    CK(cudaMalloc(&p->db, sizeof(CoreBatch)));
    std::memset(p->hb, 0, sizeof(CoreBatch));
    CK(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, device));
    for (auto &row : p->per_term)
        for (double &v : row) v = -1.0;
    // the graph: descriptor copy, zero, F, G, the pair products of each
    // shape between event-record nodes (recorded as external events, so
    // that every launch of the graph records them and the autotuner can
    // time the shapes; a plain record inside a capture only orders the
    // graph), the factorisations
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(p->db, p->hb, sizeof(CoreBatch), cudaMemcpyHostToDevice, p->stream);
    core_zero_kernel<<<dim3(8, CORE_CAP), 256, 0, p->stream>>>(p->db);
    core_fg_kernel<<<4 * p->sms, 256, 0, p->stream>>>(p->db, 0);
    core_fg_kernel<<<4 * p->sms, 256, 0, p->stream>>>(p->db, 1);
    cudaEventRecordWithFlags(p->ev_shape[0][0], p->stream, cudaEventRecordExternal);
    core_pairs_kernel<0, 16, 16, 32, 1, 1><<<8 * p->sms, 256, 0, p->stream>>>(p->db);
    cudaEventRecordWithFlags(p->ev_shape[0][1], p->stream, cudaEventRecordExternal);
    cudaEventRecordWithFlags(p->ev_shape[1][0], p->stream, cudaEventRecordExternal);
    core_pairs_kernel<1, 32, 32, 16, 2, 2><<<4 * p->sms, 256, 0, p->stream>>>(p->db);
    cudaEventRecordWithFlags(p->ev_shape[1][1], p->stream, cudaEventRecordExternal);
    cudaEventRecordWithFlags(p->ev_shape[2][0], p->stream, cudaEventRecordExternal);
    core_pairs_kernel<2, 64, 64, 16, 4, 4><<<2 * p->sms, 256, 0, p->stream>>>(p->db);
    cudaEventRecordWithFlags(p->ev_shape[2][1], p->stream, cudaEventRecordExternal);
    core_potrf_kernel<<<CORE_CAP, CORE_POTRF_THREADS, 0, p->stream>>>(p->db);
    cudaError_t cap = cudaStreamEndCapture(p->stream, &g);
    if (cap != cudaSuccess) throw Error(ERR_CUDA, std::string("batched core: graph capture failed: ") + cudaGetErrorString(cap));
    CK(cudaGraphInstantiate(&p->exec, g, 0));
    CK(cudaGraphDestroy(g));
}

CoreEngine::~CoreEngine() {
    if (!p) return;
    cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    for (auto &e : p->ev_shape) {
        cudaEventDestroy(e[0]);
        cudaEventDestroy(e[1]);
    }
    cudaEventDestroy(p->done);
    cudaStreamDestroy(p->stream);
    cudaFreeHost(p->hb);
    cudaFree(p->db);
    delete p;
}

void CoreEngine::enter() {
    std::lock_guard<std::mutex> lk(mu);
    ++active;
}

void CoreEngine::leave() {
    std::unique_lock<std::mutex> lk(mu);
    --active;
    if (!p->pending.empty() && (int)p->pending.size() >= active) launch_or_fail_locked();
    cv.notify_all();
}

// Runs under mu: the pending problems as one graph launch.
void CoreEngine::launch_locked() {
    Impl &I = *p;
    CoreBatch &b = *I.hb;
    const int cnt = (int)I.pending.size();
    // the shape of each problem: its class's choice, or (while the class is
    // measured) the next candidate it has not timed
    int cls_shape[4];
    for (int cl = 0; cl < 4; ++cl) {
        if (I.chosen[cl] >= 0) {
            cls_shape[cl] = I.chosen[cl];
        } else {
            cls_shape[cl] = I.trial[cl] % CORE_SHAPES;
        }
    }
    b.count = cnt;
    b.fg_off[0] = 0;
    for (int s = 0; s < CORE_SHAPES; ++s) b.tile_off[s][0] = 0;
    double terms[CORE_SHAPES] = {0, 0, 0};
    int cls_of_shape[CORE_SHAPES] = {-1, -1, -1};
    for (int q = 0; q < cnt; ++q) {
        Context &c = *I.pending[q];
        const BlockDev &bd = *c.blocks[0];
        CoreItem &it = b.it[q];
        it.m = c.m;
        it.n = bd.n;
        it.A = bd.dense.p + bd.h_dense_off[bd.h_perm[0]];
        it.con = bd.con.p;
        it.perm = bd.perm.p;
        it.X = c.X.buf.p;
        it.Zi = c.invZ.buf.p;
        it.F = c.Fbuf.p;
        it.G = c.Gbuf.p;
        it.B = c.B.p;
        it.info = c.info.p;
        const int ntl = (bd.n + 31) / 32;
        b.fg_off[q + 1] = b.fg_off[q] + c.m * ntl * ntl;
        const int cl = size_class(c.m);
        const int s = cls_shape[cl];
        b.shape[q] = s;
        for (int t = 0; t < CORE_SHAPES; ++t) {
            long tiles = 0;
            if (t == s) {
                const long tr = (c.m + SHAPES[t].bm - 1) / SHAPES[t].bm, tc = (c.m + SHAPES[t].bn - 1) / SHAPES[t].bn;
                tiles = tr * tc;
            }
            b.tile_off[t][q + 1] = b.tile_off[t][q] + tiles;
        }
        terms[s] += 0.5 * (double)c.m * (c.m + 1) * bd.n * bd.n;
        if (cls_of_shape[s] < 0 || I.chosen[cls_of_shape[s]] >= 0) cls_of_shape[s] = cl; // the class that measures it
        // the problem's inputs (X, Z^-1 on its own stream) come first
        CK(cudaEventRecord(c.core_ready, c.stream));
        CK(cudaStreamWaitEvent(I.stream, c.core_ready, 0));
    }
    b.total_fg = b.fg_off[cnt];
    CK(cudaGraphLaunch(I.exec, I.stream));
    CK(cudaEventRecord(I.done, I.stream));
    for (int q = 0; q < cnt; ++q) CK(cudaStreamWaitEvent(I.pending[q]->stream, I.done, 0));
    // autotuner: time the shapes this batch measured (one class each)
    bool measuring = false;
    for (int cl = 0; cl < 4; ++cl) measuring |= I.chosen[cl] < 0;
    if (measuring) {
        CK(cudaEventSynchronize(I.done));
        for (int s = 0; s < CORE_SHAPES; ++s) {
            if (terms[s] <= 0.0 || cls_of_shape[s] < 0) continue;
            const int cl = cls_of_shape[s];
            if (I.chosen[cl] >= 0 || I.trial[cl] % CORE_SHAPES != s) continue;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, I.ev_shape[s][0], I.ev_shape[s][1]));
            I.per_term[cl][s] = ms / terms[s];
            ++I.trial[cl];
            if (I.trial[cl] >= CORE_SHAPES) {
                int best = 0;
                for (int t = 1; t < CORE_SHAPES; ++t)
                    if (I.per_term[cl][t] >= 0.0 && I.per_term[cl][t] < I.per_term[cl][best]) best = t;
                I.chosen[cl] = best;
            }
        }
    }
    ++generation;
    I.pending.clear();
}

// launch_locked; a failure ends the gathering for all its members.
void CoreEngine::launch_or_fail_locked() {
    const unsigned long gen = generation;
    try {
        launch_locked();
    } catch (const Error &e) {
        failed_generation = gen;
        failed_msg = e.what();
        p->pending.clear();
        ++generation;
    }
    cv.notify_all();
}

int CoreEngine::schur_factor(Context &c) {
    CK(cudaMemsetAsync(c.info.p, 0, sizeof(int), c.stream));
    c.winv_valid = false;
    {
        std::unique_lock<std::mutex> lk(mu);
        if (p->pending.empty()) p->first_wait = std::chrono::steady_clock::now();
        p->pending.push_back(&c);
        const unsigned long gen = generation;
        if ((int)p->pending.size() >= active || (int)p->pending.size() >= CORE_CAP) {
            launch_or_fail_locked();
        } else {
            while (generation == gen) {
                const auto deadline = p->first_wait + std::chrono::microseconds(CORE_WAIT_US);
                if (cv.wait_until(lk, deadline) == std::cv_status::timeout && generation == gen) launch_or_fail_locked();
            }
        }
        if (failed_generation == gen) throw Error(ERR_CUDA, "batched core: " + failed_msg);
    }
    int info = 0;
    d2h(c, &info, c.info.p, sizeof(int));
    return potrf_info_check(info);
}

std::string CoreEngine::tuning() const {
    std::string s;
    for (int cl = 0; cl < 4; ++cl) {
        static const char *names[4] = {"m<=64", "m<=128", "m<=256", "m<=1024"};
        if (!s.empty()) s += ", ";
        s += names[cl];
        s += ": ";
        if (p->chosen[cl] < 0) {
            s += "untuned";
        } else {
            s += std::to_string(SHAPES[p->chosen[cl]].bm) + "x" + std::to_string(SHAPES[p->chosen[cl]].bn);
        }
    }
    return s;
}

} // namespace sddd
