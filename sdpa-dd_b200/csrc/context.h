// Device-resident solver state: the problem in its per-block layout and the
// iterate, direction and work spaces of the reference's Solutions /
// Newton / Residuals / WorkVariables (sdpa_dataset.h, sdpa_newton.h), all
// in HBM for the whole solve.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "blas.h"
#include "common.cuh"
#include "ozaki.h"
#include "problem.h"

namespace sddd {

// Device buffer owning cudaMalloc'd memory.  The capacity only grows: a
// context that takes a smaller problem next keeps its memory, so uploads
// in a long-lived context (a batch worker) neither allocate nor free
// (cudaFree would synchronise the whole device).  n is the logical length.
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0, cap = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = cap = 0;
    }
    void alloc(size_t count) {
        if (p && count <= cap) {
            n = count;
            return;
        }
        release();
        if (count == 0) return;
        CK(cudaMalloc(&p, sizeof(T) * count));
        n = cap = count;
    }
    void upload(const std::vector<T> &v, cudaStream_t st) {
        alloc(v.size());
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
    }
};

// Kernel-side view of one block's problem data (pointers into BlockDev).
// Largest single block (bytes of n x n dd) whose constraint inner products
// take the shared-memory form (constraint_inner).
constexpr size_t INNER_DENSE1_SMEM = 160 * 1024;

struct BlockView {
    int n, nc, nsparse, all_dense;
    const int *con, *formula, *perm, *coo_off, *nnz;
    const long *dense_off;
    const int *row, *col;
    const dd_t *val, *dense;
    const int *el_ptr, *el_con;
    const dd_t *el_val;
    int c_present, c_dense, c_nnz;
    const dd_t *c_dense_val;
    const int *c_row, *c_col;
    const dd_t *c_val;
    const int *c_el_ptr;
    const dd_t *c_el_val;
};

// Per-SDP-block problem data on the device.
//  t  : position of a constraint in the block's constraint list (ascending k)
//  s  : position in the order sorted by (NonZeroEffect, k); a pair (i, j) is
//       evaluated by its owner i when s(j) <= s(i) (sdpa_newton.cpp:1024)
struct BlockDev {
    int n = 0, nc = 0;
    int nsparse = 0; // sparse matrices occupy sorted positions [0, nsparse)
    DBuf<int> con;       // [t] constraint index
    DBuf<int> formula;   // [t]
    DBuf<int> effect;    // [t]
    DBuf<int> perm;      // [s] -> t
    DBuf<int> coo_off;   // [t] offset into row/col/val (sparse), -1 dense
    DBuf<int> nnz;       // [t]
    DBuf<long> dense_off; // [t] offset (elements) into dense (dense), -1 sparse
    DBuf<int> row, col;
    DBuf<dd_t> val;
    DBuf<dd_t> dense;    // dense matrices, t order, n*n each
    bool all_dense = false;
    // sum_k y_k A_k by element (when not all dense): CSR over the n*n entries
    DBuf<int> el_ptr, el_con;
    DBuf<dd_t> el_val;
    // C of this block: dense or element lists
    bool c_present = false, c_dense = false;
    DBuf<dd_t> c_dense_val;       // n*n
    DBuf<int> c_row, c_col;       // COO in input order (for the inner product)
    DBuf<dd_t> c_val;
    DBuf<int> c_el_ptr;           // CSR over entries for C accumulation
    DBuf<dd_t> c_el_val;
    // Schur owner lists (sorted positions, ascending)
    std::vector<int> h_ownFG, h_ownF3;
    DBuf<int> ownFG, ownF3;
    DBuf<int> fg_index;  // [s] -> index in ownFG or -1
    bool fg_dense_contig = false; // all FG owners dense and contiguous in t
    // F = A_i Z^-1 for sparse FG owners as row lists: row i of F is the
    // ordered sum of v * (row src of Z^-1) (Raxpy row updates,
    // sdpa_linear.cpp:832-893); per owner r: rl_off[r] into rl_ptr (n+1)
    std::vector<int> h_rl_off;
    DBuf<int> rl_off, rl_ptr, rl_src;
    DBuf<dd_t> rl_val;
    std::vector<int> h_perm;
    std::vector<long> h_dense_off;
    BlockView view() const;
    int nFG() const { return (int)h_ownFG.size(); }
    int nF3() const { return (int)h_ownF3.size(); }
};

// A block space (DenseLinearSpace restricted to SDP blocks): one device
// buffer, block l at offset off[l], n_l x n_l column-major.
struct Space {
    DBuf<dd_t> buf;
    dd_t *blk(const std::vector<long> &off, int l) const { return buf.p + off[l]; }
};

class CoreEngine;
struct SparseDev;

// The Schur build of a problem with many blocks as one CUDA graph (schur.cu):
// every block's pairs on one of a few parallel branches, each with its own
// F/G scratch, the pair values into per-block staging squares, then one
// kernel that adds each entry's block values to B in block order.
struct SchurGraph {
    unsigned long gen = 0;     // upload generation the graph was built for (0: none)
    bool eligible = false;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> joined;
    cudaEvent_t forked = nullptr;
    DBuf<dd_t> stage, F, G;
    DBuf<int> ent;             // per B entry (i >= j): i, j
    DBuf<int> ptr;             // per entry: its contributions [ptr[e], ptr[e+1])
    DBuf<long> src;            // contributions: staging offsets, blocks in order
    int nent = 0;
    ~SchurGraph();
};

// Consecutive SDP blocks of one order: they lie back to back in every
// space (block first + t at off[first] + t n^2), so the per-block dense
// kernels run once for the whole run with a batch stride of n^2.
struct BlockRun {
    int first, count, n;
};

struct Context {
    int device = 0;
    // a batch worker's batched Newton core (batched.h), or null; the event
    // marks the core's inputs ready on this context's stream
    CoreEngine *core = nullptr;
    cudaEvent_t core_ready = nullptr;
    cudaStream_t stream = nullptr;
    // a second stream for work independent of the main stream's (the
    // inverses of Z beside those of X), joined back through events
    cudaStream_t aux = nullptr;
    cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
    bool shared_gpu = false; // a batch worker: other contexts' streams share the GPU
    // pinned host staging for the small device-to-host reads of the solver
    // (scalars, status words): a copy into pageable memory goes through the
    // driver's shared staging path, which ties the streams of concurrent
    // contexts together
    static constexpr size_t H_PIN_BYTES = 1 << 16;
    void *h_pin = nullptr;
    // with shared_gpu: a blocking-sync event the host waits on instead of
    // spinning in cudaStreamSynchronize (many workers share the host cores)
    cudaEvent_t sync_ev = nullptr;
    std::string last_error;
    bool have_problem = false;
    Problem prob;
    int m = 0, nSDP = 0;
    long nDim = 0;
    std::vector<int> sizes;
    std::vector<long> off; // block offsets within a space
    std::vector<BlockRun> runs;
    // result slot of each block with a C part (inner_C), built on first use
    std::vector<int> c_slot_host;
    DBuf<int> c_slot;
    int c_nslots = 0;
    long space_len = 0;
    std::vector<std::unique_ptr<BlockDev>> blocks;
    DBuf<BlockView> views; // [l]
    DBuf<long> d_off;      // [l] block offsets within a space
    DBuf<int> d_sizes;     // [l] block sizes
    // per constraint: (block, t) pairs ascending by block
    DBuf<int> cb_ptr, cb_block, cb_t;
    // every constraint is one dense matrix of the single SDP block, whose
    // order fits the shared-memory form of the constraint inner products
    bool inner_dense1 = false;
    DBuf<dd_t> b;
    // iterate and derived (Solutions)
    Space X, Z, invCholX, invCholZ, invZ;
    DBuf<dd_t> y;
    // Newton
    Space Dx, Dz, rzinv, xrdzinv;
    DBuf<dd_t> Dy, g;
    DBuf<dd_t> B;   // m x m Schur matrix, factored in place
    // Residuals
    Space dualMat;
    DBuf<dd_t> primalVec;
    // WorkVariables
    Space W1, W2;
    // Schur work: F_i and G_i of FG owners (largest block)
    DBuf<dd_t> Fbuf, Gbuf;
    // small scratch
    DBuf<dd_t> scal;   // device scalars: max(64, 4 nSDP + 8) result slots
    DBuf<dd_t> red;    // reduction scratch
    DBuf<int> info;
    DBuf<dd_t> rdiag;
    DBuf<int> trsv_flags; // progress words of the one-launch triangular solve
    // step-length eigenvalue work: block lists and Lanczos vectors (kept, so
    // that no call allocates or frees)
    DBuf<int> eig_ids_big, eig_ids_small;
    unsigned long eig_ids_gen = 0;
    DBuf<dd_t> eig_work;
    TrsvSync trsv;
    // budget of every bounded device wait of this context's kernels (the
    // triangular solves' block flags, the split kernel's barriers), and a
    // block whose completion flag the triangular solves withhold (-1: none;
    // set only by tests of the bounded waits)
    unsigned long long wait_ns = 2000000000ull;
    int withhold_block = -1;
    // tensor-core split of the Cholesky trailing updates of B: slices per
    // value (8..16), 0 = plain dd GEMMs (the reference's operation order)
    int tc_slices = 0;
    // inverses of the 64 x 64 diagonal blocks of the split form's factor of
    // B (the blocked solves' W_c); valid from a successful split
    // factorisation until the next factorisation
    DBuf<dd_t> trsv_winv;
    bool winv_valid = false;
    DBuf<int8_t> tc_slice_buf;
    DBuf<int> tc_exps, tc_err;
    OzakiWork tc;
    // the split of the Schur complement's F1 pair products (W^T V over K =
    // n^2): slices, row exponents, error word, and the pair values
    DBuf<int8_t> tcg_sw, tcg_sv;
    DBuf<int> tcg_ew, tcg_ev, tcg_err;
    DBuf<dd_t> tcg_pairs;
    OzakiGemmWork tcg;
    // a user-given initial point (the reference's -id / -is), used by the
    // solver's start in place of lambda I
    bool has_init = false;
    Space init_X, init_Z;
    DBuf<dd_t> init_y;
    // adjoint of the final iterate (adjoint.cu): u = B^-1 (g_y - A(g_Z')),
    // the symmetric gradient R of the dual constraint's right-hand side,
    // and work; allocated on first use
    DBuf<dd_t> adj_u, adj_v, adj_x;
    Space adj_R, adj_T;
    bool adj_valid = false;
    // the limit at the optimum (adjoint_limit): eigenvectors of X (Q, and
    // Q with the range first), work, the saved X and Z^-1, the three
    // central-point adjoints and the null-space inverse K per block
    Space lim_Q, lim_Qp, lim_T, lim_M, lim_Xs, lim_Zs, lim_R[3];
    DBuf<dd_t> lim_u[3], lim_lam, lim_K, lim_Kw;
    DBuf<int> lim_perm, lim_sweeps;
    DBuf<double> lim_offr;
    // algorithmic dd-flop counts of one Make_bMat and one Cholesky of B
    double schur_flops = 0, chol_flops = 0;
    // Schur form: SchurMode of sparse_schur.h (the reference's thresholds,
    // always dense, always sparse) and, when B is sparse, its ordering,
    // symbolic factor and tiles (sparse_chol.h)
    int schur_mode = 0;
    SparseDev *sp = nullptr;
    // problem uploads so far (cached graphs and plans are per upload)
    unsigned long upload_gen = 0;
    SchurGraph *sg = nullptr;
    bool sparse_active() const;
    ~Context();
};

Context *create_context(int device);
void upload_problem(Context &c, Problem &&p);
void alloc_state(Context &c);
// The triangular-solve progress words, grown (and zeroed) to cover order n.
TrsvSync &trsv_sync(Context &c, int n);
// The split workspace for an order-n factorisation with `slices` slices
// (grown as needed).
OzakiWork &tc_work(Context &c, int n, int slices);
// The split workspace for an n x n pair product over K values (grown as
// needed).
OzakiGemmWork &tcg_work(Context &c, int n, long K, int slices);

// Marks the context as one of many sharing the GPU (a batch worker): short
// triangular solves in one CTA; with blocking_waits, host waits block on an
// event instead of spinning (for more workers than host cores).
void set_shared_gpu(Context &c, bool blocking_waits);
// Waits for the context's stream (blocking on an event when shared).
void stream_sync(Context &c);
// dst <- bytes at device address src, staged through the context's pinned
// buffer; synchronises the context's stream.
void d2h(Context &c, void *dst, const void *src, size_t bytes);

// Host<->device for spaces laid out as the C-ABI defines: SDP blocks
// concatenated, each n_l x n_l column-major.
void space_to_host(Context &c, const Space &s, dd_t *out);
void space_from_host(Context &c, Space &s, const dd_t *in);

} // namespace sddd
