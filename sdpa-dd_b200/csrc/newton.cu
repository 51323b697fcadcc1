// The device side of the reference's Newton step, update and residuals
// (sdpa_newton.cpp, sdpa_dataset.cpp), on block spaces resident in HBM.
#include "newton.h"

#include <algorithm>
#include <cstring>

#include "blas.h"
#include "devops.cuh"
#include "sparse_chol.h"

namespace sddd {

static const dd_t ONE = {1.0, 0.0};
static const dd_t MONE = {-1.0, 0.0};

// --------------------------------------------------- per-constraint A_k . M
// InputData::multi_InnerProductToA (sdpa_dataset.cpp:477-485) followed by
// "v = v * (-1); v = v + w" (the callers' Lal::let pair, Rscal then Raxpy).
__global__ void constraint_inner_kernel(int m, const BlockView *views, const long *off, const int *cb_ptr, const int *cb_block, const int *cb_t,
                                        const dd_t *M, const dd_t *addv, dd_t *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    dd_t ret = dd_zero();
    for (int p = cb_ptr[i]; p < cb_ptr[i + 1]; ++p) {
        const int l = cb_block[p], t = cb_t[p];
        const BlockView &v = views[l];
        const dd_t *Ml = M + off[l];
        dd_t tmp;
        const long doff = v.dense_off[t];
        if (doff >= 0) {
            tmp = seq_dot((long)v.n * v.n, v.dense + doff, Ml);
        } else {
            const int o = v.coo_off[t];
            tmp = sparse_dot_dense(v.n, v.nnz[t], v.row + o, v.col + o, v.val + o, Ml);
        }
        ret = dd_acc(ret, tmp);
    }
    st_dd(out + i, dd_acc(dd_mul(MONE, ret), dd_mul(ONE, ld_dd(addv + i))));
}

// The same for one SDP block whose constraints are all dense: the block of
// M is staged in shared memory once per CTA (every thread reads the same
// entry at the same step), and each thread streams its constraint's n^2
// entries with the next 16 in flight while it sums the current 16, in
// Rdot's order.
constexpr int INNER_CHUNK = 16;
constexpr int INNER_DENSE1_THREADS = 128;
__global__ void __launch_bounds__(INNER_DENSE1_THREADS) constraint_inner_dense1_kernel(int m, const BlockView *views, const int *cb_ptr,
                                                                                     const int *cb_t, const dd_t *M, const dd_t *addv, dd_t *out) {
    extern __shared__ double2 ms[];
    const int n = views[0].n;
    const long nn = (long)n * n;
    for (long e = threadIdx.x; e < nn; e += blockDim.x) ms[e] = *reinterpret_cast<const double2 *>(M + e);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const dd_t *A = views[0].dense + views[0].dense_off[cb_t[cb_ptr[i]]];
    dd_t t = dd_zero();
    dd_t a[INNER_CHUNK], b[INNER_CHUNK];
    const long full = nn / INNER_CHUNK * INNER_CHUNK;
    if (full > 0) {
#pragma unroll
        for (int u = 0; u < INNER_CHUNK; ++u) a[u] = ld_dd(A + u);
    }
    for (long k = 0; k < full; k += INNER_CHUNK) {
#pragma unroll
        for (int u = 0; u < INNER_CHUNK; ++u) b[u] = a[u];
        if (k + INNER_CHUNK < full) {
#pragma unroll
            for (int u = 0; u < INNER_CHUNK; ++u) a[u] = ld_dd(A + k + INNER_CHUNK + u);
        }
#pragma unroll
        for (int u = 0; u < INNER_CHUNK; ++u) {
            const double2 y = ms[k + u];
            t = dd_acc(t, dd_mul(b[u], dd_make(y.x, y.y)));
        }
    }
    for (long k = full; k < nn; ++k) {
        const double2 y = ms[k];
        t = dd_acc(t, dd_mul(ld_dd(A + k), dd_make(y.x, y.y)));
    }
    // seq_dot's "0 + templ", then the caller's ret += tmp from zero
    const dd_t ret = dd_acc(dd_zero(), dd_acc(dd_zero(), t));
    st_dd(out + i, dd_acc(dd_mul(MONE, ret), dd_mul(ONE, ld_dd(addv + i))));
}

void constraint_inner(Context &c, const Space &M, const dd_t *addv, dd_t *out) {
    if (c.inner_dense1) {
        const size_t smem = sizeof(dd_t) * (size_t)c.sizes[0] * c.sizes[0];
        static thread_local bool attr[64] = {};
        int dev = 0;
        CK(cudaGetDevice(&dev));
        if (!attr[dev & 63]) {
            CK(cudaFuncSetAttribute(constraint_inner_dense1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INNER_DENSE1_SMEM));
            attr[dev & 63] = true;
        }
        constraint_inner_dense1_kernel<<<ceil_div(c.m, INNER_DENSE1_THREADS), INNER_DENSE1_THREADS, smem, c.stream>>>(
            c.m, c.views.p, c.cb_ptr.p, c.cb_t.p, M.buf.p + c.off[0], addv, out);
        CK_LAUNCH();
        return;
    }
    constraint_inner_kernel<<<ceil_div(c.m, 64), 64, 0, c.stream>>>(c.m, c.views.p, c.d_off.p, c.cb_ptr.p, c.cb_block.p, c.cb_t.p, M.buf.p, addv, out);
    CK_LAUNCH();
}

// ------------------------------------------------------- sum_k y_k A_k
// InputData::multi_plusToA (sdpa_dataset.cpp:488-493), entry by entry, then
// mode 0 (compute_DzMat, sdpa_newton.cpp:1318-1327): r = -r (+ D)
// mode 1 (Residuals::compute, sdpa_dataset.cpp:632-636): r = -r + C - Z
// One launch per run of equal blocks: CTA row t takes block first + t.
__global__ void sum_yA_kernel(const BlockView *views, int first, long nn, const dd_t *y, dd_t *out, int mode, const dd_t *D, const dd_t *Z) {
    const BlockView v = views[first + blockIdx.y];
    const long ne = (long)v.n * v.n;
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    out += blockIdx.y * nn;
    if (D) D += blockIdx.y * nn;
    if (Z) Z += blockIdx.y * nn;
    dd_t acc = dd_zero();
    if (v.all_dense) {
        // the operands of eight steps go out ahead of their terms (the
        // sum's order is unchanged)
        int t = 0;
        for (; t + 8 <= v.nc; t += 8) {
            long o[8];
            int k[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                o[u] = v.dense_off[t + u];
                k[u] = v.con[t + u];
            }
            dd_t a[8], b[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                a[u] = ld_dd(v.dense + o[u] + e);
                b[u] = ld_dd(y + k[u]);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) acc = dd_acc(acc, dd_mul(a[u], b[u]));
        }
        for (; t < v.nc; ++t) acc = dd_acc(acc, dd_mul(ld_dd(v.dense + v.dense_off[t] + e), ld_dd(y + v.con[t])));
    } else {
        for (int q = v.el_ptr[e]; q < v.el_ptr[e + 1]; ++q) acc = dd_acc(acc, dd_mul(v.el_val[q], ld_dd(y + v.el_con[q])));
    }
    dd_t r = dd_mul(MONE, acc);
    if (mode == 0) {
        if (D) r = dd_acc(r, dd_mul(ONE, ld_dd(D + e)));
    } else {
        if (v.c_present) {
            if (v.c_dense) {
                r = dd_acc(r, dd_mul(ONE, ld_dd(v.c_dense_val + e)));
            } else {
                for (int q = v.c_el_ptr[e]; q < v.c_el_ptr[e + 1]; ++q) r = dd_acc(r, dd_mul(v.c_el_val[q], ONE));
            }
        }
        r = dd_acc(r, dd_mul(MONE, ld_dd(Z + e)));
    }
    st_dd(out + e, r);
}

void sum_yA(Context &c, const dd_t *y, Space &out, int mode, const Space *D, const Space *Z) {
    for (const BlockRun &r : c.runs) {
        const long nn = (long)r.n * r.n;
        for (int b0 = 0; b0 < r.count; b0 += MAX_GRID_YZ) {
            const int l = r.first + b0;
            sum_yA_kernel<<<dim3(ceil_div(nn, 128), std::min(MAX_GRID_YZ, r.count - b0)), 128, 0, c.stream>>>(
                c.views.p, l, nn, y, out.blk(c.off, l), mode, D ? D->blk(c.off, l) : nullptr, Z ? Z->blk(c.off, l) : nullptr);
            CK_LAUNCH();
        }
    }
}

// ------------------------------------------------------------ init point
__global__ void set_identity_kernel(dd_t *A, int n, dd_t v) {
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    st_dd(A + e, (e % n == e / n) ? v : dd_zero());
}
static void set_identity(Context &c, Space &s, dd_t v) {
    for (int l = 0; l < c.nSDP; ++l) {
        int n = c.sizes[l];
        set_identity_kernel<<<ceil_div((long)n * n, 256), 256, 0, c.stream>>>(s.blk(c.off, l), n, v);
        CK_LAUNCH();
    }
}

void init_point(Context &c, dd_t lambda) {
    set_identity(c, c.X, lambda);
    set_identity(c, c.Z, lambda);
    fill(c.stream, c.y.p, c.m, dd_zero());
    dd_t ris = dd_div(ONE, dd_sqrt(lambda));
    set_identity(c, c.invCholX, ris);
    set_identity(c, c.invCholZ, ris);
    set_identity(c, c.invZ, dd_div(ONE, lambda));
}

// ------------------------------------------------------- inverses of X, Z
// Jal::getInvChol / getInvCholAndInv (sdpa_jordan.cpp:123-170): copy,
// Rpotrf, zero the upper triangle, Rtrsm on the identity; for Z also
// Z^-1 = L_Z^-T L_Z^-1 by Rtrmm.
void compute_inverse_async(Context &c) {
    cudaStream_t st = c.stream;
    if (!c.aux) {
        CK(cudaStreamCreateWithFlags(&c.aux, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c.aux_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c.aux_join, cudaEventDisableTiming));
    }
    CK(cudaMemsetAsync(c.info.p, 0, sizeof(int) * 2, st));
    CK(cudaMemcpyAsync(c.W1.buf.p, c.X.buf.p, sizeof(dd_t) * c.space_len, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c.W2.buf.p, c.Z.buf.p, sizeof(dd_t) * c.space_len, cudaMemcpyDeviceToDevice, st));
    // X's factors on the main stream, Z's (and Z^-1) on the second one
    CK(cudaEventRecord(c.aux_fork, st));
    CK(cudaStreamWaitEvent(c.aux, c.aux_fork, 0));
    for (int side = 0; side < 2; ++side) {
        cudaStream_t s = side == 0 ? st : c.aux;
        const Space &W = side == 0 ? c.W1 : c.W2;
        Space &inv = side == 0 ? c.invCholX : c.invCholZ;
        int *info = c.info.p + side;
        dd_t *rdiag = c.rdiag.p + 128 * side;
        for (const BlockRun &r : c.runs) {
            const int n = r.n;
            const long nn = (long)n * n;
            dd_t *w = W.blk(c.off, r.first);
            if (n <= POTRF_NB) {
                potrf_batched(s, w, n, n, nn, r.count, info);
            } else {
                for (int t = 0; t < r.count; ++t) potrf(s, w + t * nn, n, n, info, rdiag);
            }
            zero_upper(s, w, n, n, r.count, nn);
            inv_lower(s, w, n, n, inv.blk(c.off, r.first), n, r.count, nn, nn);
            if (side == 1) trmm_lt(s, c.invCholZ.blk(c.off, r.first), n, n, c.invZ.blk(c.off, r.first), n, r.count, nn, nn);
        }
    }
    CK(cudaEventRecord(c.aux_join, c.aux));
    CK(cudaStreamWaitEvent(st, c.aux_join, 0));
}

bool compute_inverse(Context &c) {
    compute_inverse_async(c);
    ScalarBatch sb(c);
    const int g = sb.inverse_info();
    sb.fetch();
    return sb.inverse_ok(g);
}

int ScalarBatch::inverse_info() {
    const int g = group(1);
    CK(cudaMemcpyAsync(c.scal.p + groups[g].first, c.info.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
    return g;
}

bool ScalarBatch::inverse_ok(int g) const {
    int info[2];
    std::memcpy(info, &host[groups[g].first], sizeof(info));
    potrf_info_check(info[0]);
    potrf_info_check(info[1]);
    return info[0] == 0 && info[1] == 0;
}

// ------------------------------------------------------------ Newton step
void triple(Context &c, const Space &A, const Space &B, const Space &C, Space &out) {
    // Jal::ns_jordan_triple_product: work = A B; out = work C (two Rgemm)
    for (const BlockRun &r : c.runs) {
        const int n = r.n, l = r.first;
        const long nn = (long)n * n;
        gemm(c.stream, 'N', 'N', GEMM_STORE, n, n, n, A.blk(c.off, l), n, nn, B.blk(c.off, l), n, nn, c.W2.blk(c.off, l), n, nn, r.count, false);
        gemm(c.stream, 'N', 'N', GEMM_STORE, n, n, n, c.W2.blk(c.off, l), n, nn, C.blk(c.off, l), n, nn, out.blk(c.off, l), n, nn, r.count, false);
    }
}

void make_rhs(Context &c, bool corrector, dd_t beta_mu, bool dual_infeasible) {
    cudaStream_t st = c.stream;
    const long L = c.space_len;
    // r_zinv = beta*mu * Z^-1 - X  (compute_rMat, sdpa_newton.cpp:821-837)
    copy_scal(st, c.invZ.buf.p, c.rzinv.buf.p, L, beta_mu);
    axpy(st, c.rzinv.buf.p, c.X.buf.p, c.rzinv.buf.p, L, MONE);
    if (corrector) {
        triple(c, c.Dx, c.Dz, c.invZ, c.W1);
        axpy(st, c.rzinv.buf.p, c.W1.buf.p, c.rzinv.buf.p, L, MONE);
    }
    // Make_gVec (sdpa_newton.cpp:839-893)
    if (dual_infeasible) {
        if (!corrector) triple(c, c.X, c.dualMat, c.invZ, c.xrdzinv);
        axpy(st, c.rzinv.buf.p, c.xrdzinv.buf.p, c.W1.buf.p, L, MONE);
    } else {
        CK(cudaMemcpyAsync(c.W1.buf.p, c.rzinv.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    }
    constraint_inner(c, c.W1, c.primalVec.p, c.g.p);
}

int schur_factor(Context &c) {
    if (c.sparse_active()) {
        // Lal::getCholesky(SparseMatrix&, int*) reports no failure: a
        // negative pivot becomes a zero row (sdpa_linear.cpp:366-372)
        c.winv_valid = false;
        sparse_factor_B(c);
        return 0;
    }
    CK(cudaMemsetAsync(c.info.p, 0, sizeof(int), c.stream));
    OzakiWork *tc = c.tc_slices > 0 ? &tc_work(c, c.m, c.tc_slices) : nullptr;
    c.winv_valid = false;
    potrf(c.stream, c.B.p, c.m, c.m, c.info.p, c.rdiag.p, tc);
    int info = 0;
    d2h(c, &info, c.info.p, sizeof(int));
    potrf_info_check(info);
    if (tc) {
        ozaki_check(c.stream, *tc);
        if (info == 0) {
            // the split form's solves go by blocks (trsv_blocked)
            c.trsv_winv.alloc((size_t)ceil_div(c.m, 64) * 64 * 64);
            trsv_diag_inverse(c.stream, c.B.p, c.m, c.m, c.trsv_winv.p);
            c.winv_valid = true;
        }
    }
    return info;
}

void solve_B(Context &c, dd_t *x) {
    if (c.sparse_active()) {
        sparse_solve(c, x);
        return;
    }
    TrsvSync &sync = trsv_sync(c, c.m);
    if (c.winv_valid) {
        trsv_blocked(c.stream, 'N', c.B.p, c.m, c.m, c.trsv_winv.p, x, sync);
        trsv_blocked(c.stream, 'T', c.B.p, c.m, c.m, c.trsv_winv.p, x, sync);
    } else {
        trsv_lower(c.stream, 'N', c.B.p, c.m, c.m, x, sync, c.shared_gpu);
        trsv_lower(c.stream, 'T', c.B.p, c.m, c.m, x, sync, c.shared_gpu);
    }
    trsv_check(c.stream, sync);
}

void solve_dy(Context &c) {
    CK(cudaMemcpyAsync(c.Dy.p, c.g.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToDevice, c.stream));
    solve_B(c, c.Dy.p);
}

void make_dz_dx(Context &c, bool dual_infeasible) {
    sum_yA(c, c.Dy.p, c.Dz, 0, dual_infeasible ? &c.dualMat : nullptr, nullptr);
    triple(c, c.X, c.Dz, c.invZ, c.W1);
    axpy(c.stream, c.rzinv.buf.p, c.W1.buf.p, c.Dx.buf.p, c.space_len, MONE);
    for (const BlockRun &r : c.runs) symmetrize(c.stream, c.Dx.blk(c.off, r.first), r.n, r.count, (long)r.n * r.n);
}

// ------------------------------------------------------------ inner products
// Each reduction writes its partial results (one per block, or one) to
// slots of c.scal; a ScalarBatch lays several reductions side by side and
// reads them all back with one copy, so that independent scalars of one
// step cost one host round trip.  The host sums a group's slots in order
// from zero with "+=", as the reference sums its per-block results.
int ScalarBatch::group(int count) {
    groups.push_back({used, count});
    used += count;
    if ((size_t)used > c.scal.n) throw Error(ERR_STATE, "scalar batch: more result slots than the context holds");
    return (int)groups.size() - 1;
}

void ScalarBatch::fetch() {
    host.resize(used);
    if (used > 0) d2h(c, host.data(), c.scal.p, sizeof(dd_t) * used);
}

dd_t ScalarBatch::sum(int g) const {
    dd_t r = dd_zero();
    for (int s = 0; s < groups[g].second; ++s) r = dd_acc(r, host[groups[g].first + s]);
    return r;
}

dd_t ScalarBatch::value(int g) const { return host[groups[g].first]; }

// Lal::getInnerProduct(DenseLinearSpace, DenseLinearSpace)
// (sdpa_linear.cpp:1571-1611): Rdot per block, summed with "+=".
int ScalarBatch::inner_space(const Space &a, const Space &b) {
    const int g = group(c.nSDP);
    dd_t *out = c.scal.p + groups[g].first;
    for (const BlockRun &r : c.runs) {
        const long nn = (long)r.n * r.n;
        dot_batched(c.stream, a.blk(c.off, r.first), nn, b.blk(c.off, r.first), nn, nn, r.count, out + r.first, c.red.p);
    }
    return g;
}

__global__ void sparse_inner_kernel(int n, int nnz, const int *row, const int *col, const dd_t *val, const dd_t *D, dd_t *out) {
    if (threadIdx.x == 0) st_dd(out, sparse_dot_dense(n, nnz, row, col, val, D));
}

// The blocks whose product with C is one chain (sparse C, or dense C of at
// most DOT_SEQ_TERMS entries) in one launch: CTA l, result to its slot.
constexpr long DOT_SEQ_TERMS = 1024; // the longest dot that dot() runs as one chain
__global__ void inner_C_small_kernel(const BlockView *views, const int *slot, const long *off, const dd_t *x, dd_t *out) {
    if (threadIdx.x != 0) return;
    const int l = blockIdx.x;
    const BlockView v = views[l];
    const int s = slot[l];
    if (s < 0 || !v.c_present) return;
    const dd_t *D = x + off[l];
    if (!v.c_dense) {
        st_dd(out + s, sparse_dot_dense(v.n, v.c_nnz, v.c_row, v.c_col, v.c_val, D));
        return;
    }
    const long nn = (long)v.n * v.n;
    if (nn > DOT_SEQ_TERMS) return;
    dd_t t = dd_zero();
    for (long i = 0; i < nn; ++i) t = dd_acc(t, dd_mul(ld_dd(v.c_dense_val + i), ld_dd(D + i)));
    st_dd(out + s, dd_acc(dd_zero(), t));
}

// Lal::getInnerProduct(SparseLinearSpace C, DenseLinearSpace X)
// (sdpa_linear.cpp:1616-1650) over C's nonzero SDP blocks: one result slot
// per such block, summed in block order on the host.
int ScalarBatch::inner_C(const Space &x) {
    if (c.c_slot_host.size() != (size_t)c.nSDP) {
        c.c_slot_host.assign(c.nSDP, -1);
        c.c_nslots = 0;
        for (int l = 0; l < c.nSDP; ++l)
            if (c.blocks[l]->c_present) c.c_slot_host[l] = c.c_nslots++;
        c.c_slot.upload(c.c_slot_host, c.stream);
    }
    const int g = group(c.c_nslots);
    if (c.c_nslots == 0) return g;
    dd_t *out = c.scal.p + groups[g].first;
    inner_C_small_kernel<<<c.nSDP, 32, 0, c.stream>>>(c.views.p, c.c_slot.p, c.d_off.p, x.buf.p, out);
    CK_LAUNCH();
    for (int l = 0; l < c.nSDP; ++l) {
        const BlockDev &bd = *c.blocks[l];
        const long nn = (long)bd.n * bd.n;
        if (bd.c_present && bd.c_dense && nn > DOT_SEQ_TERMS)
            dot(c.stream, bd.c_dense_val.p, 1, x.blk(c.off, l), 1, nn, out + c.c_slot_host[l], c.red.p + 256 * (c.c_slot_host[l] % 8));
    }
    return g;
}

// Lal::getInnerProduct(Vector, Vector): Rdot over m.
int ScalarBatch::inner_b(const dd_t *v) {
    const int g = group(1);
    dot(c.stream, c.b.p, 1, v, 1, c.m, c.scal.p + groups[g].first, c.red.p);
    return g;
}

// max |x_i| (Residuals::computeMaxNorm): one slot, taken as is.
int ScalarBatch::maxabs_of(const dd_t *x, long n, int scratch) {
    const int g = group(1);
    maxabs(c.stream, x, n, c.scal.p + groups[g].first, c.red.p + 512 * scratch);
    return g;
}

dd_t inner_space(Context &c, const Space &a, const Space &b) {
    ScalarBatch sb(c);
    const int g = sb.inner_space(a, b);
    sb.fetch();
    return sb.sum(g);
}

dd_t inner_C(Context &c, const Space &x) {
    ScalarBatch sb(c);
    const int g = sb.inner_C(x);
    sb.fetch();
    return sb.sum(g);
}

dd_t inner_b(Context &c, const dd_t *v) {
    ScalarBatch sb(c);
    const int g = sb.inner_b(v);
    sb.fetch();
    return sb.sum(g);
}

// ----------------------------------------------------------------- update
void update_point(Context &c, dd_t alphaP, dd_t alphaD) {
    axpy(c.stream, c.X.buf.p, c.Dx.buf.p, c.X.buf.p, c.space_len, alphaP);
    axpy(c.stream, c.y.p, c.Dy.p, c.y.p, c.m, alphaD);
    axpy(c.stream, c.Z.buf.p, c.Dz.buf.p, c.Z.buf.p, c.space_len, alphaD);
}

// -------------------------------------------------------------- residuals
// Residuals::compute (sdpa_dataset.cpp:625-645): the primal residual vector
// and the dual residual matrix, then their max-abs norms into the batch.
void ScalarBatch::residuals(int &gPrimal, int &gDual) {
    constraint_inner(c, c.X, c.b.p, c.primalVec.p);
    sum_yA(c, c.y.p, c.dualMat, 1, nullptr, &c.Z);
    gPrimal = maxabs_of(c.primalVec.p, c.m, 0);
    gDual = maxabs_of(c.dualMat.buf.p, c.space_len, 1);
}

void residuals(Context &c, dd_t &normPrimal, dd_t &normDual) {
    ScalarBatch sb(c);
    int gp, gd;
    sb.residuals(gp, gd);
    sb.fetch();
    normPrimal = sb.value(gp);
    normDual = sb.value(gd);
}

__global__ void lambda_trace_kernel(const dd_t *S, const long *off, const int *sizes, int nb, double lambda, dd_t *out) {
    if (threadIdx.x != 0) return;
    dd_t r = dd_zero();
    for (int b = 0; b < nb; ++b) {
        const int n = sizes[b];
        for (int i = 0; i < n; ++i) r = dd_acc(r, dd_mul_d(ld_dd(S + off[b] + i + (long)n * i), lambda));
    }
    st_dd(out, r);
}

int ScalarBatch::lambda_trace(const Space &s, double lambda) {
    const int g = group(1);
    lambda_trace_kernel<<<1, 32, 0, c.stream>>>(s.buf.p, c.d_off.p, c.d_sizes.p, c.nSDP, lambda, c.scal.p + groups[g].first);
    CK_LAUNCH();
    return g;
}

dd_t lambda_trace(Context &c, const Space &s, double lambda) {
    ScalarBatch sb(c);
    const int g = sb.lambda_trace(s, lambda);
    sb.fetch();
    return sb.sum(g);
}

} // namespace sddd
