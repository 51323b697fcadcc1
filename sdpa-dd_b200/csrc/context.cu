// Upload of the problem into its device layout and allocation of the
// solver state (see context.h).
#include "context.h"
#include "sparse_chol.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace sddd {

BlockView BlockDev::view() const {
    BlockView v;
    v.n = n;
    v.nc = nc;
    v.nsparse = nsparse;
    v.all_dense = all_dense ? 1 : 0;
    v.con = con.p;
    v.formula = formula.p;
    v.perm = perm.p;
    v.coo_off = coo_off.p;
    v.nnz = nnz.p;
    v.dense_off = dense_off.p;
    v.row = row.p;
    v.col = col.p;
    v.val = val.p;
    v.dense = dense.p;
    v.el_ptr = el_ptr.p;
    v.el_con = el_con.p;
    v.el_val = el_val.p;
    v.c_present = c_present ? 1 : 0;
    v.c_dense = c_dense ? 1 : 0;
    v.c_nnz = (int)c_row.n;
    v.c_dense_val = c_dense_val.p;
    v.c_row = c_row.p;
    v.c_col = c_col.p;
    v.c_val = c_val.p;
    v.c_el_ptr = c_el_ptr.p;
    v.c_el_val = c_el_val.p;
    return v;
}

bool Context::sparse_active() const { return sp && sp->active; }

SchurGraph::~SchurGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaStream_t s : branch) cudaStreamDestroy(s);
    for (cudaEvent_t e : joined) cudaEventDestroy(e);
    if (forked) cudaEventDestroy(forked);
}

Context::~Context() {
    if (stream) cudaStreamSynchronize(stream);
    delete sg;
    delete sp;
    if (tc.ev_pre) cudaEventDestroy(tc.ev_pre);
    if (tc.ev_diag) cudaEventDestroy(tc.ev_diag);
    if (tc.side) cudaStreamDestroy(tc.side);
    if (sync_ev) cudaEventDestroy(sync_ev);
    if (core_ready) cudaEventDestroy(core_ready);
    if (aux_fork) cudaEventDestroy(aux_fork);
    if (aux_join) cudaEventDestroy(aux_join);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
    if (h_pin) cudaFreeHost(h_pin);
}

void set_shared_gpu(Context &c, bool blocking_waits) {
    c.shared_gpu = true;
    if (blocking_waits && !c.sync_ev) CK(cudaEventCreateWithFlags(&c.sync_ev, cudaEventBlockingSync | cudaEventDisableTiming));
    c.trsv.wait_ev = c.sync_ev;
    c.tc.wait_ev = c.sync_ev;
}

void stream_sync(Context &c) {
    if (c.sync_ev) {
        CK(cudaEventRecord(c.sync_ev, c.stream));
        CK(cudaEventSynchronize(c.sync_ev));
    } else {
        CK(cudaStreamSynchronize(c.stream));
    }
}

void d2h(Context &c, void *dst, const void *src, size_t bytes) {
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    while (bytes > 0) {
        const size_t chunk = bytes < Context::H_PIN_BYTES ? bytes : Context::H_PIN_BYTES;
        CK(cudaMemcpyAsync(c.h_pin, s, chunk, cudaMemcpyDeviceToHost, c.stream));
        stream_sync(c);
        std::memcpy(d, c.h_pin, chunk);
        d += chunk;
        s += chunk;
        bytes -= chunk;
    }
}

OzakiWork &tc_work(Context &c, int n, int slices) {
    const int rows = (int)(ceil_div(n, OZ_ROWS_A) * OZ_ROWS_A);
    if (rows > c.tc.row_cap || !c.tc.slices) {
        CK(cudaStreamSynchronize(c.stream));
        c.tc_slice_buf.alloc((size_t)2 * OZ_MAX_SLICES * rows * OZ_K);
        c.tc_exps.alloc((size_t)rows);
        if (!c.tc_err.p) {
            c.tc_err.alloc(1);
            CK(cudaMemsetAsync(c.tc_err.p, 0, sizeof(int), c.stream));
        }
        c.tc.slices = c.tc_slice_buf.p;
        c.tc.slices_b = c.tc_slice_buf.p + (size_t)OZ_MAX_SLICES * rows * OZ_K;
        c.tc.exps = c.tc_exps.p;
        c.tc.err = c.tc_err.p;
        c.tc.h_err = static_cast<int *>(c.h_pin);
        c.tc.wait_ev = c.sync_ev;
        c.tc.row_cap = rows;
    }
    if (!c.tc.side) {
        CK(cudaStreamCreateWithFlags(&c.tc.side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c.tc.ev_pre, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c.tc.ev_diag, cudaEventDisableTiming));
    }
    c.tc.slices_used = slices;
    c.tc.wait_ns = c.wait_ns;
    return c.tc;
}

OzakiGemmWork &tcg_work(Context &c, int n, long K, int slices) {
    const size_t bytes = ozaki_gemm_slice_bytes(n, K, slices);
    const int rows = (int)(ceil_div(n, 128) * 128);
    if (bytes > c.tcg.slice_bytes || rows > c.tcg.rows_cap || !c.tcg.err) {
        CK(cudaStreamSynchronize(c.stream));
        c.tcg_sw.alloc(bytes);
        c.tcg_sv.alloc(bytes);
        c.tcg_ew.alloc((size_t)rows);
        c.tcg_ev.alloc((size_t)rows);
        if (!c.tcg_err.p) {
            c.tcg_err.alloc(1);
            CK(cudaMemsetAsync(c.tcg_err.p, 0, sizeof(int), c.stream));
        }
        c.tcg.sw = c.tcg_sw.p;
        c.tcg.sv = c.tcg_sv.p;
        c.tcg.slice_bytes = std::max(bytes, c.tcg.slice_bytes);
        c.tcg.ew = c.tcg_ew.p;
        c.tcg.ev = c.tcg_ev.p;
        c.tcg.rows_cap = std::max(rows, c.tcg.rows_cap);
        c.tcg.err = c.tcg_err.p;
        c.tcg.h_err = static_cast<int *>(c.h_pin);
        c.tcg.wait_ev = c.sync_ev;
    }
    c.tcg.slices = slices;
    c.tcg.wait_ns = c.wait_ns;
    return c.tcg;
}

TrsvSync &trsv_sync(Context &c, int n) {
    const int nblk = (int)ceil_div(n, 64);
    if (nblk > c.trsv.capacity || !c.trsv.flags) {
        CK(cudaStreamSynchronize(c.stream));
        c.trsv_flags.alloc((size_t)nblk + 1);
        CK(cudaMemsetAsync(c.trsv_flags.p, 0, sizeof(int) * ((size_t)nblk + 1), c.stream));
        c.trsv = TrsvSync{c.trsv_flags.p, nblk, 0, static_cast<int *>(c.h_pin), c.sync_ev};
    }
    c.trsv.wait_ns = c.wait_ns;
    c.trsv.withhold = c.withhold_block;
    return c.trsv;
}

Context *create_context(int device) {
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw Error(ERR_ARG, "no such CUDA device");
    CK(cudaSetDevice(device));
    auto *c = new Context();
    c->device = device;
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaMallocHost(&c->h_pin, Context::H_PIN_BYTES));
    return c;
}

static void build_block(Context &c, const Problem &P, int l, BlockDev &bd) {
    const int n = P.sdpSize[l];
    const auto &cl = P.cons[l];
    const int nc = (int)cl.size();
    bd.n = n;
    bd.nc = nc;
    std::vector<int> con(cl.begin(), cl.end()), formula(P.formula[l]), effect(nc), coo_off(nc, -1), nnz(nc);
    std::vector<long> dense_off(nc, -1);
    std::vector<int> row, col;
    std::vector<dd_t> val, dense;
    int ndense = 0;
    for (int t = 0; t < nc; ++t) {
        const BlockMat &M = P.A[cl[t]].at(l);
        effect[t] = M.effect;
        if (M.dense) {
            dense_off[t] = (long)ndense * n * n;
            dense.insert(dense.end(), M.val.begin(), M.val.end());
            ++ndense;
            nnz[t] = n * n;
        } else {
            coo_off[t] = (int)row.size();
            nnz[t] = (int)M.row.size();
            row.insert(row.end(), M.row.begin(), M.row.end());
            col.insert(col.end(), M.col.begin(), M.col.end());
            val.insert(val.end(), M.val.begin(), M.val.end());
        }
    }
    std::vector<int> perm(nc);
    std::iota(perm.begin(), perm.end(), 0);
    std::sort(perm.begin(), perm.end(), [&](int a, int b) { return effect[a] != effect[b] ? effect[a] < effect[b] : con[a] < con[b]; });
    bd.nsparse = nc - ndense;
    for (int s = 0; s < nc; ++s) {
        bool sp = coo_off[perm[s]] >= 0;
        if (sp != (s < bd.nsparse)) throw Error(ERR_STATE, "internal: sparse matrices do not sort before dense ones");
    }
    bd.all_dense = (bd.nsparse == 0);
    cudaStream_t st = c.stream;
    bd.h_perm = perm;
    bd.h_dense_off = dense_off;
    bd.con.upload(con, st);
    bd.formula.upload(formula, st);
    bd.effect.upload(effect, st);
    bd.perm.upload(perm, st);
    bd.coo_off.upload(coo_off, st);
    bd.nnz.upload(nnz, st);
    bd.dense_off.upload(dense_off, st);
    bd.row.upload(row, st);
    bd.col.upload(col, st);
    bd.val.upload(val, st);
    bd.dense.upload(dense, st);
    // element lists for sum_k y_k A_k (InputData::multi_plusToA order:
    // k ascending, entries of one matrix in input order)
    if (!bd.all_dense) {
        const long ne = (long)n * n;
        std::vector<int> cnt(ne + 1, 0);
        for (int t = 0; t < nc; ++t) {
            const BlockMat &M = P.A[cl[t]].at(l);
            if (M.dense) {
                for (long e = 0; e < ne; ++e) cnt[e + 1]++;
            } else {
                for (size_t q = 0; q < M.row.size(); ++q) {
                    int i = M.row[q], j = M.col[q];
                    cnt[i + (long)n * j + 1]++;
                    if (i != j) cnt[j + (long)n * i + 1]++;
                }
            }
        }
        for (long e = 0; e < ne; ++e) cnt[e + 1] += cnt[e];
        std::vector<int> el_con(cnt[ne]);
        std::vector<dd_t> el_val(cnt[ne]);
        std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
        for (int t = 0; t < nc; ++t) {
            const BlockMat &M = P.A[cl[t]].at(l);
            if (M.dense) {
                for (long e = 0; e < ne; ++e) {
                    el_con[fillp[e]] = cl[t];
                    el_val[fillp[e]++] = M.val[e];
                }
            } else {
                for (size_t q = 0; q < M.row.size(); ++q) {
                    int i = M.row[q], j = M.col[q];
                    long e1 = i + (long)n * j, e2 = j + (long)n * i;
                    el_con[fillp[e1]] = cl[t];
                    el_val[fillp[e1]++] = M.val[q];
                    if (i != j) {
                        el_con[fillp[e2]] = cl[t];
                        el_val[fillp[e2]++] = M.val[q];
                    }
                }
            }
        }
        bd.el_ptr.upload(cnt, st);
        bd.el_con.upload(el_con, st);
        bd.el_val.upload(el_val, st);
    }
    // C of this block
    auto it = P.C.find(l);
    bd.c_present = it != P.C.end();
    if (bd.c_present) {
        const BlockMat &M = it->second;
        bd.c_dense = M.dense;
        if (M.dense) {
            bd.c_dense_val.upload(M.val, st);
        } else {
            bd.c_row.upload(M.row, st);
            bd.c_col.upload(M.col, st);
            bd.c_val.upload(M.val, st);
            const long ne = (long)n * n;
            std::vector<int> cnt(ne + 1, 0);
            for (size_t q = 0; q < M.row.size(); ++q) {
                int i = M.row[q], j = M.col[q];
                cnt[i + (long)n * j + 1]++;
                if (i != j) cnt[j + (long)n * i + 1]++;
            }
            for (long e = 0; e < ne; ++e) cnt[e + 1] += cnt[e];
            std::vector<dd_t> ev(cnt[ne]);
            std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
            for (size_t q = 0; q < M.row.size(); ++q) {
                int i = M.row[q], j = M.col[q];
                ev[fillp[i + (long)n * j]++] = M.val[q];
                if (i != j) ev[fillp[j + (long)n * i]++] = M.val[q];
            }
            bd.c_el_ptr.upload(cnt, st);
            bd.c_el_val.upload(ev, st);
        }
    }
    // Schur owners
    bd.h_ownFG.clear();
    bd.h_ownF3.clear();
    std::vector<int> fg_index(nc, -1);
    for (int s = 0; s < nc; ++s) {
        int f = formula[perm[s]];
        if (f == F3) {
            bd.h_ownF3.push_back(s);
        } else {
            fg_index[s] = (int)bd.h_ownFG.size();
            bd.h_ownFG.push_back(s);
        }
    }
    // row lists of the sparse FG owners
    {
        std::vector<int> rl_off(bd.h_ownFG.size(), -1), rl_ptr, rl_src;
        std::vector<dd_t> rl_val;
        for (size_t r = 0; r < bd.h_ownFG.size(); ++r) {
            int t = perm[bd.h_ownFG[r]];
            const BlockMat &M = P.A[cl[t]].at(l);
            if (M.dense) continue;
            rl_off[r] = (int)rl_ptr.size();
            std::vector<std::vector<std::pair<int, dd_t>>> rows(n);
            for (size_t q = 0; q < M.row.size(); ++q) {
                if (dd_is_zero(M.val[q])) continue; // Raxpy returns when da == 0
                int i = M.row[q], j = M.col[q];
                rows[i].push_back({j, M.val[q]});
                if (i != j) rows[j].push_back({i, M.val[q]});
            }
            int base = (int)rl_src.size();
            for (int i = 0; i < n; ++i) {
                rl_ptr.push_back(base);
                for (auto &pr : rows[i]) {
                    rl_src.push_back(pr.first);
                    rl_val.push_back(pr.second);
                    ++base;
                }
            }
            rl_ptr.push_back(base);
        }
        bd.h_rl_off = rl_off;
        bd.rl_off.upload(rl_off, st);
        bd.rl_ptr.upload(rl_ptr, st);
        bd.rl_src.upload(rl_src, st);
        bd.rl_val.upload(rl_val, st);
    }
    // algorithmic dd-flops of this block's part of Make_bMat: per owner the
    // two n^3 products (F and G), 2 per term of the pair inner products,
    // and for calF3 3 per product term (two multiplies, one add) plus the
    // outer accumulation
    {
        double fl = 0;
        const double n3 = 2.0 * n * (double)n * n;
        std::vector<double> eff_s(nc);
        for (int q = 0; q < nc; ++q) eff_s[q] = effect[perm[q]];
        for (int q = 0; q < nc; ++q) {
            const int f = formula[perm[q]];
            const double ei = eff_s[q];
            if (f == F3) {
                double se = 0;
                for (int r = 0; r <= q; ++r) se += eff_s[r];
                fl += 3.0 * ei * se + 2.0 * se;
            } else {
                fl += (coo_off[perm[q]] >= 0 ? 2.0 * n * ei : n3) + n3;
                for (int r = 0; r <= q; ++r) {
                    const bool dense_partner = coo_off[perm[r]] < 0;
                    if (dense_partner) fl += 2.0 * n * n;
                    else fl += (f == F1 ? 2.0 * eff_s[r] : 2.0 * n * eff_s[r] + 2.0 * eff_s[r]);
                }
            }
        }
        c.schur_flops += fl;
    }
    bd.ownFG.upload(bd.h_ownFG, st);
    bd.ownF3.upload(bd.h_ownF3, st);
    bd.fg_index.upload(fg_index, st);
    bd.fg_dense_contig = !bd.h_ownFG.empty();
    for (size_t r = 0; r < bd.h_ownFG.size(); ++r) {
        int t = perm[bd.h_ownFG[r]];
        if (dense_off[t] < 0 || dense_off[t] != dense_off[perm[bd.h_ownFG[0]]] + (long)r * n * n) bd.fg_dense_contig = false;
    }
}

void upload_problem(Context &c, Problem &&p) {
    if (p.nSDP == 0) throw Error(ERR_ARG, "no SDP block");
    CK(cudaSetDevice(c.device));
    c.prob = std::move(p);
    const Problem &P = c.prob;
    c.m = P.m;
    c.nSDP = P.nSDP;
    c.nDim = P.nDim();
    c.sizes = P.sdpSize;
    c.off.assign(c.nSDP + 1, 0);
    for (int l = 0; l < c.nSDP; ++l) c.off[l + 1] = c.off[l] + (long)c.sizes[l] * c.sizes[l];
    c.space_len = c.off[c.nSDP];
    ++c.upload_gen;
    c.c_slot_host.clear();
    c.runs.clear();
    for (int l = 0; l < c.nSDP; ++l) {
        if (!c.runs.empty() && c.runs.back().n == c.sizes[l])
            ++c.runs.back().count;
        else
            c.runs.push_back({l, 1, c.sizes[l]});
    }
    // block objects (and their device buffers) are reused across uploads
    if ((int)c.blocks.size() > c.nSDP) c.blocks.resize(c.nSDP);
    while ((int)c.blocks.size() < c.nSDP) c.blocks.emplace_back(new BlockDev());
    c.schur_flops = 0;
    c.chol_flops = (double)c.m * c.m * c.m / 3.0;
    for (int l = 0; l < c.nSDP; ++l) build_block(c, P, l, *c.blocks[l]);
    std::vector<BlockView> views;
    for (auto &bd : c.blocks) views.push_back(bd->view());
    c.views.upload(views, c.stream);
    c.d_off.upload(c.off, c.stream);
    c.d_sizes.upload(c.sizes, c.stream);
    std::vector<int> ptr(c.m + 1, 0), bl, tt;
    for (int k = 0; k < c.m; ++k) {
        for (auto &kv : P.A[k]) {
            int l = kv.first;
            const auto &cl = P.cons[l];
            int t = (int)(std::lower_bound(cl.begin(), cl.end(), k) - cl.begin());
            bl.push_back(l);
            tt.push_back(t);
        }
        ptr[k + 1] = (int)bl.size();
    }
    c.inner_dense1 = c.nSDP == 1 && c.m > 0 && (int)bl.size() == c.m && c.blocks[0]->all_dense &&
                     (size_t)c.sizes[0] * c.sizes[0] * sizeof(dd_t) <= INNER_DENSE1_SMEM;
    c.cb_ptr.upload(ptr, c.stream);
    c.cb_block.upload(bl, c.stream);
    c.cb_t.upload(tt, c.stream);
    c.b.upload(P.b, c.stream);
    alloc_state(c);
    sparse_setup(c);
    if (c.sparse_active()) c.chol_flops = 2.0 * (double)c.sp->sched.exact_terms;
    CK(cudaStreamSynchronize(c.stream));
    c.adj_valid = false;
    c.has_init = false;
    c.have_problem = true;
}

void alloc_state(Context &c) {
    const size_t sl = (size_t)c.space_len;
    for (Space *s : {&c.X, &c.Z, &c.invCholX, &c.invCholZ, &c.invZ, &c.Dx, &c.Dz, &c.rzinv, &c.xrdzinv, &c.dualMat, &c.W1, &c.W2}) s->buf.alloc(sl);
    c.y.alloc(c.m);
    c.Dy.alloc(c.m);
    c.g.alloc(c.m);
    c.primalVec.alloc(c.m);
    c.B.alloc((size_t)c.m * c.m);
    size_t fg = 0;
    for (auto &bd : c.blocks) fg = std::max(fg, (size_t)bd->nFG() * bd->n * bd->n);
    c.Fbuf.alloc(std::max<size_t>(fg, 1));
    c.Gbuf.alloc(std::max<size_t>(fg, 1));
    // result slots: the per-block inner products (inner_space, inner_C) use
    // at most nSDP; the step-length eigenvalues of up to two spaces use 2
    // nSDP (per space: big blocks first, then the small ones) plus 2 nSDP
    // for the Lanczos launch's own outputs
    c.scal.alloc(std::max<size_t>(64, 4 * (size_t)c.nSDP + 8));
    c.red.alloc(4096);
    c.info.alloc(4);
    c.rdiag.alloc(256);
}

void space_to_host(Context &c, const Space &s, dd_t *out) {
    CK(cudaMemcpyAsync(out, s.buf.p, sizeof(dd_t) * c.space_len, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
}
void space_from_host(Context &c, Space &s, const dd_t *in) {
    CK(cudaMemcpyAsync(s.buf.p, in, sizeof(dd_t) * c.space_len, cudaMemcpyHostToDevice, c.stream));
}

} // namespace sddd
