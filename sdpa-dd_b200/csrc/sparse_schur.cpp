// Host side of the sparse Schur complement: the reference's choice between
// the dense and the sparse form of B, the minimum-degree ordering, the
// symbolic factor, and the tile schedule of the device factor and solves.
#include "sparse_schur.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <queue>
#include <string>

#include "common.cuh"

namespace sddd {

namespace {

// Rows of an m x m bit matrix.
struct BitRows {
    int m = 0, W = 0;
    std::vector<uint64_t> w;
    explicit BitRows(int m_) : m(m_), W((m_ + 63) / 64), w((size_t)m_ * ((m_ + 63) / 64), 0) {}
    uint64_t *row(int i) { return w.data() + (size_t)i * W; }
    const uint64_t *row(int i) const { return w.data() + (size_t)i * W; }
    void set(int i, int j) { row(i)[j >> 6] |= 1ull << (j & 63); }
    void clear(int i, int j) { row(i)[j >> 6] &= ~(1ull << (j & 63)); }
    long count(int i) const {
        long n = 0;
        const uint64_t *r = row(i);
        for (int k = 0; k < W; ++k) n += __builtin_popcountll(r[k]);
        return n;
    }
    template <class F>
    void each(int i, F f) const {
        const uint64_t *r = row(i);
        for (int k = 0; k < W; ++k)
            for (uint64_t x = r[k]; x; x &= x - 1) f(k * 64 + __builtin_ctzll(x));
    }
};

// Minimum degree on a bit adjacency without self entries (G is consumed).
std::vector<int> min_degree_bits(BitRows &G, std::vector<std::vector<int>> *structs) {
    const int m = G.m;
    std::vector<int> deg(m), order;
    std::vector<char> alive(m, 1);
    order.reserve(m);
    if (structs) structs->assign(m, {});
    using Key = std::pair<int, int>; // (degree, vertex): the smallest pops first
    std::priority_queue<Key, std::vector<Key>, std::greater<Key>> heap;
    for (int v = 0; v < m; ++v) {
        deg[v] = (int)G.count(v);
        heap.push({deg[v], v});
    }
    std::vector<int> nb;
    while ((int)order.size() < m) {
        const Key k = heap.top();
        heap.pop();
        const int v = k.second;
        if (!alive[v] || k.first != deg[v]) continue; // a stale entry
        order.push_back(v);
        alive[v] = 0;
        nb.clear();
        G.each(v, [&](int u) { nb.push_back(u); });
        if (structs) (*structs)[v] = nb;
        if (nb.empty()) continue;
        const uint64_t *rv = G.row(v);
        const int w0 = nb.front() >> 6, w1 = nb.back() >> 6;
        for (int u : nb) {
            uint64_t *ru = G.row(u);
            int d = deg[u];
            // v leaves u's neighbourhood
            ru[v >> 6] &= ~(1ull << (v & 63));
            --d;
            // u joins the clique of v's live neighbours
            for (int q = w0; q <= w1; ++q) {
                uint64_t nw = ru[q] | rv[q];
                if (q == (u >> 6)) nw &= ~(1ull << (u & 63));
                d += __builtin_popcountll(nw) - __builtin_popcountll(ru[q]);
                ru[q] = nw;
            }
            deg[u] = d;
            heap.push({d, u});
        }
    }
    return order;
}

SparseStructure structure_of(int m, const std::vector<int> &order, const std::vector<std::vector<int>> &structs) {
    std::vector<int> rev(m);
    for (int i = 0; i < m; ++i) rev[order[i]] = i;
    SparseStructure s;
    s.m = m;
    s.rowptr.assign(m + 1, 0);
    for (int b = 0; b < m; ++b) s.rowptr[b + 1] = s.rowptr[b] + 1 + (int)structs[order[b]].size();
    s.col.resize(s.rowptr[m]);
    for (int b = 0; b < m; ++b) {
        int *c = s.col.data() + s.rowptr[b];
        c[0] = b;
        int k = 1;
        for (int u : structs[order[b]]) c[k++] = rev[u];
        std::sort(c + 1, c + k);
    }
    return s;
}

} // namespace

std::vector<int> min_degree_order(int m, const std::vector<std::vector<int>> &adj, std::vector<std::vector<int>> *structs) {
    BitRows G(m);
    for (int i = 0; i < m; ++i)
        for (int j : adj[i])
            if (j != i) {
                G.set(i, j);
                G.set(j, i);
            }
    return min_degree_bits(G, structs);
}

SparsePlan plan_schur(const Problem &p, int mode) {
    SparsePlan r;
    const int m = p.m;
    if (mode == SCHUR_DENSE) {
        r.dense_reason = "the dense form was requested";
        return r;
    }
    // Chordal::initialize (sdpa_chordal.cpp:42-58)
    int m_thr = 100, b_thr = 5;
    double agg = 0.25, ext = 0.4;
    if (mode == SCHUR_SPARSE) {
        m_thr = 0;
        b_thr = 0;
        agg = 2.0;
        ext = 2.0;
    }
    // Chordal::ordering_bMat (sdpa_chordal.cpp:348-438); the LP entries are
    // blocks of their own here as there (nBlock2 = SDP + LP blocks)
    if (m <= m_thr || p.nSDP <= b_thr) {
        r.dense_reason = m <= m_thr ? "m is at most 100" : "there are at most 5 blocks";
        return r;
    }
    for (int l = 0; l < p.nSDP; ++l)
        if ((double)p.cons[l].size() > m * std::sqrt(agg)) {
            r.dense_reason = "a block touches more than half of the constraints";
            return r;
        }
    // aggregate pattern (Chordal::makeGraph, sdpa_chordal.cpp:141-240): i
    // and j adjacent when some block holds both; i is its own neighbour
    BitRows G(m);
    for (int l = 0; l < p.nSDP; ++l) {
        const auto &cl = p.cons[l];
        std::vector<uint64_t> bits(G.W, 0);
        for (int k : cl) bits[k >> 6] |= 1ull << (k & 63);
        int w0 = G.W, w1 = -1;
        for (int q = 0; q < G.W; ++q)
            if (bits[q]) {
                w0 = std::min(w0, q);
                w1 = q;
            }
        for (int k : cl) {
            uint64_t *rk = G.row(k);
            for (int q = w0; q <= w1; ++q) rk[q] |= bits[q];
        }
    }
    for (int i = 0; i < m; ++i) r.aggregate += G.count(i);
    if ((double)r.aggregate > agg * m * m) {
        r.dense_reason = "the aggregate pattern is denser than the threshold";
        return r;
    }
    for (int i = 0; i < m; ++i) G.clear(i, i);
    std::vector<std::vector<int>> structs;
    std::vector<int> order = min_degree_bits(G, &structs);
    SparseStructure s = structure_of(m, order, structs);
    r.extended = 2 * s.nnz() - m;
    if ((double)r.extended > ext * m * m) {
        r.dense_reason = "the factor's fill is above the threshold";
        return r;
    }
    r.sparse = true;
    r.order = std::move(order);
    r.s = std::move(s);
    return r;
}

std::string check_structure(const SparseStructure &s) {
    const int m = s.m;
    if ((int)s.rowptr.size() != m + 1 || s.rowptr[0] != 0) return "rowptr must hold m + 1 offsets from 0";
    for (int b = 0; b < m; ++b) {
        const int p0 = s.rowptr[b], p1 = s.rowptr[b + 1];
        if (p1 <= p0 || p1 > (long)s.col.size()) return "row " + std::to_string(b) + " has no diagonal entry or runs past the column list";
        if (s.col[p0] != b) return "row " + std::to_string(b) + " does not start with its diagonal";
        for (int q = p0 + 1; q < p1; ++q)
            if (s.col[q] <= s.col[q - 1] || s.col[q] >= m) return "row " + std::to_string(b) + " is not strictly ascending within 0..m-1";
    }
    if ((long)s.col.size() != s.nnz()) return "the column list is longer than rowptr[m]";
    // closure: a, c in struct(b) with a < c  =>  c in struct(a)
    for (int b = 0; b < m; ++b) {
        const int p0 = s.rowptr[b] + 1, p1 = s.rowptr[b + 1];
        for (int q = p0; q < p1; ++q) {
            const int a = s.col[q];
            const int *r0 = s.col.data() + s.rowptr[a], *r1 = s.col.data() + s.rowptr[a + 1];
            const int *it = r0;
            for (int t = q + 1; t < p1; ++t) {
                it = std::lower_bound(it, r1, s.col[t]);
                if (it == r1 || *it != s.col[t])
                    return "entry (" + std::to_string(s.col[t]) + ", " + std::to_string(a) + ") is filled by row " + std::to_string(b) + " but missing";
            }
        }
    }
    return "";
}

TileSchedule make_tile_schedule(const SparseStructure &s) {
    TileSchedule t;
    const int m = s.m, nb = (m + SP_T - 1) / SP_T;
    t.m = m;
    t.nblk = nb;
    t.tile_of.assign((size_t)nb * nb, -1);
    auto tile = [&](int I, int J) -> int {
        int &id = t.tile_of[I + (size_t)nb * J];
        if (id < 0) {
            id = t.ntiles++;
            t.tI.push_back(I);
            t.tJ.push_back(J);
            t.mask.resize((size_t)t.ntiles * SP_T, 0);
        }
        return id;
    };
    // Row b of the factor is column b of the lower triangle: entry (a, b).
    for (int b = 0; b < m; ++b) {
        const int J = b / SP_T;
        for (int q = s.rowptr[b]; q < s.rowptr[b + 1]; ++q) {
            const int a = s.col[q];
            const int id = tile(a / SP_T, J);
            t.mask[(size_t)id * SP_T + (b % SP_T)] |= 1ull << (a % SP_T);
        }
        const long len = s.rowptr[b + 1] - s.rowptr[b] - 1;
        t.exact_terms += len * (len + 1) / 2;
    }
    // column and row lists
    t.col_ptr.assign(nb + 1, 0);
    t.row_ptr.assign(nb + 1, 0);
    for (int J = 0; J < nb; ++J)
        for (int I = J + 1; I < nb; ++I)
            if (t.tile_of[I + (size_t)nb * J] >= 0) {
                t.col_tiles.push_back(t.tile_of[I + (size_t)nb * J]);
                t.col_ptr[J + 1]++;
            }
    for (int J = 0; J < nb; ++J) t.col_ptr[J + 1] += t.col_ptr[J];
    for (int I = 0; I < nb; ++I) {
        for (int J = 0; J < I; ++J)
            if (t.tile_of[I + (size_t)nb * J] >= 0) t.row_tiles.push_back(t.tile_of[I + (size_t)nb * J]);
        t.row_ptr[I + 1] = (int)t.row_tiles.size();
    }
    // trailing updates: target (I, K) of panel J when one column b of J has
    // entries in row blocks I and K (both below J)
    t.upd_ptr.assign(nb + 1, 0);
    for (int J = 0; J < nb; ++J) {
        const int c0 = J * SP_T, c1 = std::min(m, c0 + SP_T);
        std::vector<int> blocks;
        std::vector<char> seen((size_t)nb * nb, 0); // (I, K) pairs already listed, I >= K
        std::vector<std::pair<int, int>> tg;
        for (int b = c0; b < c1; ++b) {
            blocks.clear();
            for (int q = s.rowptr[b] + 1; q < s.rowptr[b + 1]; ++q) {
                const int B = s.col[q] / SP_T;
                if (B > J && (blocks.empty() || blocks.back() != B)) blocks.push_back(B);
            }
            for (size_t x = 0; x < blocks.size(); ++x)
                for (size_t y = 0; y <= x; ++y) {
                    const int I = blocks[x], K = blocks[y];
                    char &sn = seen[I + (size_t)nb * K];
                    if (!sn) {
                        sn = 1;
                        tg.push_back({K, I});
                    }
                }
        }
        std::sort(tg.begin(), tg.end());
        for (auto &kv : tg) {
            const int K = kv.first, I = kv.second;
            const int target = t.tile_of[I + (size_t)nb * K];
            const int sI = t.tile_of[I + (size_t)nb * J], sK = t.tile_of[K + (size_t)nb * J];
            if (target < 0 || sI < 0 || sK < 0) throw Error(ERR_ARG, "sparse Schur: the factor's structure is not closed under elimination");
            t.upd.push_back(target);
            t.upd.push_back(sI);
            t.upd.push_back(sK);
        }
        t.upd_ptr[J + 1] = t.upd_ptr[J] + (int)tg.size();
        t.update_terms += (long)tg.size() * SP_T * SP_T * SP_T;
    }
    return t;
}

} // namespace sddd
