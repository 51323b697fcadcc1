// Working stand-ins for the SPOOLES entry points the reference calls
// (sdpa_chordal.cpp, sdpa_newton.cpp:225-340).  Test infrastructure: oracle
// build only.
//
// The SPOOLES library itself is not part of the reference's sources, so the
// reference's sparse-Schur path runs here with this ordering in its place:
// an exact minimum-degree elimination (the live vertex of least current
// degree, ties to the smallest index; its live neighbours become a clique),
// written independently of the product's ordering (sorted neighbour lists
// and a linear scan here, bit rows and a heap there), and the symbolic
// factor of that ordering, one front per vertex: front l lists the l-th
// eliminated vertex, then its neighbours at elimination in elimination
// order (old numbers).  That is the list layout
// Newton::initialize_sparse_bMat and Chordal::countNonZero walk.
//
// Every ordering routine the reference may call (orderViaMMD / ND / MS /
// BestOfNDandMS) returns this ordering; with OrderOnlyByMDO
// (sdpa_chordal.cpp:24) only orderViaMMD is reached.
#include <algorithm>
#include <cstdio>
#include <vector>
extern "C" {
#include "spooles_types.h"
}

struct _IV {
    std::vector<int> v;
};
struct _IVL {
    std::vector<std::vector<int>> lists;
};
struct _Graph {
    int nvtx = 0;
    IVL *adj = nullptr; // owned, as SPOOLES's Graph owns its adjacency
};
struct _ETree {
    std::vector<int> newToOld;
    std::vector<std::vector<int>> fronts; // old numbers
};

namespace {

// Minimum-degree elimination of the graph (self entries ignored).
_ETree *min_degree(const Graph *g) {
    const int n = g->nvtx;
    std::vector<std::vector<int>> adj(n);
    for (int i = 0; i < n; ++i) {
        for (int j : g->adj->lists[i])
            if (j != i) {
                adj[i].push_back(j);
                adj[j].push_back(i);
            }
    }
    for (auto &a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    std::vector<char> alive(n, 1);
    std::vector<std::vector<int>> nbrs(n);
    _ETree *t = new _ETree();
    std::vector<int> merged;
    for (int step = 0; step < n; ++step) {
        int v = -1;
        for (int u = 0; u < n; ++u)
            if (alive[u] && (v < 0 || adj[u].size() < adj[v].size())) v = u;
        t->newToOld.push_back(v);
        alive[v] = 0;
        nbrs[v] = adj[v];
        for (int u : adj[v]) {
            merged.clear();
            std::set_union(adj[u].begin(), adj[u].end(), adj[v].begin(), adj[v].end(), std::back_inserter(merged));
            merged.erase(std::remove_if(merged.begin(), merged.end(), [&](int w) { return w == u || w == v; }), merged.end());
            adj[u].swap(merged);
        }
        adj[v].clear();
    }
    std::vector<int> pos(n);
    for (int i = 0; i < n; ++i) pos[t->newToOld[i]] = i;
    t->fronts.resize(n);
    for (int l = 0; l < n; ++l) {
        const int v = t->newToOld[l];
        std::vector<int> f = nbrs[v];
        std::sort(f.begin(), f.end(), [&](int a, int b) { return pos[a] < pos[b]; });
        t->fronts[l].push_back(v);
        t->fronts[l].insert(t->fronts[l].end(), f.begin(), f.end());
    }
    return t;
}

} // namespace

extern "C" {
void IV_free(IV *iv) { delete iv; }
int *IV_entries(IV *iv) { return iv->v.data(); }
IVL *IVL_new(void) { return new _IVL(); }
void IVL_init1(IVL *ivl, int, int n) { ivl->lists.assign(n, {}); }
void IVL_setList(IVL *ivl, int i, int size, int *ivec) { ivl->lists[i].assign(ivec, ivec + size); }
int IVL_tsize(IVL *ivl) {
    long s = 0;
    for (auto &l : ivl->lists) s += (long)l.size();
    return (int)s;
}
int IVL_nlist(IVL *ivl) { return (int)ivl->lists.size(); }
void IVL_listAndSize(IVL *ivl, int i, int *size, int **ptr) {
    *size = (int)ivl->lists[i].size();
    *ptr = ivl->lists[i].data();
}
void IVL_free(IVL *ivl) { delete ivl; }
int IVL_writeForHumanEye(IVL *ivl, FILE *fp) {
    for (size_t i = 0; i < ivl->lists.size(); ++i) {
        std::fprintf(fp, "%zu :", i);
        for (int x : ivl->lists[i]) std::fprintf(fp, " %d", x);
        std::fprintf(fp, "\n");
    }
    return 1;
}
Graph *Graph_new(void) { return new _Graph(); }
void Graph_init2(Graph *g, int, int nvtx, int, int, int, int, IVL *adj, IV *, IVL *) {
    g->nvtx = nvtx;
    g->adj = adj;
}
void Graph_free(Graph *g) {
    if (!g) return;
    delete g->adj;
    delete g;
}
void ETree_free(ETree *t) { delete t; }
IV *ETree_newToOldVtxPerm(ETree *t) {
    IV *iv = new _IV();
    iv->v = t->newToOld;
    return iv;
}
IVL *SymbFac_initFromGraph(ETree *t, Graph *) {
    IVL *ivl = new _IVL();
    ivl->lists = t->fronts;
    return ivl;
}
ETree *orderViaMMD(Graph *g, int, int, FILE *) { return min_degree(g); }
ETree *orderViaND(Graph *g, int, int, int, FILE *) { return min_degree(g); }
ETree *orderViaMS(Graph *g, int, int, int, FILE *) { return min_degree(g); }
ETree *orderViaBestOfNDandMS(Graph *g, int, int, int, int, int, FILE *) { return min_degree(g); }
}
