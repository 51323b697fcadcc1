// Abort-only stand-ins for the SPOOLES entry points the reference names.
//
// Oracle build only.  The reference's sparse-Schur path (sdpa_chordal.cpp,
// the *_sparse_* functions of sdpa_newton.cpp) needs SPOOLES, whose sources
// are not available.  Chordal::ordering_bMat returns the dense path before
// any SPOOLES call when m <= 100 or nBlock <= 5 (sdpa_chordal.cpp:349-352),
// which covers every workload this repository exercises; reaching a stub
// means the input needs the sparse path and the oracle stops loudly.
#include <cstdio>
#include <cstdlib>
extern "C" {
#include "spooles_types.h"
}

[[noreturn]] static void spooles_missing(const char *name) {
    std::fprintf(stderr, "oracle: SPOOLES entry point %s reached; sparse Schur path is not available\n", name);
    std::abort();
}

extern "C" {
void IV_free(IV *) { spooles_missing("IV_free"); }
int *IV_entries(IV *) { spooles_missing("IV_entries"); }
IVL *IVL_new(void) { spooles_missing("IVL_new"); }
void IVL_init1(IVL *, int, int) { spooles_missing("IVL_init1"); }
void IVL_setList(IVL *, int, int, int *) { spooles_missing("IVL_setList"); }
int IVL_tsize(IVL *) { spooles_missing("IVL_tsize"); }
int IVL_nlist(IVL *) { spooles_missing("IVL_nlist"); }
void IVL_listAndSize(IVL *, int, int *, int **) { spooles_missing("IVL_listAndSize"); }
void IVL_free(IVL *) { spooles_missing("IVL_free"); }
int IVL_writeForHumanEye(IVL *, FILE *) { spooles_missing("IVL_writeForHumanEye"); }
Graph *Graph_new(void) { spooles_missing("Graph_new"); }
void Graph_init2(Graph *, int, int, int, int, int, int, IVL *, IV *, IVL *) { spooles_missing("Graph_init2"); }
void Graph_free(Graph *) { spooles_missing("Graph_free"); }
void ETree_free(ETree *) { spooles_missing("ETree_free"); }
IV *ETree_newToOldVtxPerm(ETree *) { spooles_missing("ETree_newToOldVtxPerm"); }
IVL *SymbFac_initFromGraph(ETree *, Graph *) { spooles_missing("SymbFac_initFromGraph"); }
ETree *orderViaMMD(Graph *, int, int, FILE *) { spooles_missing("orderViaMMD"); }
ETree *orderViaND(Graph *, int, int, int, FILE *) { spooles_missing("orderViaND"); }
ETree *orderViaMS(Graph *, int, int, int, FILE *) { spooles_missing("orderViaMS"); }
ETree *orderViaBestOfNDandMS(Graph *, int, int, int, int, int, FILE *) { spooles_missing("orderViaBestOfNDandMS"); }
}
