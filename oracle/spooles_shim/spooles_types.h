#ifndef ORACLE_SPOOLES_TYPES_H
#define ORACLE_SPOOLES_TYPES_H
/* Opaque SPOOLES types and the prototypes the reference calls
 * (sdpa_chordal.cpp, sdpa_newton.cpp), implemented in spooles_shim.cpp. */
#include <stdio.h>
#include <time.h>
typedef struct _IV IV;
typedef struct _IVL IVL;
typedef struct _Graph Graph;
typedef struct _ETree ETree;
typedef struct _InpMtx InpMtx;
typedef struct _SymbFac SymbFac;
#define IVL_CHUNKED 1
#ifndef CLK_TCK
#define CLK_TCK CLOCKS_PER_SEC
#endif
void IV_free(IV *);
int *IV_entries(IV *);
IVL *IVL_new(void);
void IVL_init1(IVL *, int, int);
void IVL_setList(IVL *, int, int, int *);
int IVL_tsize(IVL *);
int IVL_nlist(IVL *);
void IVL_listAndSize(IVL *, int, int *, int **);
void IVL_free(IVL *);
int IVL_writeForHumanEye(IVL *, FILE *);
Graph *Graph_new(void);
void Graph_init2(Graph *, int, int, int, int, int, int, IVL *, IV *, IVL *);
void Graph_free(Graph *);
void ETree_free(ETree *);
IV *ETree_newToOldVtxPerm(ETree *);
IVL *SymbFac_initFromGraph(ETree *, Graph *);
ETree *orderViaMMD(Graph *, int, int, FILE *);
ETree *orderViaND(Graph *, int, int, int, FILE *);
ETree *orderViaMS(Graph *, int, int, int, FILE *);
ETree *orderViaBestOfNDandMS(Graph *, int, int, int, int, int, FILE *);
#endif
