// C entry points into the reference build (test infrastructure only).
//
// Compiled against the reference sources by oracle/Makefile into
// oracle/_ref/libsdpadd_ref.so.  Nothing here is product code: tests load
// this library through ctypes to obtain golden values from the reference's
// own arithmetic (QD 2.3.23), its MPLAPACK kernels, and its Newton /
// step-length / update code, one piece at a time.
//
// dd values cross this boundary as interleaved (hi, lo) doubles, the byte
// layout of QD's dd_real.  Block spaces are the SDP blocks in order, each
// n_l x n_l column-major, followed by the LP entries.
#include <sdpa_io.h>
#include <mpblas_dd.h>
#include <mplapack_dd.h>

#include <qd/qd_real.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

using namespace sdpa;

namespace {

inline dd_real ld(const double *p) { return dd_real(p[0], p[1]); }
inline void st(double *p, const dd_real &v) {
    p[0] = v.x[0];
    p[1] = v.x[1];
}

size_t space_len(DenseLinearSpace &s) {
    size_t n = 0;
    for (int l = 0; l < s.SDP_nBlock; ++l) n += (size_t)s.SDP_block[l].nRow * s.SDP_block[l].nCol;
    return n + (size_t)s.LP_nBlock;
}
void space_get(DenseLinearSpace &s, double *out) {
    size_t k = 0;
    for (int l = 0; l < s.SDP_nBlock; ++l) {
        size_t len = (size_t)s.SDP_block[l].nRow * s.SDP_block[l].nCol;
        for (size_t i = 0; i < len; ++i, ++k) st(out + 2 * k, s.SDP_block[l].de_ele[i]);
    }
    for (int l = 0; l < s.LP_nBlock; ++l, ++k) st(out + 2 * k, s.LP_block[l]);
}
void space_set(DenseLinearSpace &s, const double *in) {
    size_t k = 0;
    for (int l = 0; l < s.SDP_nBlock; ++l) {
        size_t len = (size_t)s.SDP_block[l].nRow * s.SDP_block[l].nCol;
        for (size_t i = 0; i < len; ++i, ++k) s.SDP_block[l].de_ele[i] = ld(in + 2 * k);
    }
    for (int l = 0; l < s.LP_nBlock; ++l, ++k) s.LP_block[l] = ld(in + 2 * k);
}
void vec_get(Vector &v, double *out) {
    for (int i = 0; i < v.nDim; ++i) st(out + 2 * i, v.ele[i]);
}
void vec_set(Vector &v, const double *in) {
    for (int i = 0; i < v.nDim; ++i) v.ele[i] = ld(in + 2 * i);
}

// Everything pinpal (sdpa_main.cpp:43-292) sets up before its main loop,
// kept alive so the loop body can be driven one piece at a time.
struct RefSolver {
    ComputeTime com;
    Parameter param;
    int m = 0, nBlock = 0, SDP_nBlock = 0, SOCP_nBlock = 0, LP_nBlock = 0;
    std::vector<int> blockStruct, blockType, blockNumber, SDP_blockStruct, SOCP_blockStruct;
    InputData inputData;
    Newton *newton = nullptr;
    Solutions currentPt;
    WorkVariables work;
    Residuals *initRes = nullptr;
    Residuals currentRes;
    StepLength alpha;
    DirectionParameter beta;
    Switch reduction;
    AverageComplementarity mu;
    RatioInitResCurrentRes theta;
    SolveInfo solveInfo;
    Phase phase;
    int pIteration = 0;
    // captured intermediates of the last pass
    DenseMatrix bCaptured;
    Vector gPred;
    DenseLinearSpace dxPred, dzPred;
    Vector dyPred;
    dd_real alphaPredP, alphaPredD, betaPred, betaCorr, minEigX, minEigZ;
    dd_real muAtStep, thetaPAtStep, thetaDAtStep;
    dd_real objPAtStep, objDAtStep;
    int phaseAtStep = 0;
    // false: ref_step runs the stock loop body only (no copies of B, g and
    // the predictor direction, no extra eigenvalue calls), for timing
    bool capture = true;
};

} // namespace

extern "C" {

// ---------------------------------------------------------------- arithmetic
int ref_dd_read(const char *s, double *out) {
    dd_real a;
    int rc = a.read(s, a);
    st(out, a);
    return rc;
}

// op: 0 a+b, 1 a+=b, 2 a-b, 3 a-=b, 4 a*b, 5 a*=b, 6 a/b, 7 sqrt(a),
//     8 a*double(b.hi), 9 a+double(b.hi), 10 a-double(b.hi),
//     11 double(a.hi)-b, 12 a/double(b.hi), 13 double(a.hi)/b, 14 -a,
//     15 abs(a), 16 sqr(a), 17 double(a.hi)+double(b.hi) (exact sum)
void ref_dd_op(int op, long n, const double *a, const double *b, double *out) {
    for (long i = 0; i < n; ++i) {
        dd_real x = ld(a + 2 * i), y = ld(b + 2 * i), r;
        switch (op) {
        case 0: r = x + y; break;
        case 1: r = x; r += y; break;
        case 2: r = x - y; break;
        case 3: r = x; r -= y; break;
        case 4: r = x * y; break;
        case 5: r = x; r *= y; break;
        case 6: r = x / y; break;
        case 7: r = sqrt(x); break;
        case 8: r = x * y.x[0]; break;
        case 9: r = x + y.x[0]; break;
        case 10: r = x - y.x[0]; break;
        case 11: r = x.x[0] - y; break;
        case 12: r = x / y.x[0]; break;
        case 13: r = x.x[0] / y; break;
        case 14: r = -x; break;
        case 15: r = abs(x); break;
        case 16: r = sqr(x); break;
        case 17: r = dd_real::add(x.x[0], y.x[0]); break;
        default: r = 0.0; break;
        }
        st(out + 2 * i, r);
    }
}

// npwr / ^ : used by the decimal reader for 10^e
void ref_dd_npwr(const double *a, int n, double *out) { st(out, npwr(ld(a), n)); }

// QD's decimal formatting (dd_real::to_string with scientific flags), as
// printed by the reference for the 32-digit objective lines.
int ref_dd_to_string(const double *a, int precision, char *buf, int buflen) {
    std::string s = ld(a).to_string(precision, 0, std::ios_base::fmtflags(0));
    if ((int)s.size() + 1 > buflen) return -1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)s.size();
}

// ---------------------------------------------------------- MPLAPACK kernels
// All matrices are interleaved dd, column-major, leading dimensions in dd
// elements.  Scalars point to one (hi, lo) pair.
void ref_Rgemm(const char *ta, const char *tb, long m, long n, long k, const double *alpha, double *A, long lda, double *B, long ldb, const double *beta, double *C, long ldc) {
    Rgemm(ta, tb, m, n, k, ld(alpha), (dd_real *)A, lda, (dd_real *)B, ldb, ld(beta), (dd_real *)C, ldc);
}
void ref_Rsyrk(const char *uplo, const char *trans, long n, long k, const double *alpha, double *A, long lda, const double *beta, double *C, long ldc) {
    Rsyrk(uplo, trans, n, k, ld(alpha), (dd_real *)A, lda, ld(beta), (dd_real *)C, ldc);
}
void ref_Rtrsm(const char *side, const char *uplo, const char *ta, const char *diag, long m, long n, const double *alpha, double *A, long lda, double *B, long ldb) {
    Rtrsm(side, uplo, ta, diag, m, n, ld(alpha), (dd_real *)A, lda, (dd_real *)B, ldb);
}
void ref_Rtrmm(const char *side, const char *uplo, const char *ta, const char *diag, long m, long n, const double *alpha, double *A, long lda, double *B, long ldb) {
    Rtrmm(side, uplo, ta, diag, m, n, ld(alpha), (dd_real *)A, lda, (dd_real *)B, ldb);
}
void ref_Rtrsv(const char *uplo, const char *trans, const char *diag, long n, double *A, long lda, double *x, long incx) {
    Rtrsv(uplo, trans, diag, n, (dd_real *)A, lda, (dd_real *)x, incx);
}
void ref_Rtrmv(const char *uplo, const char *trans, const char *diag, long n, double *A, long lda, double *x, long incx) {
    Rtrmv(uplo, trans, diag, n, (dd_real *)A, lda, (dd_real *)x, incx);
}
void ref_Rgemv(const char *trans, long m, long n, const double *alpha, double *A, long lda, double *x, long incx, const double *beta, double *y, long incy) {
    Rgemv(trans, m, n, ld(alpha), (dd_real *)A, lda, (dd_real *)x, incx, ld(beta), (dd_real *)y, incy);
}
void ref_Rdot(long n, double *x, long incx, double *y, long incy, double *out) { st(out, Rdot(n, (dd_real *)x, incx, (dd_real *)y, incy)); }
long ref_Rpotrf(const char *uplo, long n, double *A, long lda) {
    mplapackint info = 0;
    Rpotrf(uplo, n, (dd_real *)A, lda, info);
    return (long)info;
}
// Lal::getCholesky(SparseMatrix&, int*) (sdpa_linear.cpp:353-395) on a
// matrix in the sparse_bMat layout: row b holds column_index[diagonalIndex[b]
// .. diagonalIndex[b+1]) (b first, ascending); vals[nnz] factored in place.
static void sparse_from(SparseMatrix &A, int m, const int *diagonalIndex, const int *column_index, const double *vals) {
    const int nnz = diagonalIndex[m];
    A.initialize(m, m, SparseMatrix::SPARSE, nnz);
    for (int b = 0; b < m; ++b)
        for (int q = diagonalIndex[b]; q < diagonalIndex[b + 1]; ++q) {
            A.row_index[q] = b;
            A.column_index[q] = column_index[q];
            A.sp_ele[q] = ld(vals + 2 * q);
        }
    A.NonZeroCount = nnz;
}
void ref_sparse_getCholesky(int m, const int *diagonalIndex, const int *column_index, double *vals) {
    SparseMatrix A;
    sparse_from(A, m, diagonalIndex, column_index, vals);
    std::vector<int> di(diagonalIndex, diagonalIndex + m + 1);
    Lal::getCholesky(A, di.data());
    for (int q = 0; q < diagonalIndex[m]; ++q) st(vals + 2 * q, A.sp_ele[q]);
}
// Lal::solveSystems(Vector&, SparseMatrix&, Vector&) (sdpa_linear.cpp:
// 654-810): x <- (L L^T)^-1 x for a factor from ref_sparse_getCholesky.
void ref_sparse_solveSystems(int m, const int *diagonalIndex, const int *column_index, const double *vals, double *x) {
    SparseMatrix A;
    sparse_from(A, m, diagonalIndex, column_index, vals);
    Vector b(m), y(m);
    for (int i = 0; i < m; ++i) b.ele[i] = ld(x + 2 * i);
    Lal::solveSystems(y, A, b);
    for (int i = 0; i < m; ++i) st(x + 2 * i, y.ele[i]);
}
long ref_Rsteqr(const char *compz, long n, double *d, double *e, double *Z, long ldz, double *work) {
    mplapackint info = 0;
    Rsteqr(compz, n, (dd_real *)d, (dd_real *)e, (dd_real *)Z, ldz, (dd_real *)work, info);
    return (long)info;
}
long ref_Rsyev(const char *jobz, const char *uplo, long n, double *A, long lda, double *w, double *work, long lwork) {
    mplapackint info = 0;
    Rsyev(jobz, uplo, n, (dd_real *)A, lda, (dd_real *)w, (dd_real *)work, lwork, info);
    return (long)info;
}
void ref_Rlamch(const char *c, double *out) { st(out, Rlamch_dd(c)); }

// ------------------------------------------------------------ SDPA level
// Lanczos minimum eigenvalue of L X L^T for one dense block
// (Lal::getMinEigen, sdpa_linear.cpp:27-122).
void ref_lanczos_min_eig(long n, double *L, double *X, double *out) {
    int nn = (int)n;
    // default-construct first: the sized constructors read members that
    // only the default constructor initialises (sdpa_struct.cpp:623-642)
    DenseMatrix lMat, xMat, Q;
    lMat.initialize(nn, nn, DenseMatrix::DENSE);
    xMat.initialize(nn, nn, DenseMatrix::DENSE);
    Q.initialize(nn, nn, DenseMatrix::DENSE);
    for (long i = 0; i < n * n; ++i) {
        lMat.de_ele[i] = ld(L + 2 * i);
        xMat.de_ele[i] = ld(X + 2 * i);
    }
    Vector o, b, r, q, qold, w, tmp, d1, d2, wv;
    for (Vector *v : {&o, &b, &r, &q, &qold, &w, &tmp, &d1, &d2}) v->initialize(nn);
    wv.initialize(std::max(1, 3 * nn - 1));
    st(out, Lal::getMinEigen(lMat, xMat, Q, o, b, r, q, qold, w, tmp, d1, d2, wv));
}

// B of the last Make_bMat as a dense m x m matrix in the constraints' own
// numbering (the sparse form's entries placed through the ordering, both
// triangles).
static void capture_B(RefSolver &s) {
    Newton &nt = *s.newton;
    if (nt.bMat_type == Newton::DENSE) {
        s.bCaptured.copyFrom(nt.bMat);
        return;
    }
    const int m = s.m;
    s.bCaptured.initialize(m, m, DenseMatrix::DENSE);
    s.bCaptured.setZero();
    for (int k = 0; k < nt.sparse_bMat.NonZeroCount; ++k) {
        const int i = nt.ordering[nt.sparse_bMat.row_index[k]], j = nt.ordering[nt.sparse_bMat.column_index[k]];
        s.bCaptured.de_ele[i + (long)m * j] = nt.sparse_bMat.sp_ele[k];
        s.bCaptured.de_ele[j + (long)m * i] = nt.sparse_bMat.sp_ele[k];
    }
}

// Opens a problem exactly as pinpal does before its main loop.
// paramFile may be NULL (defaults).  schurMode 0 keeps the reference's
// thresholds of Chordal::initialize (sdpa_chordal.cpp:42-45); 1 and 2 set
// its "DENSE computation for debugging" and "SPARSE computation for
// debugging" values (sdpa_chordal.cpp:47-58).  Returns NULL on failure.
void *ref_open_mode(const char *dataFile, const char *paramFile, double kappa, int schurMode) {
    FILE *fp = fopen(dataFile, "r");
    if (!fp) return nullptr;
    RefSolver *s = new RefSolver();
    s->param.setDefaultParameter(Parameter::PARAMETER_DEFAULT);
    if (paramFile) {
        FILE *fpp = fopen(paramFile, "r");
        if (!fpp) {
            fclose(fp);
            delete s;
            return nullptr;
        }
        s->param.readFile(fpp);
        fclose(fpp);
    }
    FILE *devnull = fopen("/dev/null", "w");
    char title[1024];
    IO::read(fp, devnull, s->m, title);
    fclose(devnull);
    IO::read(fp, s->nBlock);
    s->blockStruct.resize(s->nBlock);
    s->blockType.resize(s->nBlock);
    s->blockNumber.resize(s->nBlock);
    IO::read(fp, s->nBlock, s->blockStruct.data());
    for (int i = 0; i < s->nBlock; ++i) {
        int &bs = s->blockStruct[i];
        if (bs >= 2) {
            s->blockType[i] = 1;
            s->blockNumber[i] = s->SDP_nBlock++;
        } else if (bs < 0) {
            s->blockType[i] = 3;
            bs = -bs;
            s->blockNumber[i] = s->LP_nBlock;
            s->LP_nBlock += bs;
        } else if (bs == 1) {
            s->blockType[i] = 3;
            s->blockNumber[i] = s->LP_nBlock;
            s->LP_nBlock += bs;
        } else {
            fclose(fp);
            delete s;
            return nullptr;
        }
    }
    for (int i = 0; i < s->nBlock; ++i)
        if (s->blockType[i] == 1) s->SDP_blockStruct.push_back(s->blockStruct[i]);
    s->SOCP_blockStruct.resize(1);
    // sparse input when the file name ends in "-s", as sdpa_main.cpp:611-614
    size_t fl = strlen(dataFile);
    bool isDataSparse = fl >= 2 && dataFile[fl - 1] == 's' && dataFile[fl - 2] == '-';
    IO::read(fp, s->m, s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock, s->nBlock, s->blockStruct.data(), s->blockType.data(), s->blockNumber.data(), s->inputData, isDataSparse);
    s->inputData.initialize_index(s->SDP_nBlock, s->SOCP_nBlock, s->LP_nBlock, s->com);
    fclose(fp);
    s->inputData.C.changeToDense();
    for (int k = 0; k < s->m; ++k) s->inputData.A[k].changeToDense();
    s->newton = new Newton(s->m, s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock);
    Chordal chordal;
    if (schurMode == 1) {
        chordal.m_threshold = 10000000;
        chordal.b_threshold = 1000000;
        chordal.aggregate_threshold = 0.0;
        chordal.extend_threshold = 0.0;
    } else if (schurMode == 2) {
        chordal.m_threshold = 0;
        chordal.b_threshold = 0;
        chordal.aggregate_threshold = 2.0;
        chordal.extend_threshold = 2.0;
    }
    FILE *devnull2 = fopen("/dev/null", "w");
    chordal.ordering_bMat(s->m, s->SDP_nBlock + s->SOCP_nBlock + s->LP_nBlock, s->inputData, devnull2);
    s->newton->initialize_bMat(s->m, chordal, s->inputData, devnull2);
    fclose(devnull2);
    chordal.terminate();
    s->newton->computeFormula_SDP(s->inputData, 0.0, kappa);
    s->currentPt.initialize(s->m, s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock, s->param.lambdaStar, s->com);
    s->work.initialize(s->m, s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock);
    s->initRes = new Residuals(s->m, s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock, s->inputData, s->currentPt);
    s->currentRes.copyFrom(*s->initRes);
    s->beta.initialize(s->param.betaStar);
    s->reduction.initialize(Switch::ON);
    s->mu.initialize(s->param.lambdaStar);
    s->theta.initialize(s->param, *s->initRes);
    s->solveInfo.initialize(s->inputData, s->currentPt, s->mu.initial, s->param.omegaStar);
    s->phase.initialize(*s->initRes, s->solveInfo, s->param, s->currentPt.nDim);
    s->bCaptured.initialize(s->m, s->m, DenseMatrix::DENSE);
    s->gPred.initialize(s->m);
    s->dyPred.initialize(s->m);
    s->dxPred.initialize(s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock);
    s->dzPred.initialize(s->SDP_nBlock, s->SDP_blockStruct.data(), s->SOCP_nBlock, s->SOCP_blockStruct.data(), s->LP_nBlock);
    return s;
}

void *ref_open(const char *dataFile, const char *paramFile, double kappa) { return ref_open_mode(dataFile, paramFile, kappa, 0); }

void ref_close(void *h) {
    RefSolver *s = (RefSolver *)h;
    if (!s) return;
    delete s->initRes;
    delete s->newton;
    delete s;
}

// Sizes: out[0]=m, out[1]=SDP_nBlock, out[2]=LP_nBlock, out[3]=nDim,
// out[4..] = SDP block sizes.
int ref_dims(void *h, int *out, int cap) {
    RefSolver *s = (RefSolver *)h;
    int need = 4 + s->SDP_nBlock;
    if (cap < need) return -need;
    out[0] = s->m;
    out[1] = s->SDP_nBlock;
    out[2] = s->LP_nBlock;
    out[3] = s->currentPt.nDim;
    for (int l = 0; l < s->SDP_nBlock; ++l) out[4 + l] = s->SDP_blockStruct[l];
    return need;
}

// Formula table useFormula[i * SDP_nBlock + l] (0=F1, 1=F2, 2=F3).
void ref_formula(void *h, int *out) {
    RefSolver *s = (RefSolver *)h;
    for (int i = 0; i < s->m * s->SDP_nBlock; ++i) out[i] = (int)s->newton->useFormula[i];
}

// One pass of pinpal's main loop (sdpa_main.cpp:294-376) with the
// intermediates captured.  Returns 0 when the loop continues, 1 when the
// loop condition ended it before this pass, 2 on Cholesky failure of B,
// 3 on the pdFEAS early stop, 4 on "cannot move".
int ref_step(void *h) {
    RefSolver *s = (RefSolver *)h;
    if (!(s->phase.updateCheck(s->currentRes, s->solveInfo, s->param) && s->pIteration < s->param.maxIteration)) return 1;
    s->phaseAtStep = (int)s->phase.value;
    s->reduction.MehrotraPredictor(s->phase);
    s->beta.MehrotraPredictor(s->phase, s->reduction, s->param);
    s->betaPred = s->beta.value;
    Newton &nt = *s->newton;
    // Newton::Mehrotra(PREDICTOR) split open (sdpa_newton.cpp:1345-1384)
    nt.Make_gVec(Newton::PREDICTOR, s->inputData, s->currentPt, s->currentRes, s->mu, s->beta, s->phase, s->work, s->com);
    if (s->capture) s->gPred.copyFrom(nt.gVec);
    nt.Make_bMat(s->inputData, s->currentPt, s->work, s->com);
    if (s->capture) capture_B(*s);
    if (!nt.compute_DyVec(Newton::PREDICTOR, s->inputData, s->currentPt, s->work, s->com)) return 2;
    nt.compute_DzMat(s->inputData, s->currentRes, s->phase, s->com);
    nt.compute_DxMat(s->currentPt, s->work, s->com);
    if (s->capture) {
        s->dxPred.copyFrom(nt.DxMat);
        s->dyPred.copyFrom(nt.DyVec);
        s->dzPred.copyFrom(nt.DzMat);
    }
    s->alpha.MehrotraPredictor(s->inputData, s->currentPt, s->phase, nt, s->work, s->com);
    s->alphaPredP = s->alpha.primal;
    s->alphaPredD = s->alpha.dual;
    s->beta.MehrotraCorrector(s->phase, s->alpha, s->currentPt, nt, s->mu, s->param);
    s->betaCorr = s->beta.value;
    if ((s->phase.value == SolveInfo::pdFEAS) && ((s->beta.value > 5) || (s->solveInfo.objValPrimal < s->solveInfo.objValDual))) return 3;
    nt.Mehrotra(Newton::CORRECTOR, s->inputData, s->currentPt, s->currentRes, s->mu, s->beta, s->reduction, s->phase, s->work, s->com);
    if (s->capture) {
        s->minEigX = Jal::getMinEigen(s->currentPt.invCholeskyX, nt.DxMat, s->work);
        s->minEigZ = Jal::getMinEigen(s->currentPt.invCholeskyZ, nt.DzMat, s->work);
    }
    s->alpha.MehrotraCorrector(s->inputData, s->currentPt, s->phase, s->reduction, nt, s->mu, s->theta, s->work, s->param, s->com);
    s->muAtStep = s->mu.current;
    s->thetaPAtStep = s->theta.primal;
    s->thetaDAtStep = s->theta.dual;
    s->objPAtStep = s->solveInfo.objValPrimal;
    s->objDAtStep = s->solveInfo.objValDual;
    if (!s->currentPt.update(s->alpha, nt, s->work, s->com)) return 4;
    s->theta.update(s->reduction, s->alpha);
    s->mu.update(s->currentPt);
    s->currentRes.update(s->m, s->inputData, s->currentPt, s->com);
    s->theta.update_exact(*s->initRes, s->currentRes);
    s->solveInfo.update(s->param.lambdaStar, s->inputData, s->currentPt, s->currentRes, s->mu, s->theta, s->param);
    s->pIteration++;
    return 0;
}

// Arrays.  what: 0 X, 1 Z, 2 y, 3 invCholX, 4 invCholZ, 5 invZ,
// 6 B (Schur matrix before factorisation, m x m), 7 B factor (after the
// last Cholesky, lower part meaningful), 8 g (predictor RHS), 9 Dx, 10 Dy,
// 11 Dz (corrector), 12 Dx, 13 Dy, 14 Dz (predictor), 15 dual residual
// matrix, 16 primal residual vector.  Returns the number of dd values, or
// -1 for an unknown selector.  With out == NULL only the size is returned.
long ref_get(void *h, int what, double *out) {
    RefSolver *s = (RefSolver *)h;
    Newton &nt = *s->newton;
    DenseLinearSpace *sp = nullptr;
    Vector *v = nullptr;
    DenseMatrix *dm = nullptr;
    switch (what) {
    case 0: sp = &s->currentPt.xMat; break;
    case 1: sp = &s->currentPt.zMat; break;
    case 2: v = &s->currentPt.yVec; break;
    case 3: sp = &s->currentPt.invCholeskyX; break;
    case 4: sp = &s->currentPt.invCholeskyZ; break;
    case 5: sp = &s->currentPt.invzMat; break;
    case 6: dm = &s->bCaptured; break;
    case 7: dm = &nt.bMat; break;
    case 8: v = &s->gPred; break;
    case 9: sp = &nt.DxMat; break;
    case 10: v = &nt.DyVec; break;
    case 11: sp = &nt.DzMat; break;
    case 12: sp = &s->dxPred; break;
    case 13: v = &s->dyPred; break;
    case 14: sp = &s->dzPred; break;
    case 15: sp = &s->currentRes.dualMat; break;
    case 16: v = &s->currentRes.primalVec; break;
    default: return -1;
    }
    if (sp) {
        if (out) space_get(*sp, out);
        return (long)space_len(*sp);
    }
    if (v) {
        if (out) vec_get(*v, out);
        return v->nDim;
    }
    long len = (long)dm->nRow * dm->nCol;
    if (out)
        for (long i = 0; i < len; ++i) st(out + 2 * i, dm->de_ele[i]);
    return len;
}

// Overwrites the current point and refreshes everything pinpal derives from
// it in Solutions::update and the loop tail (inverses, mu, residuals,
// theta.update_exact, solveInfo).  Returns 0, or 1 when an inverse
// Cholesky fails.
int ref_set_point(void *h, const double *X, const double *y, const double *Z) {
    RefSolver *s = (RefSolver *)h;
    space_set(s->currentPt.xMat, X);
    vec_set(s->currentPt.yVec, y);
    space_set(s->currentPt.zMat, Z);
    bool ok = s->currentPt.computeInverse(s->work, s->com);
    s->mu.update(s->currentPt);
    s->currentRes.update(s->m, s->inputData, s->currentPt, s->com);
    s->theta.update_exact(*s->initRes, s->currentRes);
    s->solveInfo.update(s->param.lambdaStar, s->inputData, s->currentPt, s->currentRes, s->mu, s->theta, s->param);
    return ok ? 0 : 1;
}

// Schur matrix B of the current point (Newton::Make_bMat,
// sdpa_newton.cpp:1223-1244) without touching the loop state.
void ref_schur(void *h, double *out) {
    RefSolver *s = (RefSolver *)h;
    s->newton->Make_bMat(s->inputData, s->currentPt, s->work, s->com);
    capture_B(*s);
    long len = (long)s->m * s->m;
    for (long i = 0; i < len; ++i) st(out + 2 * i, s->bCaptured.de_ele[i]);
}

// 1 when Newton::initialize_bMat chose the sparse Schur form.
int ref_schur_sparse(void *h) { return ((RefSolver *)h)->newton->bMat_type == Newton::SPARSE ? 1 : 0; }

// The sparse form's layout: ordering[m] (new -> old), diagonalIndex[m + 1],
// column_index[nnz] (any of them may be NULL).  Returns nnz, or -1 when B
// is dense.
long ref_sparse_layout(void *h, int *ordering, int *diagonalIndex, int *column_index) {
    RefSolver *s = (RefSolver *)h;
    Newton &nt = *s->newton;
    if (nt.bMat_type != Newton::SPARSE) return -1;
    const long nnz = nt.sparse_bMat.NonZeroCount;
    if (ordering) std::copy(nt.ordering, nt.ordering + s->m, ordering);
    if (diagonalIndex) std::copy(nt.diagonalIndex, nt.diagonalIndex + s->m + 1, diagonalIndex);
    if (column_index) std::copy(nt.sparse_bMat.column_index, nt.sparse_bMat.column_index + nnz, column_index);
    return nnz;
}

// The sparse form's entries (after a pass: the factor of the last
// Cholesky).  Returns nnz, or -1 when B is dense.
long ref_sparse_values(void *h, double *out) {
    RefSolver *s = (RefSolver *)h;
    Newton &nt = *s->newton;
    if (nt.bMat_type != Newton::SPARSE) return -1;
    const long nnz = nt.sparse_bMat.NonZeroCount;
    if (out)
        for (long k = 0; k < nnz; ++k) st(out + 2 * k, nt.sparse_bMat.sp_ele[k]);
    return nnz;
}

// Scalars of the last pass / current state:
//  0 mu.current 1 mu.initial 2 theta.primal 3 theta.dual 4 alpha.primal
//  5 alpha.dual 6 beta (corrector) 7 objValPrimal 8 objValDual
//  9 normPrimalVec 10 normDualMat 11 rho 12 etaPrimal 13 etaDual
// 14 alphaPred.primal 15 alphaPred.dual 16 betaPred 17 minEig(L_X Dx L_X^T)
// 18 minEig(L_Z Dz L_Z^T) 19 mu at the printed line 20 thetaP printed
// 21 thetaD printed 22 objP printed 23 objD printed
int ref_scalar(void *h, int what, double *out) {
    RefSolver *s = (RefSolver *)h;
    dd_real v;
    switch (what) {
    case 0: v = s->mu.current; break;
    case 1: v = s->mu.initial; break;
    case 2: v = s->theta.primal; break;
    case 3: v = s->theta.dual; break;
    case 4: v = s->alpha.primal; break;
    case 5: v = s->alpha.dual; break;
    case 6: v = s->beta.value; break;
    case 7: v = s->solveInfo.objValPrimal; break;
    case 8: v = s->solveInfo.objValDual; break;
    case 9: v = s->currentRes.normPrimalVec; break;
    case 10: v = s->currentRes.normDualMat; break;
    case 11: v = s->solveInfo.rho; break;
    case 12: v = s->solveInfo.etaPrimal; break;
    case 13: v = s->solveInfo.etaDual; break;
    case 14: v = s->alphaPredP; break;
    case 15: v = s->alphaPredD; break;
    case 16: v = s->betaPred; break;
    case 17: v = s->minEigX; break;
    case 18: v = s->minEigZ; break;
    case 19: v = s->muAtStep; break;
    case 20: v = s->thetaPAtStep; break;
    case 21: v = s->thetaDAtStep; break;
    case 22: v = s->objPAtStep; break;
    case 23: v = s->objDAtStep; break;
    default: return -1;
    }
    st(out, v);
    return 0;
}

// on != 0 (the default): ref_step keeps copies of the last pass's
// intermediates; 0: it runs the stock loop body only.
void ref_set_capture(void *h, int on) { ((RefSolver *)h)->capture = on != 0; }

// The reference's own accumulated timers (ComputeTime, sdpa_parts.h):
// out[0] "Make bMat" seconds (sdpa_newton.cpp:1243), out[1] "Cholesky bMat"
// seconds (sdpa_newton.cpp:1299).
void ref_times(void *h, double *out) {
    RefSolver *s = (RefSolver *)h;
    out[0] = s->com.makebMat;
    out[1] = s->com.choleskybMat;
}

// Phase (SolveInfo::phaseType as int) and iteration counter.
int ref_phase(void *h) { return (int)((RefSolver *)h)->phase.value; }
// Phase at the start of the last pass (before the step's updates).
int ref_phase_at_step(void *h) { return ((RefSolver *)h)->phaseAtStep; }
int ref_iteration(void *h) { return ((RefSolver *)h)->pIteration; }

} // extern "C"

// ----------------------------------------------------------------------
// Quad-double (qd_real, QD 2.3.23, ~212 bits) error oracle: the same
// quantities as the dd path computed in qd_real from the same dd inputs, so
// that the error of a dd result can be stated against a value 2^-100 more
// accurate.  qd values cross as 4 doubles per entry.
namespace {
inline qd_real ldq(const double *p) { return qd_real(p[0], p[1], p[2], p[3]); }
inline void stq(double *p, const qd_real &v) {
    for (int i = 0; i < 4; ++i) p[i] = v.x[i];
}
inline qd_real from_dd(const double *p) { return qd_real(dd_real(p[0], p[1])); }
} // namespace

extern "C" {

// Lower Cholesky of the symmetric n x n dd matrix A (column-major, lower
// triangle read) in qd; L receives n*n qd values (upper triangle zero).
// Returns 0 or the 1-based failing column.
long qd_potrf(long n, const double *A, double *L) {
    std::vector<qd_real> a((size_t)n * n);
    for (long j = 0; j < n; ++j)
        for (long i = 0; i < n; ++i) a[i + n * j] = i >= j ? from_dd(A + 2 * (i + n * j)) : qd_real(0.0);
    for (long j = 0; j < n; ++j) {
        qd_real d = a[j + n * j];
        for (long k = 0; k < j; ++k) d -= a[j + n * k] * a[j + n * k];
        if (!(d > 0.0)) return j + 1;
        d = sqrt(d);
        a[j + n * j] = d;
        for (long i = j + 1; i < n; ++i) {
            qd_real v = a[i + n * j];
            for (long k = 0; k < j; ++k) v -= a[i + n * k] * a[j + n * k];
            a[i + n * j] = v / d;
        }
    }
    for (size_t e = 0; e < a.size(); ++e) stq(L + 4 * e, a[e]);
    return 0;
}

// x = (L L^T)^-1 b in qd for a qd lower factor L and a dd right-hand side.
void qd_chol_solve(long n, const double *L, const double *b, double *x) {
    std::vector<qd_real> v(n);
    for (long i = 0; i < n; ++i) v[i] = from_dd(b + 2 * i);
    for (long i = 0; i < n; ++i) {
        for (long k = 0; k < i; ++k) v[i] -= ldq(L + 4 * (i + n * k)) * v[k];
        v[i] /= ldq(L + 4 * (i + n * i));
    }
    for (long i = n - 1; i >= 0; --i) {
        for (long k = i + 1; k < n; ++k) v[i] -= ldq(L + 4 * (k + n * i)) * v[k];
        v[i] /= ldq(L + 4 * (i + n * i));
    }
    for (long i = 0; i < n; ++i) stq(x + 4 * i, v[i]);
}

// B_ij = A_j . (X A_i Zi) in qd for m dense symmetric n x n dd matrices A
// (consecutive, column-major) and dd X, Zi: the Schur matrix of the F1
// formula (sdpa_newton.cpp:895) without rounding.  B: m*m qd values.
void qd_schur_dense(long n, long m, const double *A, const double *X, const double *Zi, double *B) {
    const long nn = n * n;
    std::vector<qd_real> x(nn), z(nn), a((size_t)m * nn), t(nn), g(nn);
    for (long e = 0; e < nn; ++e) {
        x[e] = from_dd(X + 2 * e);
        z[e] = from_dd(Zi + 2 * e);
    }
    for (long e = 0; e < m * nn; ++e) a[e] = from_dd(A + 2 * e);
    for (long i = 0; i < m; ++i) {
        const qd_real *ai = a.data() + i * nn;
        for (long c = 0; c < n; ++c) // t = A_i Zi
            for (long r = 0; r < n; ++r) {
                qd_real s = 0.0;
                for (long k = 0; k < n; ++k) s += ai[r + n * k] * z[k + n * c];
                t[r + n * c] = s;
            }
        for (long c = 0; c < n; ++c) // g = X t
            for (long r = 0; r < n; ++r) {
                qd_real s = 0.0;
                for (long k = 0; k < n; ++k) s += x[r + n * k] * t[k + n * c];
                g[r + n * c] = s;
            }
        for (long j = 0; j < m; ++j) {
            const qd_real *aj = a.data() + j * nn;
            qd_real s = 0.0;
            for (long e = 0; e < nn; ++e) s += aj[e] * g[e];
            stq(B + 4 * (i + m * j), s);
        }
    }
}

// out[0] = max_e |dd_e - qd_e|, out[1] = max_e |qd_e| (leading doubles),
// over n entries; with lower != 0 only the lower triangle of the square
// order-ord matrix counts.
void qd_maxdiff(long n, const double *dd, const double *qd, int lower, long ord, double *out) {
    double md = 0.0, mq = 0.0;
    for (long e = 0; e < n; ++e) {
        if (lower && (e % ord) < (e / ord)) continue;
        const qd_real q = ldq(qd + 4 * e);
        const qd_real d = from_dd(dd + 2 * e) - q;
        md = std::max(md, std::fabs(d.x[0]));
        mq = std::max(mq, std::fabs(q.x[0]));
    }
    out[0] = md;
    out[1] = mq;
}

} // extern "C"
