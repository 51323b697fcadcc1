/*
 * sddd.h - C ABI of the B200 double-double (dd) Newton hot path of SDPA-DD.
 *
 * One opaque context per host thread; all problem, iterate and Newton data
 * stay resident on one GPU.  dd values cross the boundary as sddd_dd
 * {hi, lo}, byte-compatible with QD's dd_real (double x[2]).  Block spaces
 * (X, Z, Dx, ...) are the SDP blocks of the problem in order, each
 * n_l x n_l column-major, concatenated.
 *
 * Every call returns an int status: SDDD_OK (0); > 0 only from the
 * Cholesky entry points, the 1-based column where the matrix stopped being
 * positive definite (LAPACK info, as the reference's Rpotrf returns);
 * < 0 an error (sddd_last_error() gives the message).  Nothing calls exit().
 *
 * Reference interfaces replaced (file:line in nakatamaho/sdpa-dd 7.1.3):
 *   reading / InputData   sdpa_io.cpp:428-786, sdpa_dataset.cpp:470-493
 *   Solutions             sdpa_dataset.cpp:35-143
 *   Newton                sdpa_newton.cpp:694-1384
 *   StepLength etc.       sdpa_parts.cpp:244-954
 *   pinpal / sdpa_dd      sdpa_main.cpp:43-672
 *   MPLAPACK kernels      mplapack/mpblas_dd.h:38-56, mplapack_dd.h:38-92
 */
#ifndef SDDD_H
#define SDDD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double hi, lo;
} sddd_dd;

typedef struct sddd_ctx sddd_ctx;

#define SDDD_OK 0
#define SDDD_ERR_ARG (-1)
#define SDDD_ERR_CUDA (-2)
#define SDDD_ERR_NOCONV (-3)
#define SDDD_ERR_STATE (-4)
#define SDDD_ERR_NOMEM (-5)
#define SDDD_ERR_IO (-6)
#define SDDD_ERR_UNSUPPORTED (-7)

/* Parameter (sdpa_parts.h:85-104; defaults sdpa_parts.cpp:136-171). */
typedef struct {
    int maxIteration;
    double epsilonStar, lambdaStar, omegaStar, lowerBound, upperBound, betaStar, betaBar, gammaStar, epsilonDash;
} sddd_param;

/* Outcome of a solve (the numbers IO::printLastInfo reports,
 * sdpa_io.cpp:1015-1203, with REVERSE_PRIMAL_DUAL applied). */
typedef struct {
    int phase;            /* SolveInfo::phaseType after Phase::reverse */
    int iterations;
    int stop_reason;      /* 1 loop condition, 2 Cholesky(B) failed, 3 pdFEAS early stop, 4 cannot move */
    sddd_dd mu, relative_gap, gap;
    sddd_dd objValPrimal; /* printed "objValPrimal" = -b.y */
    sddd_dd objValDual;   /* printed "objValDual" = -C.X */
    sddd_dd pfeas_error, dfeas_error;
    double main_loop_seconds, schur_seconds, cholesky_seconds;
} sddd_result;

const char *sddd_version(void);
const char *sddd_last_error(const sddd_ctx *ctx);

/* Context on CUDA device `device`. */
int sddd_create(int device, sddd_ctx **out);
int sddd_destroy(sddd_ctx *ctx);

/* -- parameters (Parameter::setDefaultParameter / readFile) -- */
int sddd_param_default(int type, sddd_param *out); /* 0 default, 1 fast, 2 stable */
int sddd_param_read(const char *path, sddd_param *out);

/* -- problem (IO::read + InputData::initialize_index + changeToDense +
 *    Newton::computeFormula_SDP) -- */
/* Read SDPA text: sparse (.dat-s) when `sparse` != 0, else dense (.dat). */
int sddd_read_problem(sddd_ctx *ctx, const char *path, int sparse, double kappa);
/* The same from memory: nnz entries (k, blk, i, j, val) in SDPA's
 * conventions (k = 0 is F_0, 1-based block/row/column, upper triangle);
 * block_struct as in the file (negative = LP).  Data is copied. */
int sddd_upload_problem(sddd_ctx *ctx, int m, int nblock, const int *block_struct, const sddd_dd *b, long nnz, const int *k, const int *blk,
                        const int *i, const int *j, const sddd_dd *val, double kappa);
/* m, number of SDP blocks, nDim; sizes[] gets the SDP block sizes.  LP
 * entries (negative block sizes) are carried as SDP blocks of order 1 after
 * the data's SDP blocks, one per entry in the file's LP order: they count
 * in nsdp and sizes[], and every block space (points, gradients) holds them
 * there.  The result file and initial-point files keep the reference's LP
 * layout. */
int sddd_dims(const sddd_ctx *ctx, int *m, int *nsdp, long *ndim, int *sizes, int cap);
/* The same dimensions for a problem file, read on the host only (no device,
 * no context): for sizing buffers or planning a batch before any GPU work.
 * space_len is the length in dd of a block space of that problem. */
int sddd_problem_info(const char *path, int sparse, int *m, int *nsdp, long *space_len, int *sizes, int cap);
/* Length in dd of a block space. */
long sddd_space_len(const sddd_ctx *ctx);
/* Formula table useFormula[k * nsdp + l] (0 F1, 1 F2, 2 F3, -1 absent). */
int sddd_formula(const sddd_ctx *ctx, int *out);

/* -- iterate (Solutions) -- */
int sddd_init_point(sddd_ctx *ctx, sddd_dd lambda);
/* Set X, y, Z (host arrays) and recompute L_X^-1, L_Z^-1, Z^-1; returns 1
 * when a Cholesky factorisation of X or Z fails. */
int sddd_set_point(sddd_ctx *ctx, const sddd_dd *X, const sddd_dd *y, const sddd_dd *Z);
int sddd_get_point(sddd_ctx *ctx, sddd_dd *X, sddd_dd *y, sddd_dd *Z);
int sddd_compute_inverse(sddd_ctx *ctx);

/* -- Newton pieces (Newton::Mehrotra split open) -- */
/* compute_rMat + Make_gVec; dual_infeasible = phase is pFEAS or noINFO. */
int sddd_newton_rhs(sddd_ctx *ctx, int corrector, sddd_dd beta_mu, int dual_infeasible);
int sddd_schur_build(sddd_ctx *ctx);   /* Make_bMat */
int sddd_schur_factor(sddd_ctx *ctx);  /* Cholesky of B; > 0 = failing column */
int sddd_solve_dy(sddd_ctx *ctx);      /* Dy = B^-1 g */
int sddd_make_dz_dx(sddd_ctx *ctx, int dual_infeasible);
/* min eigenvalue of L D L^T for the step length: which = 0 (L_X^-1, Dx) or 1 (L_Z^-1, Dz). */
int sddd_min_eig(sddd_ctx *ctx, int which, sddd_dd *out);
/* The same eigenvalue for ONE block of order n, with no device allocation.
 * It has no counterpart in the reference.  It is for callers that cannot
 * let a library allocate: a process whose memory pool already holds the
 * GPU (cudaMalloc would fail) or whose other streams must not stall
 * (cudaFree synchronises the device).  L (lower triangle read), D
 * (symmetric) and out (one dd) are device pointers, n x n column-major;
 * the work goes on `stream` (a cudaStream_t, NULL = legacy default) of the
 * current device and *out is written asynchronously on it.
 * Scratch is a static device array that every GPU loading the library holds
 * until exit: about 320 KiB, enough for n <= SDDD_MIN_EIG_NOALLOC_MAX_N;
 * a larger n returns SDDD_ERR_ARG with a message in sddd_last_error(NULL).
 * The first call on each device looks up the array's address (make it
 * before any stream capture).  All calls share the array: calls that
 * overlap on the GPU race. */
#define SDDD_MIN_EIG_NOALLOC_MAX_N 4096
int sddd_min_eig_noalloc(void *stream, long n, const sddd_dd *L, const sddd_dd *D, sddd_dd *out);
int sddd_update(sddd_ctx *ctx, sddd_dd alpha_primal, sddd_dd alpha_dual);
int sddd_residuals(sddd_ctx *ctx, sddd_dd *norm_primal, sddd_dd *norm_dual);
/* Inner products: 0 C.X, 1 b.y, 2 X.Z, 3 C.Dx, 4 b.Dy, 5 X.Dz, 6 Dx.Z, 7 Dx.Dz */
int sddd_inner(sddd_ctx *ctx, int which, sddd_dd *out);
/* Device arrays to host: 0 X 1 Z 2 y 3 invCholX 4 invCholZ 5 invZ 6 B
 * 7 g 8 Dx 9 Dy 10 Dz 11 dual residual 12 primal residual, after
 * sddd_adjoint 13 its u 14 its R.  Returns the
 * number of dd written (with out == NULL: the number it would write). */
long sddd_get(sddd_ctx *ctx, int what, sddd_dd *out);
int sddd_set(sddd_ctx *ctx, int what, const sddd_dd *in);

/* -- initial point (the reference's -id / -is files, sdpa_main.cpp:237-251,
 *    sdpa_io.cpp:152-283) --
 * The next solves start from it instead of lambda I, with the reference's
 * initial mu (X.Z / nDim) and its eta bookkeeping (SolveInfo::update with
 * the initial point).  sddd_read_initial_point reads an init file (sparse
 * != 0: "target block i j value" lines, target 1 = X, 2 = Y; else dense),
 * whose unset entries keep lambda I (pass param.lambdaStar, as the
 * reference starts from it); sddd_set_initial_point takes the file's x (m),
 * X and Y (block spaces) directly.  A new problem clears it. */
int sddd_read_initial_point(sddd_ctx *ctx, const char *path, int sparse, double lambda);
int sddd_set_initial_point(sddd_ctx *ctx, const sddd_dd *x, const sddd_dd *X, const sddd_dd *Y);
int sddd_clear_initial_point(sddd_ctx *ctx);
/* The current point (after a solve: the final one) as an initial-point file
 * that sddd_read_initial_point, the -id / -is options and the reference's
 * own reader (sdpa_io.cpp:152-283) take, every number with 34 significant
 * digits, so a later solve can start from it (warm start, checkpoint).  The
 * reference writes only the high doubles of its result (sdpa_io.cpp:1205-
 * 1234); read back, this file gives the
 * dd point to a few units in its last place.  sparse != 0: "target block i
 * j value" lines (diagonal always, other zeros left out); else dense. */
int sddd_write_point(sddd_ctx *ctx, const char *path, int sparse);
/* v as a correctly rounded decimal string of `digits` (1..60) significant
 * digits ("d.ddd...e+XX"), exact from hi + lo; writes at most len bytes with
 * the terminating zero and returns the string length (needs no device). */
int sddd_dd_to_decimal(sddd_dd v, int digits, char *buf, int len);

/* -- the whole solve (pinpal) -- */
/* display/result may be NULL.  The result file gets the reference's
 * layout; `display` is the console stream. */
int sddd_solve(sddd_ctx *ctx, const sddd_param *param, const char *result_path, int print, sddd_result *out);
/* Step-wise driving of the same loop: start, then sddd_iterate until it
 * returns non-zero (1 = converged / loop ended, 2, 3, 4 as stop_reason). */
int sddd_solver_start(sddd_ctx *ctx, const sddd_param *param);
int sddd_iterate(sddd_ctx *ctx);
int sddd_solver_result(sddd_ctx *ctx, sddd_result *out);
/* The reference's command line (sdpa_main.cpp:493-672). */
int sddd_cli_main(int argc, char **argv);

/* -- adjoint of a finished solve (no counterpart in the reference) --
 * Gradients with respect to the file's data c, F_0, F_1..F_m at the
 * context's current iterate (normally where sddd_solve stopped), for
 * weights on the outputs: g_x on x (m), g_Y on Y and g_X on X (block
 * spaces), g_obj on the optimal value c.x; host arrays, NULL = zero.
 * It differentiates the central-path equations at the iterate (the same
 * HKM linearisation the solver's Schur matrix B comes from), builds and
 * factors B there and solves with it once; as the gap goes to zero the
 * result tends to the derivative of the optimal solution, and for g_obj to
 * the envelope gradient (x, Y, -x_k Y).  A matrix gradient G is the
 * symmetric one: d(value) = sum_ij G_ij dF_ij for a symmetric change dF
 * (an off-diagonal entry listed once in the file moves F_ij and F_ji, so
 * its derivative is 2 G_ij).  Outputs: grad_c (m) and grad_F0 (block space),
 * each may be NULL.  Returns > 0 (failing column) when B is not positive
 * definite at the iterate.  Overwrites the Newton direction and B.
 * The optimal value's part is the linearisation at the iterate; the part
 * for weights on x, Y, X is taken at the optimum: the iterate's
 * eigendecomposition (dd Jacobi) gives exactly central points X_c Z_c =
 * mu I with its range and null space, the adjoint is evaluated there at
 * mu = h, 2h, 4h and extrapolated to mu -> 0 (the iterate itself is off the
 * central path, where the HKM coupling of the two spaces is not the
 * optimum's).  Accuracy at gap 1e-25, against sixth-order finite
 * differences of whole solves (which carry ~1e-21 of solve noise
 * themselves): at most 1.75e-20 relative for the optimal value at m = 60
 * and 5.1e-20 at m = 1326 (measured on B200 over entries of c and F),
 * 1e-18 to 1e-14 for the solution.  SDP blocks up to order 1024.
 * sddd_adjoint_grad_F then gives the gradient for F_k, k = 1..m, from the
 * same adjoint.  sddd_get 13 and 14 return its vector u = B^-1 (...) and
 * the matrix R (grad_F0 = -R, grad_F_k = -u_k Y + x_k R). */
int sddd_adjoint(sddd_ctx *ctx, const sddd_dd *g_x, const sddd_dd *g_Y, const sddd_dd *g_X, sddd_dd g_obj, sddd_dd *grad_c, sddd_dd *grad_F0);
int sddd_adjoint_grad_F(sddd_ctx *ctx, int k, sddd_dd *grad_Fk);

/* -- batches of independent problems (no counterpart in the reference) --
 * Many SDPs solved on one GPU by a pool of `workers` host threads (<= 0:
 * min(8, host cores)), each with its own context and stream, so the small
 * kernels of many problems run at once.  The Schur build and Cholesky of B
 * of the problems with one block of dense constraints (the dense random
 * kind) run batched across the workers: one captured CUDA graph of
 * persistent launches per gathering, tile shapes autotuned per size class
 * (sddd_batch_set_core turns it off; sddd_batch_tuning reports the shapes).  Every problem is solved exactly as sddd_solve
 * solves it (same iterates, bit for bit).  Problems are added from SDPA
 * text or from memory (the arguments of sddd_read_problem /
 * sddd_upload_problem); the add calls return the problem's index.
 * sddd_batch_solve fills results[count] and, with with_grad != 0, the
 * gradient of each optimal value with respect to its c (sddd_adjoint with
 * g_obj = 1).  It returns the first problem error (< 0) after solving all
 * others; sddd_batch_status gives each problem's (0, > 0 failing column of
 * B at the adjoint, < 0 error).  Points and gradients are kept on the host:
 * X and Z as block spaces of that problem, y and grad_c of length m. */
typedef struct sddd_batch sddd_batch;
int sddd_batch_create(int device, int workers, sddd_batch **out);
int sddd_batch_destroy(sddd_batch *b);
const char *sddd_batch_last_error(const sddd_batch *b);
int sddd_batch_add_file(sddd_batch *b, const char *path, int sparse, double kappa);
int sddd_batch_add_problem(sddd_batch *b, int m, int nblock, const int *block_struct, const sddd_dd *bvec, long nnz, const int *k, const int *blk,
                           const int *i, const int *j, const sddd_dd *val, double kappa);
int sddd_batch_count(const sddd_batch *b);
int sddd_batch_solve(sddd_batch *b, const sddd_param *param, int with_grad, sddd_result *results);
int sddd_batch_status(const sddd_batch *b, int index);
int sddd_batch_get_point(const sddd_batch *b, int index, sddd_dd *X, sddd_dd *y, sddd_dd *Z);
int sddd_batch_grad_c(const sddd_batch *b, int index, sddd_dd *grad_c);
int sddd_batch_set_core(sddd_batch *b, int on);
const char *sddd_batch_tuning(const sddd_batch *b);

/* -- measurement -- */
/* Kernels this library has launched in this process so far. */
unsigned long long sddd_launch_count(void);
/* The context's CUDA stream (cudaStream_t) for event timing by callers. */
void *sddd_stream(sddd_ctx *ctx);
/* Per-kernel CUDA-event timing inside the library, for the calling thread:
 * enable/disable, read (collects: synchronises the stream) and reset.
 * Names: potrf_trailing_update, potrf_diag, potrf_panel, trsv,
 * schur_build, min_eig. */
int sddd_profile(sddd_ctx *ctx, int enable);
int sddd_profile_read(sddd_ctx *ctx, const char *name, double *ms, long *launches);
int sddd_profile_reset(sddd_ctx *ctx);
/* Algorithmic dd-flops of one Schur build and of one Cholesky of B. */
int sddd_work(const sddd_ctx *ctx, double *schur_ddflops, double *chol_ddflops);
/* Measured FP64 fused multiply-add throughput of the current device (GFLOP/s). */
int sddd_fp64_peak(sddd_ctx *ctx, double *gflops);

/* -- tensor-core split (no counterpart in the reference) --
 * With slices in 8..16 the Cholesky of the Schur matrix B (sddd_schur_factor,
 * sddd_Rpotrf, whole solves) runs its trailing updates C -= P P^T as
 * products of signed 7-bit integer slices of the dd operands on the INT8
 * tensor cores, exact in int32, rebuilt in dd: each value is carried to
 * 7*slices+1 bits of its row's largest entry (16 slices: 113 bits).  The
 * diagonal blocks, the panel solves and everything else stay in plain dd.
 * 0 (the default) keeps the reference's operation order, bit for bit. */
int sddd_set_tc_split(sddd_ctx *ctx, int slices);
int sddd_get_tc_split(const sddd_ctx *ctx);
/* C(i,j) -= sum_k P(i,k) P(j,k) for i >= j (device pointers, column-major,
 * P n x k with k <= 64) through the same slice products. */
int sddd_Rsyrk_tc(sddd_ctx *ctx, long n, long k, const sddd_dd *P, long ldp, sddd_dd *C, long ldc, int slices);

/* -- bounded waits (no counterpart in the reference) --
 * Every device wait of the context's kernels (the triangular solves' waits
 * for another CTA's block, the split kernel's barrier waits) gives up after
 * `seconds` (default 2, range 1e-4..60): the kernel records the block or
 * barrier, lets its copies in flight land and returns, and the call that
 * launched it returns SDDD_ERR_CUDA naming it; the context stays usable. */
int sddd_set_wait_limit(sddd_ctx *ctx, double seconds);
/* Tests of that path: the triangular solves never publish the completion
 * flag of 64-entry block `block` (-1: publish all, the default), so every
 * wait for it runs out.  Not for production use. */
int sddd_test_withhold_block(sddd_ctx *ctx, int block);

/* C(i,j) = sum_k W(i,k) V(j,k) for i >= j (device pointers; W and V n x k
 * with row i at W + i * ldw, the k values contiguous; C column-major, only
 * its lower triangle written) through the split products: each row scaled
 * once over all k and cut into `slices` signed 7-bit slices, every diagonal
 * of slice products summed exactly in int32 on the tensor cores (k <= 32767),
 * rebuilt in dd.  The Schur complement's F1 pair products in the split form
 * (no counterpart in the reference). */
int sddd_Rdot_pairs_tc(sddd_ctx *ctx, long n, long k, const sddd_dd *W, long ldw, const sddd_dd *V, long ldv, sddd_dd *C, long ldc, int slices);

/* -- sparse Schur complement --
 * The reference keeps B dense unless the problem has more than 100
 * constraints, more than 5 blocks (SDP blocks + LP entries), no block that
 * touches more than half of the constraints, an aggregate pattern of at most
 * 0.25 m^2 entries and a factor of at most 0.4 m^2 entries
 * (Chordal::ordering_bMat, sdpa_chordal.cpp:348-438); then rows of B are
 * renumbered by a minimum-degree ordering and B is factored and solved in
 * sparse form (Lal::getCholesky(SparseMatrix&, int*), sdpa_linear.cpp:353-395;
 * Lal::solveSystems(Vector&, SparseMatrix&, Vector&), :654-810).  The
 * reference orders with SPOOLES's minimum degree, a library its sources do
 * not include; here the ordering is an exact minimum degree, ties to the
 * smallest constraint index.
 * mode: 0 the reference's thresholds (default), 1 always dense, 2 always
 * sparse (the reference's "SPARSE computation for debugging" thresholds,
 * sdpa_chordal.cpp:53-58).  Setting the mode re-plans an attached problem. */
int sddd_set_schur_mode(sddd_ctx *ctx, int mode);
typedef struct {
    int sparse;      /* 1: SPARSE computation, 0: DENSE computation */
    int m;
    long aggregate;  /* entries of the aggregate pattern, diagonal included */
    long extended;   /* 2 nnz(L) - m of the ordering (0 when not ordered) */
    long nnz;        /* entries of the factor's rows (sparse only) */
    long ntiles;     /* 64 x 64 tiles the device factor stores (sparse only) */
    char reason[96]; /* why B stayed dense */
} sddd_schur_info;
/* The attached problem's Schur form; with sparse, order[m] (new -> old
 * constraint), diagonalIndex[m + 1] and column_index[nnz] (the reference's
 * sparse_bMat layout: row b holds b, then the later rows of the factor's
 * column b, ascending) when the pointers are not NULL. */
int sddd_schur_form(const sddd_ctx *ctx, sddd_schur_info *out, int *order, int *diagonalIndex, int *column_index);
/* The same decision for a problem file, on the host only (no device). */
int sddd_plan_schur(const char *path, int sparse, int mode, sddd_schur_info *out, int *order, int *diagonalIndex, int *column_index);
/* The factor of the last sddd_schur_factor in that layout (host sp_ele[nnz];
 * the diagonal holds 1 / sqrt of the pivot, as the reference stores it). */
int sddd_sparse_factor_values(sddd_ctx *ctx, sddd_dd *sp_ele);
/* Lal::getCholesky(SparseMatrix&, int*) on a caller's matrix: structure on
 * the host (diagonalIndex[m + 1], column_index[nnz]; each row starts with its
 * diagonal, ascending, closed under elimination - anything else is
 * SDDD_ERR_ARG), sp_ele[nnz] on the device, factored in place.  Like the
 * reference it reports no failure: a negative pivot gives a zero row.  Use a
 * context without a problem. */
int sddd_sparse_getCholesky(sddd_ctx *ctx, int m, const int *diagonalIndex, const int *column_index, sddd_dd *sp_ele);
/* Lal::solveSystems(Vector&, SparseMatrix&, Vector&): x (device, m) <-
 * (L L^T)^-1 x for a factor from sddd_sparse_getCholesky (sp_ele device). */
int sddd_sparse_solveSystems(sddd_ctx *ctx, int m, const int *diagonalIndex, const int *column_index, const sddd_dd *sp_ele, sddd_dd *x);

/* -- dd kernels on device memory: the MPLAPACK seam --
 * The argument lists of MPLAPACK's dd routines (mplapack/mpblas_dd.h:47,54,
 * mplapack/mplapack_dd.h:41) with the context first; pointers are device
 * pointers to column-major sddd_dd, 16-byte aligned (a cudaMalloc'd base
 * plus whole sddd_dd; an unaligned base returns SDDD_ERR_ARG naming the
 * argument).  Bad arguments return SDDD_ERR_ARG
 * naming the routine and the 1-based position the reference's Mxerbla_dd
 * would report (in its order of checks); valid forms SDPA never calls
 * return SDDD_ERR_UNSUPPORTED.  Results are the reference's bit for bit
 * (with the tensor-core split off). */
/* Rgemm (mpblas_dd.h:54, mplapack/Rgemm_omp.cpp): C = alpha op(A) op(B)
 * + beta C, transa/transb 'N', 'T' or 'C'. */
int sddd_Rgemm(sddd_ctx *ctx, char transa, char transb, long m, long n, long k, sddd_dd alpha, const sddd_dd *A, long lda, const sddd_dd *B, long ldb,
               sddd_dd beta, sddd_dd *C, long ldc);
/* Rpotrf (mplapack_dd.h:41, mplapack/Rpotrf.cpp), uplo 'L': returns info
 * (0, or the 1-based column where A stopped being positive definite).
 * With the tensor-core split on, its trailing updates are slice products. */
int sddd_Rpotrf(sddd_ctx *ctx, char uplo, long n, sddd_dd *A, long lda);
/* Rtrsv (mpblas_dd.h:47, mplapack/Rtrsv.cpp), uplo 'L', trans 'N'/'T'/'C',
 * diag 'N', incx 1: x = op(A)^-1 x. */
int sddd_Rtrsv(sddd_ctx *ctx, char uplo, char trans, char diag, long n, const sddd_dd *A, long lda, sddd_dd *x, long incx);
/* Solve A X = B from the factor of sddd_Rpotrf (LAPACK's Rpotrs; the
 * reference's MPLAPACK subset has none, SDPA calls Rtrsv twice), uplo 'L',
 * nrhs columns of B.  Split off: the two Rtrsv of each column, bit for bit.
 * Split on: blocked solves with the 64 x 64 diagonal blocks of the factor
 * inverted once per call (no division on the critical path). */
int sddd_Rpotrs(sddd_ctx *ctx, char uplo, long n, long nrhs, const sddd_dd *A, long lda, sddd_dd *B, long ldb);
/* Elementwise dd operation on n device values: 0 a+b, 1 a+=b, 2/3 a-b,
 * 4 a*b, 5 a*=b, 6 a/b, 7 sqrt(a), 8 a*b.hi, 9 a+b.hi, 10 a-b.hi,
 * 11 a.hi-b, 12 a/b.hi, 13 a.hi/b, 14 -a, 15 |a|, 16 a^2, 17 a.hi+b.hi
 * (QD 2.3.23 dd_inline.h shapes).  ctx may be NULL. */
int sddd_dd_op(sddd_ctx *ctx, int op, long n, const sddd_dd *a, const sddd_dd *b, sddd_dd *out);

/* -- host-side dd (no GPU needed) -- */
/* The same operations on host arrays, as the host scalar control uses them. */
int sddd_host_dd_op(int op, long n, const sddd_dd *a, const sddd_dd *b, sddd_dd *out);
/* Decimal string -> dd as QD's dd_real::read (dd_real.cpp:1198). */
int sddd_host_dd_read(const char *s, sddd_dd *out);
/* QD's operator<< text with `precision` digits after the point. */
int sddd_host_dd_to_string(sddd_dd a, int precision, char *buf, int buflen);

#ifdef __cplusplus
}
#endif
#endif
