// extern "C" boundary (include/sddd.h) over the device solver.
#include "../../include/sddd.h"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>

#include "adjoint.h"
#include "blas.h"
#include "capi_internal.h"
#include "context.h"
#include "newton.h"
#include "prof.h"
#include "solver.h"
#include "sparse_chol.h"

struct sddd_ctx {
    std::unique_ptr<sddd::Context> c;
    std::unique_ptr<sddd::Solver> solver;
    std::unique_ptr<sddd::Profiler> prof;
    std::string err;
    int stop_reason = 0;
};

namespace {
thread_local std::string g_err;

template <class F>
int guarded(sddd_ctx *ctx, F &&f) {
    try {
        if (ctx && ctx->c) cudaSetDevice(ctx->c->device);
        return f();
    } catch (const sddd::Error &e) {
        if (ctx) ctx->err = e.what();
        g_err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        if (ctx) ctx->err = e.what();
        g_err = e.what();
        return SDDD_ERR_STATE;
    }
}

} // namespace

void sddd_set_thread_error(const char *msg) { g_err = msg ? msg : ""; }

namespace {

sddd::Context &need_problem(sddd_ctx *ctx) {
    if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
    if (!ctx->c->have_problem) throw sddd::Error(SDDD_ERR_STATE, "no problem uploaded");
    return *ctx->c;
}

sddd::Param to_param(const sddd_param *p) {
    sddd::Param q;
    q.maxIteration = p->maxIteration;
    q.epsilonStar = p->epsilonStar;
    q.lambdaStar = p->lambdaStar;
    q.omegaStar = p->omegaStar;
    q.lowerBound = p->lowerBound;
    q.upperBound = p->upperBound;
    q.betaStar = p->betaStar;
    q.betaBar = p->betaBar;
    q.gammaStar = p->gammaStar;
    q.epsilonDash = p->epsilonDash;
    return q;
}
void from_param(const sddd::Param &q, sddd_param *p) {
    p->maxIteration = q.maxIteration;
    p->epsilonStar = q.epsilonStar;
    p->lambdaStar = q.lambdaStar;
    p->omegaStar = q.omegaStar;
    p->lowerBound = q.lowerBound;
    p->upperBound = q.upperBound;
    p->betaStar = q.betaStar;
    p->betaBar = q.betaBar;
    p->gammaStar = q.gammaStar;
    p->epsilonDash = q.epsilonDash;
}
inline dd_t D(sddd_dd v) { return dd_make(v.hi, v.lo); }
inline sddd_dd S(dd_t v) { return sddd_dd{v.hi, v.lo}; }

void fill_result(sddd_ctx *ctx, sddd_result *out) { sddd_fill_result(*ctx->solver, ctx->stop_reason, out); }
} // namespace

void sddd_fill_result(const sddd::Solver &s, int stop_reason, sddd_result *out) {
    std::memset(out, 0, sizeof(*out));
    out->phase = (int)s.phase;
    out->iterations = s.pIteration;
    out->stop_reason = stop_reason;
    dd_t mean = dd_div_d(dd_add(dd_abs(s.objValPrimal), dd_abs(s.objValDual)), 2.0);
    dd_t gap = dd_abs(dd_sub(s.objValPrimal, s.objValDual));
    out->mu = S(s.mu_current);
    out->relative_gap = S(dd_lt_d(mean, 1.0) ? gap : dd_div(gap, mean));
    out->gap = S(dd_mul_d(s.mu_current, (double)s.c.nDim));
    out->objValPrimal = S(dd_neg(s.objValDual));
    out->objValDual = S(dd_neg(s.objValPrimal));
    out->pfeas_error = S(s.normDualMat);
    out->dfeas_error = S(s.normPrimalVec);
    out->main_loop_seconds = s.tm.mainLoop;
    out->schur_seconds = s.tm.makebMat;
    out->cholesky_seconds = s.tm.choleskybMat;
}

extern "C" {

const char *sddd_version(void) { return "sdpa-dd_b200 0.1 (sm_100a, dd on the FP64 pipe)"; }
const char *sddd_last_error(const sddd_ctx *ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int sddd_create(int device, sddd_ctx **out) {
    if (!out) return SDDD_ERR_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        auto *ctx = new sddd_ctx();
        ctx->c.reset(sddd::create_context(device));
        *out = ctx;
        return SDDD_OK;
    });
}

int sddd_destroy(sddd_ctx *ctx) {
    if (!ctx) return SDDD_OK;
    if (ctx->prof && sddd::g_prof == ctx->prof.get()) sddd::g_prof = nullptr;
    ctx->prof.reset();
    ctx->solver.reset();
    if (ctx->c) cudaSetDevice(ctx->c->device);
    ctx->c.reset();
    delete ctx;
    return SDDD_OK;
}

int sddd_param_default(int type, sddd_param *out) {
    if (!out || type < 0 || type > 2) return SDDD_ERR_ARG;
    from_param(sddd::default_param(type), out);
    return SDDD_OK;
}

int sddd_param_read(const char *path, sddd_param *out) {
    if (!path || !out) return SDDD_ERR_ARG;
    return guarded(nullptr, [&] {
        from_param(sddd::read_param(path), out);
        return SDDD_OK;
    });
}

int sddd_read_problem(sddd_ctx *ctx, const char *path, int sparse, double kappa) {
    if (!ctx || !path) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Problem p = sddd::read_problem(path, sparse != 0);
        sddd::finalize_problem(p, kappa);
        ctx->solver.reset();
        sddd::upload_problem(*ctx->c, std::move(p));
        return SDDD_OK;
    });
}

int sddd_upload_problem(sddd_ctx *ctx, int m, int nblock, const int *block_struct, const sddd_dd *b, long nnz, const int *k, const int *blk,
                        const int *i, const int *j, const sddd_dd *val, double kappa) {
    if (!ctx || !block_struct || !b || (nnz > 0 && (!k || !blk || !i || !j || !val))) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Problem p = sddd::make_problem(m, nblock, block_struct, reinterpret_cast<const dd_t *>(b), nnz, k, blk, i, j,
                                             reinterpret_cast<const dd_t *>(val));
        sddd::finalize_problem(p, kappa);
        ctx->solver.reset();
        sddd::upload_problem(*ctx->c, std::move(p));
        return SDDD_OK;
    });
}

int sddd_dims(const sddd_ctx *cctx, int *m, int *nsdp, long *ndim, int *sizes, int cap) {
    sddd_ctx *ctx = const_cast<sddd_ctx *>(cctx);
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (m) *m = c.m;
        if (nsdp) *nsdp = c.nSDP;
        if (ndim) *ndim = c.nDim;
        if (sizes)
            for (int l = 0; l < c.nSDP && l < cap; ++l) sizes[l] = c.sizes[l];
        return SDDD_OK;
    });
}

long sddd_space_len(const sddd_ctx *ctx) { return (ctx && ctx->c && ctx->c->have_problem) ? ctx->c->space_len : -1; }

int sddd_problem_info(const char *path, int sparse, int *m, int *nsdp, long *space_len, int *sizes, int cap) {
    if (!path) return SDDD_ERR_ARG;
    return guarded(nullptr, [&] {
        const sddd::Problem p = sddd::read_problem(path, sparse != 0);
        if (m) *m = p.m;
        if (nsdp) *nsdp = p.nSDP;
        long len = 0;
        for (int n : p.sdpSize) len += (long)n * n;
        if (space_len) *space_len = len;
        if (sizes)
            for (int l = 0; l < p.nSDP && l < cap; ++l) sizes[l] = p.sdpSize[l];
        return SDDD_OK;
    });
}

int sddd_formula(const sddd_ctx *cctx, int *out) {
    sddd_ctx *ctx = const_cast<sddd_ctx *>(cctx);
    if (!out) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        for (long q = 0; q < (long)c.m * c.nSDP; ++q) out[q] = -1;
        for (int l = 0; l < c.nSDP; ++l)
            for (size_t t = 0; t < c.prob.cons[l].size(); ++t) out[(long)c.prob.cons[l][t] * c.nSDP + l] = c.prob.formula[l][t];
        return SDDD_OK;
    });
}

int sddd_init_point(sddd_ctx *ctx, sddd_dd lambda) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::init_point(c, D(lambda));
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_set_point(sddd_ctx *ctx, const sddd_dd *X, const sddd_dd *y, const sddd_dd *Z) {
    if (!X || !y || !Z) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::space_from_host(c, c.X, reinterpret_cast<const dd_t *>(X));
        sddd::space_from_host(c, c.Z, reinterpret_cast<const dd_t *>(Z));
        CK(cudaMemcpyAsync(c.y.p, y, sizeof(dd_t) * c.m, cudaMemcpyHostToDevice, c.stream));
        return sddd::compute_inverse(c) ? SDDD_OK : 1;
    });
}

int sddd_get_point(sddd_ctx *ctx, sddd_dd *X, sddd_dd *y, sddd_dd *Z) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (X) sddd::space_to_host(c, c.X, reinterpret_cast<dd_t *>(X));
        if (Z) sddd::space_to_host(c, c.Z, reinterpret_cast<dd_t *>(Z));
        if (y) {
            CK(cudaMemcpyAsync(y, c.y.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToHost, c.stream));
            CK(cudaStreamSynchronize(c.stream));
        }
        return SDDD_OK;
    });
}

int sddd_compute_inverse(sddd_ctx *ctx) {
    return guarded(ctx, [&] { return sddd::compute_inverse(need_problem(ctx)) ? SDDD_OK : 1; });
}

int sddd_newton_rhs(sddd_ctx *ctx, int corrector, sddd_dd beta_mu, int dual_infeasible) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::make_rhs(c, corrector != 0, D(beta_mu), dual_infeasible != 0);
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_schur_build(sddd_ctx *ctx) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::schur_build(c);
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_schur_factor(sddd_ctx *ctx) {
    return guarded(ctx, [&] { return sddd::schur_factor(need_problem(ctx)); });
}

int sddd_solve_dy(sddd_ctx *ctx) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::solve_dy(c);
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_make_dz_dx(sddd_ctx *ctx, int dual_infeasible) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::make_dz_dx(c, dual_infeasible != 0);
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_min_eig(sddd_ctx *ctx, int which, sddd_dd *out) {
    if (!out || which < 0 || which > 1) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        *out = S(which == 0 ? sddd::min_eig(c, c.invCholX, c.Dx) : sddd::min_eig(c, c.invCholZ, c.Dz));
        return SDDD_OK;
    });
}

int sddd_update(sddd_ctx *ctx, sddd_dd ap, sddd_dd ad) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        sddd::update_point(c, D(ap), D(ad));
        return sddd::compute_inverse(c) ? SDDD_OK : 1;
    });
}

int sddd_residuals(sddd_ctx *ctx, sddd_dd *np, sddd_dd *nd) {
    return guarded(ctx, [&] {
        dd_t a, b;
        sddd::residuals(need_problem(ctx), a, b);
        if (np) *np = S(a);
        if (nd) *nd = S(b);
        return SDDD_OK;
    });
}

int sddd_inner(sddd_ctx *ctx, int which, sddd_dd *out) {
    if (!out) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        dd_t v;
        switch (which) {
        case 0: v = sddd::inner_C(c, c.X); break;
        case 1: v = sddd::inner_b(c, c.y.p); break;
        case 2: v = sddd::inner_space(c, c.X, c.Z); break;
        case 3: v = sddd::inner_C(c, c.Dx); break;
        case 4: v = sddd::inner_b(c, c.Dy.p); break;
        case 5: v = sddd::inner_space(c, c.X, c.Dz); break;
        case 6: v = sddd::inner_space(c, c.Dx, c.Z); break;
        case 7: v = sddd::inner_space(c, c.Dx, c.Dz); break;
        default: throw sddd::Error(SDDD_ERR_ARG, "unknown inner product");
        }
        *out = S(v);
        return SDDD_OK;
    });
}

static void *target_of(sddd::Context &c, int what, long &len) {
    const long L = c.space_len;
    switch (what) {
    case 0: len = L; return c.X.buf.p;
    case 1: len = L; return c.Z.buf.p;
    case 2: len = c.m; return c.y.p;
    case 3: len = L; return c.invCholX.buf.p;
    case 4: len = L; return c.invCholZ.buf.p;
    case 5: len = L; return c.invZ.buf.p;
    case 6: len = (long)c.m * c.m; return c.B.p;
    case 7: len = c.m; return c.g.p;
    case 8: len = L; return c.Dx.buf.p;
    case 9: len = c.m; return c.Dy.p;
    case 10: len = L; return c.Dz.buf.p;
    case 11: len = L; return c.dualMat.buf.p;
    case 12: len = c.m; return c.primalVec.p;
    case 13:
    case 14:
        if (!c.adj_valid) throw sddd::Error(SDDD_ERR_STATE, "no adjoint computed");
        if (what == 13) {
            len = c.m;
            return c.adj_u.p;
        }
        len = L;
        return c.adj_R.buf.p;
    default: throw sddd::Error(SDDD_ERR_ARG, "unknown array selector");
    }
}

long sddd_get(sddd_ctx *ctx, int what, sddd_dd *out) {
    long result = 0;
    int rc = guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        long len = 0;
        void *p = target_of(c, what, len);
        if (out) {
            CK(cudaMemcpyAsync(out, p, sizeof(dd_t) * len, cudaMemcpyDeviceToHost, c.stream));
            CK(cudaStreamSynchronize(c.stream));
        }
        result = len;
        return SDDD_OK;
    });
    return rc == SDDD_OK ? result : rc;
}

int sddd_set(sddd_ctx *ctx, int what, const sddd_dd *in) {
    if (!in) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        long len = 0;
        void *p = target_of(c, what, len);
        CK(cudaMemcpyAsync(p, in, sizeof(dd_t) * len, cudaMemcpyHostToDevice, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

static void store_init(sddd::Context &c, const dd_t *X, const dd_t *y, const dd_t *Z) {
    c.init_X.buf.alloc(c.space_len);
    c.init_Z.buf.alloc(c.space_len);
    c.init_y.alloc(c.m);
    sddd::space_from_host(c, c.init_X, X);
    sddd::space_from_host(c, c.init_Z, Z);
    CK(cudaMemcpyAsync(c.init_y.p, y, sizeof(dd_t) * c.m, cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.has_init = true;
}

int sddd_read_initial_point(sddd_ctx *ctx, const char *path, int sparse, double lambda) {
    if (!path) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        std::vector<dd_t> X, y, Z;
        sddd::read_init_point(path, sparse != 0, c.prob, lambda, X, y, Z);
        store_init(c, X.data(), y.data(), Z.data());
        return SDDD_OK;
    });
}

int sddd_set_initial_point(sddd_ctx *ctx, const sddd_dd *x, const sddd_dd *X, const sddd_dd *Y) {
    if (!x || !X || !Y) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        std::vector<dd_t> y(c.m);
        for (int k = 0; k < c.m; ++k) y[k] = dd_neg(D(x[k])); // the internal y is -x
        // the internal X is the file's Y, the internal Z its X
        store_init(c, reinterpret_cast<const dd_t *>(Y), y.data(), reinterpret_cast<const dd_t *>(X));
        return SDDD_OK;
    });
}

int sddd_write_point(sddd_ctx *ctx, const char *path, int sparse) {
    if (!path) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        std::vector<dd_t> X(c.space_len), Z(c.space_len), y(c.m);
        sddd::space_to_host(c, c.X, X.data());
        sddd::space_to_host(c, c.Z, Z.data());
        CK(cudaMemcpyAsync(y.data(), c.y.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        const std::string text = sddd::write_init_point_text(c.prob, X, y, Z, sparse != 0);
        FILE *f = std::fopen(path, "wb");
        if (!f) throw sddd::Error(SDDD_ERR_IO, std::string("cannot open ") + path);
        const size_t w = std::fwrite(text.data(), 1, text.size(), f);
        const int rc = std::fclose(f);
        if (w != text.size() || rc != 0) throw sddd::Error(SDDD_ERR_IO, std::string("cannot write ") + path);
        return SDDD_OK;
    });
}

int sddd_dd_to_decimal(sddd_dd v, int digits, char *buf, int len) {
    if (!buf || len <= 0 || digits < 1 || digits > 60) return SDDD_ERR_ARG;
    return guarded(nullptr, [&] {
        const std::string s = sddd::dd_to_decimal(D(v), digits);
        const int n = (int)std::min<size_t>(s.size(), (size_t)len - 1);
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
        return (int)s.size();
    });
}

int sddd_clear_initial_point(sddd_ctx *ctx) {
    return guarded(ctx, [&] {
        need_problem(ctx).has_init = false;
        return SDDD_OK;
    });
}

int sddd_adjoint(sddd_ctx *ctx, const sddd_dd *g_x, const sddd_dd *g_Y, const sddd_dd *g_X, sddd_dd g_obj, sddd_dd *grad_c, sddd_dd *grad_F0) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        const int info = sddd::adjoint_combined(c, reinterpret_cast<const dd_t *>(g_x), reinterpret_cast<const dd_t *>(g_Y),
                                                reinterpret_cast<const dd_t *>(g_X), D(g_obj));
        if (info != 0) return info;
        if (grad_c) {
            sddd::adjoint_grad_c(c, D(g_obj), c.adj_v.p);
            CK(cudaMemcpyAsync(grad_c, c.adj_v.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToHost, c.stream));
        }
        if (grad_F0) {
            sddd::adjoint_grad_F0(c, c.adj_T.buf.p);
            sddd::space_to_host(c, c.adj_T, reinterpret_cast<dd_t *>(grad_F0));
        }
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_adjoint_grad_F(sddd_ctx *ctx, int k, sddd_dd *grad_Fk) {
    if (!grad_Fk) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (!c.adj_valid) throw sddd::Error(SDDD_ERR_STATE, "no adjoint computed");
        if (k < 1 || k > c.m) throw sddd::Error(SDDD_ERR_ARG, "constraint index out of range");
        sddd::adjoint_grad_F(c, k - 1, c.adj_T.buf.p);
        sddd::space_to_host(c, c.adj_T, reinterpret_cast<dd_t *>(grad_Fk));
        return SDDD_OK;
    });
}

int sddd_solver_start(sddd_ctx *ctx, const sddd_param *param) {
    if (!param) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        ctx->solver.reset(new sddd::Solver(c, to_param(param)));
        ctx->solver->start();
        ctx->stop_reason = 0;
        return SDDD_OK;
    });
}

int sddd_iterate(sddd_ctx *ctx) {
    return guarded(ctx, [&] {
        if (!ctx->solver) throw sddd::Error(SDDD_ERR_STATE, "solver not started");
        int rc = ctx->solver->step(nullptr, nullptr);
        if (rc != 0) ctx->stop_reason = rc;
        return rc;
    });
}

int sddd_solver_result(sddd_ctx *ctx, sddd_result *out) {
    if (!out) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->solver) throw sddd::Error(SDDD_ERR_STATE, "solver not started");
        fill_result(ctx, out);
        return SDDD_OK;
    });
}

int sddd_solve(sddd_ctx *ctx, const sddd_param *param, const char *result_path, int print, sddd_result *out) {
    if (!param) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        FILE *fo = nullptr;
        if (result_path) {
            fo = std::fopen(result_path, "w");
            if (!fo) throw sddd::Error(SDDD_ERR_IO, std::string("Cannot open out file ") + result_path);
        }
        FILE *disp = print ? stdout : nullptr;
        const auto t0 = std::chrono::steady_clock::now();
        ctx->solver.reset(new sddd::Solver(c, to_param(param)));
        sddd::Solver &s = *ctx->solver;
        s.start();
        if (fo) std::fprintf(fo, "   mu      thetaP  thetaD  objP      objD      alphaP  alphaD  beta \n");
        if (disp) std::fprintf(disp, "   mu      thetaP  thetaD  objP      objD      alphaP  alphaD  beta \n");
        int rc = 0;
        while ((rc = s.step(disp, fo)) == 0) {
        }
        ctx->stop_reason = rc;
        s.finish();
        const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        s.tm.total = total;
        s.print_last_info(disp, fo, total, "");
        if (fo) std::fclose(fo);
        if (out) fill_result(ctx, out);
        return SDDD_OK;
    });
}

unsigned long long sddd_launch_count(void) { return sddd::g_launches.load(); }

void *sddd_stream(sddd_ctx *ctx) { return (ctx && ctx->c) ? (void *)ctx->c->stream : nullptr; }

int sddd_profile(sddd_ctx *ctx, int enable) {
    if (!ctx || !ctx->c) return SDDD_ERR_ARG;
    if (enable) {
        if (!ctx->prof) ctx->prof.reset(new sddd::Profiler());
        sddd::g_prof = ctx->prof.get();
    } else if (sddd::g_prof == ctx->prof.get()) {
        sddd::g_prof = nullptr;
    }
    return SDDD_OK;
}

int sddd_profile_read(sddd_ctx *ctx, const char *name, double *ms, long *launches) {
    if (!ctx || !ctx->c || !name) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->prof) {
            if (ms) *ms = 0;
            if (launches) *launches = 0;
            return SDDD_OK;
        }
        ctx->prof->collect(ctx->c->stream);
        auto it = ctx->prof->totals.find(name);
        if (ms) *ms = it == ctx->prof->totals.end() ? 0.0 : it->second.first;
        if (launches) *launches = it == ctx->prof->totals.end() ? 0 : it->second.second;
        return SDDD_OK;
    });
}

int sddd_profile_reset(sddd_ctx *ctx) {
    if (!ctx || !ctx->c) return SDDD_ERR_ARG;
    if (ctx->prof) {
        ctx->prof->collect(ctx->c->stream);
        ctx->prof->totals.clear();
    }
    return SDDD_OK;
}

int sddd_work(const sddd_ctx *cctx, double *schur_ddflops, double *chol_ddflops) {
    sddd_ctx *ctx = const_cast<sddd_ctx *>(cctx);
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (schur_ddflops) *schur_ddflops = c.schur_flops;
        if (chol_ddflops) *chol_ddflops = c.chol_flops;
        return SDDD_OK;
    });
}

namespace {
inline char up(char c) { return (c >= 'a' && c <= 'z') ? (char)(c - 'a' + 'A') : c; }
inline dd_t from(sddd_dd v) { return dd_t{v.hi, v.lo}; }
// MPLAPACK's argument errors (Mxerbla_dd: the routine's name and the
// 1-based position of the first bad argument) as an SDDD_ERR_ARG.
[[noreturn]] void bad_arg(const char *routine, int pos, const char *what) {
    throw sddd::Error(SDDD_ERR_ARG, std::string(routine) + ": parameter " + std::to_string(pos) + " (" + what + ") is invalid");
}
// Device matrices are read and written as 16-byte dd pairs (and staged
// with bulk copies), so their base must be 16-byte aligned.
void need_aligned(const char *routine, int pos, const char *what, const void *p) {
    if (p && (reinterpret_cast<uintptr_t>(p) & 15u) != 0) bad_arg(routine, pos, (std::string(what) + ", not 16-byte aligned").c_str());
}
} // namespace

int sddd_Rgemm(sddd_ctx *ctx, char transa, char transb, long m, long n, long k, sddd_dd alpha, const sddd_dd *A, long lda, const sddd_dd *B, long ldb,
               sddd_dd beta, sddd_dd *C, long ldc) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        const char ta = up(transa), tb = up(transb);
        const bool nota = ta == 'N', notb = tb == 'N';
        const long nrowa = nota ? m : k, nrowb = notb ? k : n;
        // the checks and their order of mplapack/Rgemm_omp.cpp
        if (!nota && ta != 'C' && ta != 'T') bad_arg("Rgemm", 1, "transa");
        if (!notb && tb != 'C' && tb != 'T') bad_arg("Rgemm", 2, "transb");
        if (m < 0) bad_arg("Rgemm", 3, "m");
        if (n < 0) bad_arg("Rgemm", 4, "n");
        if (k < 0) bad_arg("Rgemm", 5, "k");
        if (lda < std::max(1L, nrowa)) bad_arg("Rgemm", 8, "lda");
        if (ldb < std::max(1L, nrowb)) bad_arg("Rgemm", 10, "ldb");
        if (ldc < std::max(1L, m)) bad_arg("Rgemm", 13, "ldc");
        need_aligned("Rgemm", 7, "A", A);
        need_aligned("Rgemm", 9, "B", B);
        need_aligned("Rgemm", 12, "C", C);
        sddd::gemm_ab(ctx->c->stream, nota ? 'N' : 'T', notb ? 'N' : 'T', (int)m, (int)n, (int)k, from(alpha), reinterpret_cast<const dd_t *>(A), lda,
                      reinterpret_cast<const dd_t *>(B), ldb, from(beta), reinterpret_cast<dd_t *>(C), ldc);
        CK(cudaStreamSynchronize(ctx->c->stream));
        return SDDD_OK;
    });
}

int sddd_Rpotrf(sddd_ctx *ctx, char uplo, long n, sddd_dd *A, long lda) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        const char u = up(uplo);
        if (u != 'L' && u != 'U') bad_arg("Rpotrf", 1, "uplo");
        if (n < 0) bad_arg("Rpotrf", 2, "n");
        if (lda < std::max(1L, n)) bad_arg("Rpotrf", 4, "lda");
        need_aligned("Rpotrf", 3, "A", A);
        if (u == 'U') throw sddd::Error(SDDD_ERR_UNSUPPORTED, "Rpotrf: only uplo = 'L' (the form SDPA calls) is implemented");
        if (n == 0) return SDDD_OK;
        sddd::Context &c = *ctx->c;
        if (!c.info.p) c.info.alloc(4);
        if (!c.rdiag.p) c.rdiag.alloc(256);
        CK(cudaMemsetAsync(c.info.p, 0, sizeof(int), c.stream));
        sddd::OzakiWork *tc = c.tc_slices > 0 ? &sddd::tc_work(c, (int)n, c.tc_slices) : nullptr;
        sddd::potrf(c.stream, reinterpret_cast<dd_t *>(A), lda, (int)n, c.info.p, c.rdiag.p, tc);
        int info = 0;
        CK(cudaMemcpyAsync(&info, c.info.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        if (tc) sddd::ozaki_check(c.stream, *tc);
        return sddd::potrf_info_check(info);
    });
}

int sddd_set_wait_limit(sddd_ctx *ctx, double seconds) {
    if (!ctx || !ctx->c) return SDDD_ERR_ARG;
    if (!(seconds >= 1e-4 && seconds <= 60.0)) {
        ctx->err = "sddd_set_wait_limit: seconds must lie in [1e-4, 60]";
        return SDDD_ERR_ARG;
    }
    ctx->c->wait_ns = (unsigned long long)(seconds * 1e9);
    return SDDD_OK;
}

int sddd_test_withhold_block(sddd_ctx *ctx, int block) {
    if (!ctx || !ctx->c || block < -1) return SDDD_ERR_ARG;
    ctx->c->withhold_block = block;
    return SDDD_OK;
}

int sddd_set_tc_split(sddd_ctx *ctx, int slices) {
    if (!ctx || !ctx->c) return SDDD_ERR_ARG;
    if (slices != 0 && (slices < 8 || slices > sddd::OZ_MAX_SLICES)) {
        ctx->err = "sddd_set_tc_split: slices must be 0 (off) or 8..16";
        return SDDD_ERR_ARG;
    }
    ctx->c->tc_slices = slices;
    return SDDD_OK;
}

int sddd_get_tc_split(const sddd_ctx *ctx) { return (ctx && ctx->c) ? ctx->c->tc_slices : SDDD_ERR_ARG; }

int sddd_Rsyrk_tc(sddd_ctx *ctx, long n, long k, const sddd_dd *P, long ldp, sddd_dd *C, long ldc, int slices) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        if (n < 0 || k < 0 || k > sddd::OZ_K || ldp < std::max(1L, n) || ldc < std::max(1L, n) || slices < 8 || slices > sddd::OZ_MAX_SLICES)
            throw sddd::Error(SDDD_ERR_ARG, "sddd_Rsyrk_tc: need 0 <= k <= 64, ld >= n and 8 <= slices <= 16");
        need_aligned("sddd_Rsyrk_tc", 3, "P", P);
        need_aligned("sddd_Rsyrk_tc", 5, "C", C);
        if (n == 0 || k == 0) return SDDD_OK;
        sddd::Context &c = *ctx->c;
        sddd::OzakiWork &w = sddd::tc_work(c, (int)n, slices);
        sddd::ozaki_syrk_sub_lower(c.stream, reinterpret_cast<const dd_t *>(P), ldp, (int)n, (int)k, reinterpret_cast<dd_t *>(C), ldc, w);
        sddd::ozaki_check(c.stream, w);
        if (c.tc_slices > 0) c.tc.slices_used = c.tc_slices;
        return SDDD_OK;
    });
}

int sddd_Rdot_pairs_tc(sddd_ctx *ctx, long n, long k, const sddd_dd *W, long ldw, const sddd_dd *V, long ldv, sddd_dd *C, long ldc, int slices) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        if (n < 0 || k < 1 || k > sddd::OG_MAX_K || ldw < k || ldv < k || ldc < std::max(1L, n) || slices < 8 || slices > sddd::OZ_MAX_SLICES)
            throw sddd::Error(SDDD_ERR_ARG, "sddd_Rdot_pairs_tc: need 1 <= k <= 32767, ldw, ldv >= k, ldc >= n and 8 <= slices <= 16");
        need_aligned("sddd_Rdot_pairs_tc", 3, "W", W);
        need_aligned("sddd_Rdot_pairs_tc", 5, "V", V);
        need_aligned("sddd_Rdot_pairs_tc", 7, "C", C);
        if (n == 0) return SDDD_OK;
        sddd::Context &c = *ctx->c;
        sddd::OzakiGemmWork &w = sddd::tcg_work(c, (int)n, k, slices);
        sddd::ozaki_gemm_lower(c.stream, reinterpret_cast<const dd_t *>(W), ldw, reinterpret_cast<const dd_t *>(V), ldv, (int)n, k,
                               reinterpret_cast<dd_t *>(C), ldc, w);
        sddd::ozaki_gemm_check(c.stream, w);
        return SDDD_OK;
    });
}

int sddd_Rtrsv(sddd_ctx *ctx, char uplo, char trans, char diag, long n, const sddd_dd *A, long lda, sddd_dd *x, long incx) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        const char u = up(uplo), t = up(trans), d = up(diag);
        // the checks and their order of mplapack/Rtrsv.cpp
        if (u != 'U' && u != 'L') bad_arg("Rtrsv", 1, "uplo");
        if (t != 'N' && t != 'T' && t != 'C') bad_arg("Rtrsv", 2, "trans");
        if (d != 'U' && d != 'N') bad_arg("Rtrsv", 3, "diag");
        if (n < 0) bad_arg("Rtrsv", 4, "n");
        if (lda < std::max(1L, n)) bad_arg("Rtrsv", 6, "lda");
        if (incx == 0) bad_arg("Rtrsv", 8, "incx");
        need_aligned("Rtrsv", 5, "A", A);
        need_aligned("Rtrsv", 7, "x", x);
        if (u != 'L' || d != 'N' || incx != 1)
            throw sddd::Error(SDDD_ERR_UNSUPPORTED, "Rtrsv: only uplo = 'L', diag = 'N', incx = 1 (the form SDPA calls) is implemented");
        if (n == 0) return SDDD_OK;
        sddd::TrsvSync &sync = sddd::trsv_sync(*ctx->c, (int)n);
        sddd::trsv_lower(ctx->c->stream, t == 'N' ? 'N' : 'T', reinterpret_cast<const dd_t *>(A), lda, (int)n, reinterpret_cast<dd_t *>(x), sync);
        sddd::trsv_check(ctx->c->stream, sync);
        return SDDD_OK;
    });
}

int sddd_Rpotrs(sddd_ctx *ctx, char uplo, long n, long nrhs, const sddd_dd *A, long lda, sddd_dd *B, long ldb) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        const char u = up(uplo);
        if (u != 'L' && u != 'U') bad_arg("Rpotrs", 1, "uplo");
        if (n < 0) bad_arg("Rpotrs", 2, "n");
        if (nrhs < 0) bad_arg("Rpotrs", 3, "nrhs");
        if (lda < std::max(1L, n)) bad_arg("Rpotrs", 5, "lda");
        if (ldb < std::max(1L, n)) bad_arg("Rpotrs", 7, "ldb");
        need_aligned("Rpotrs", 4, "A", A);
        need_aligned("Rpotrs", 6, "B", B);
        if (u == 'U') throw sddd::Error(SDDD_ERR_UNSUPPORTED, "Rpotrs: only uplo = 'L' is implemented");
        if (n == 0 || nrhs == 0) return SDDD_OK;
        sddd::Context &c = *ctx->c;
        const dd_t *L = reinterpret_cast<const dd_t *>(A);
        sddd::TrsvSync &sync = sddd::trsv_sync(c, (int)n);
        if (c.tc_slices > 0) {
            // the split form's blocked solves; the inverted diagonal blocks
            // take the context's buffer (a Newton solve in progress
            // recomputes them at its next factorisation)
            c.winv_valid = false;
            c.trsv_winv.alloc((size_t)sddd::ceil_div(n, 64L) * 64 * 64);
            sddd::trsv_diag_inverse(c.stream, L, lda, (int)n, c.trsv_winv.p);
            for (long r = 0; r < nrhs; ++r) {
                dd_t *x = reinterpret_cast<dd_t *>(B) + ldb * r;
                sddd::trsv_blocked(c.stream, 'N', L, lda, (int)n, c.trsv_winv.p, x, sync);
                sddd::trsv_blocked(c.stream, 'T', L, lda, (int)n, c.trsv_winv.p, x, sync);
            }
        } else {
            for (long r = 0; r < nrhs; ++r) {
                dd_t *x = reinterpret_cast<dd_t *>(B) + ldb * r;
                sddd::trsv_lower(c.stream, 'N', L, lda, (int)n, x, sync);
                sddd::trsv_lower(c.stream, 'T', L, lda, (int)n, x, sync);
            }
        }
        sddd::trsv_check(c.stream, sync);
        return SDDD_OK;
    });
}

} // extern "C"

// ---------------------------------------------------------------- CLI glue
// (C++ linkage: used by cli.cpp only)
void sddd_attach_problem(sddd_ctx *ctx, sddd::Problem &&p) {
    ctx->solver.reset();
    sddd::upload_problem(*ctx->c, std::move(p));
}

int sddd_solve_stream(sddd_ctx *ctx, const sddd_param *param, FILE *disp, FILE *fo, double fileRead, double *mainLoop) {
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        const auto t0 = std::chrono::steady_clock::now();
        ctx->solver.reset(new sddd::Solver(c, to_param(param)));
        sddd::Solver &s = *ctx->solver;
        s.start();
        s.tm.fileRead = fileRead;
        if (fo) std::fprintf(fo, "   mu      thetaP  thetaD  objP      objD      alphaP  alphaD  beta \n");
        if (disp) std::fprintf(disp, "   mu      thetaP  thetaD  objP      objD      alphaP  alphaD  beta \n");
        int rc = 0;
        const auto tl = std::chrono::steady_clock::now();
        while ((rc = s.step(disp, fo)) == 0) {
        }
        const double ml = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
        ctx->stop_reason = rc;
        s.finish();
        s.tm.mainLoop = ml;
        const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() + fileRead;
        s.tm.total = total;
        s.print_last_info(disp, fo, total, "");
        if (mainLoop) *mainLoop = ml;
        return SDDD_OK;
    });
}

// ----------------------------------------------------- sparse Schur form
namespace {
void fill_form(const sddd::SparsePlan &pl, const sddd::TileSchedule *t, int m, sddd_schur_info *out, int *order, int *diagonalIndex, int *column_index) {
    if (out) {
        out->sparse = pl.sparse ? 1 : 0;
        out->m = m;
        out->aggregate = pl.aggregate;
        out->extended = pl.extended;
        out->nnz = pl.sparse ? pl.s.nnz() : 0;
        out->ntiles = (pl.sparse && t) ? t->ntiles : 0;
        std::snprintf(out->reason, sizeof(out->reason), "%s", pl.sparse ? "" : pl.dense_reason);
    }
    if (!pl.sparse) return;
    if (order) std::copy(pl.order.begin(), pl.order.end(), order);
    if (diagonalIndex) std::copy(pl.s.rowptr.begin(), pl.s.rowptr.end(), diagonalIndex);
    if (column_index) std::copy(pl.s.col.begin(), pl.s.col.end(), column_index);
}

sddd::SparseStructure structure_from(int m, const int *diagonalIndex, const int *column_index) {
    if (m < 0 || !diagonalIndex || (m > 0 && !column_index)) throw sddd::Error(SDDD_ERR_ARG, "sparse factor: m >= 0 and the structure arrays are required");
    sddd::SparseStructure s;
    s.m = m;
    s.rowptr.assign(diagonalIndex, diagonalIndex + m + 1);
    if (s.rowptr[m] < 0) throw sddd::Error(SDDD_ERR_ARG, "sparse factor: diagonalIndex[m] is negative");
    s.col.assign(column_index, column_index + s.rowptr[m]);
    return s;
}

// Sets the context's tiles up for a caller's structure, reusing the last one
// when it is the same.
void use_structure(sddd::Context &c, const sddd::SparseStructure &s) {
    if (c.sp && c.sp->active && c.sp->plan.s.m == s.m && c.sp->plan.s.rowptr == s.rowptr && c.sp->plan.s.col == s.col && !c.have_problem) return;
    if (c.have_problem) throw sddd::Error(SDDD_ERR_STATE, "sparse factor: the context holds a problem; use a context of its own");
    sddd::sparse_setup_structure(c, s);
}
} // namespace

int sddd_set_schur_mode(sddd_ctx *ctx, int mode) {
    if (!ctx || !ctx->c || mode < 0 || mode > 2) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = *ctx->c;
        c.schur_mode = mode;
        if (c.have_problem) {
            ctx->solver.reset();
            sddd::sparse_setup(c);
            c.chol_flops = c.sparse_active() ? 2.0 * (double)c.sp->sched.exact_terms : (double)c.m * c.m * c.m / 3.0;
        }
        return SDDD_OK;
    });
}

int sddd_schur_form(const sddd_ctx *cctx, sddd_schur_info *out, int *order, int *diagonalIndex, int *column_index) {
    sddd_ctx *ctx = const_cast<sddd_ctx *>(cctx);
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (!c.sp) throw sddd::Error(SDDD_ERR_STATE, "no Schur form planned");
        fill_form(c.sp->plan, &c.sp->sched, c.m, out, order, diagonalIndex, column_index);
        return SDDD_OK;
    });
}

int sddd_plan_schur(const char *path, int sparse, int mode, sddd_schur_info *out, int *order, int *diagonalIndex, int *column_index) {
    if (!path || mode < 0 || mode > 2) return SDDD_ERR_ARG;
    return guarded(nullptr, [&] {
        sddd::Problem p = sddd::read_problem(path, sparse != 0);
        sddd::finalize_problem(p, 1.2);
        const sddd::SparsePlan pl = sddd::plan_schur(p, mode);
        if (pl.sparse) {
            const sddd::TileSchedule t = sddd::make_tile_schedule(pl.s);
            fill_form(pl, &t, p.m, out, order, diagonalIndex, column_index);
        } else {
            fill_form(pl, nullptr, p.m, out, order, diagonalIndex, column_index);
        }
        return SDDD_OK;
    });
}

int sddd_sparse_factor_values(sddd_ctx *ctx, sddd_dd *sp_ele) {
    if (!sp_ele) return SDDD_ERR_ARG;
    return guarded(ctx, [&] {
        sddd::Context &c = need_problem(ctx);
        if (!c.sparse_active()) throw sddd::Error(SDDD_ERR_STATE, "the Schur matrix is dense");
        const long nnz = c.sp->plan.s.nnz();
        sddd::DBuf<dd_t> tmp;
        tmp.alloc((size_t)std::max(1L, nnz));
        sddd::sparse_values(c, tmp.p);
        CK(cudaMemcpyAsync(sp_ele, tmp.p, sizeof(dd_t) * nnz, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_sparse_getCholesky(sddd_ctx *ctx, int m, const int *diagonalIndex, const int *column_index, sddd_dd *sp_ele) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        sddd::Context &c = *ctx->c;
        const sddd::SparseStructure s = structure_from(m, diagonalIndex, column_index);
        if (m == 0) return SDDD_OK;
        if (!sp_ele) throw sddd::Error(SDDD_ERR_ARG, "sparse factor: sp_ele is required");
        use_structure(c, s);
        sddd::sparse_factor_values(c, reinterpret_cast<const dd_t *>(sp_ele));
        sddd::sparse_values(c, reinterpret_cast<dd_t *>(sp_ele));
        CK(cudaStreamSynchronize(c.stream));
        return SDDD_OK;
    });
}

int sddd_sparse_solveSystems(sddd_ctx *ctx, int m, const int *diagonalIndex, const int *column_index, const sddd_dd *sp_ele, sddd_dd *x) {
    return guarded(ctx, [&] {
        if (!ctx || !ctx->c) throw sddd::Error(SDDD_ERR_ARG, "null context");
        sddd::Context &c = *ctx->c;
        const sddd::SparseStructure s = structure_from(m, diagonalIndex, column_index);
        if (m == 0) return SDDD_OK;
        if (!sp_ele || !x) throw sddd::Error(SDDD_ERR_ARG, "sparse solve: sp_ele and x are required");
        use_structure(c, s);
        sddd::sparse_load_values(c, reinterpret_cast<const dd_t *>(sp_ele));
        sddd::sparse_solve_raw(c, reinterpret_cast<dd_t *>(x));
        return SDDD_OK;
    });
}
