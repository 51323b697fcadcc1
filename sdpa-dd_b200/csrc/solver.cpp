// Interior-point driver and scalar control (see solver.h).  Every dd
// expression below is written in the operand order and with the operator
// shapes (operator+, +=, -, *, *=, /) of the reference line it cites.
#include "solver.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "batched.h"
#include "newton.h"

namespace sddd {

static const dd_t ZERO = {0.0, 0.0};
static const dd_t ONE = {1.0, 0.0};

// std::max / std::min as the reference's calls resolve (using namespace std)
static dd_t smax(dd_t a, dd_t b) { return dd_lt(a, b) ? b : a; }
static dd_t smin(dd_t a, dd_t b) { return dd_lt(b, a) ? b : a; }

namespace {
// Phase timing with CUDA events on the solver stream; elapsed times are
// read after the next stream synchronisation.
struct EvSpan {
    cudaEvent_t a = nullptr, b = nullptr;
    double *acc = nullptr;
};
struct EvClock {
    Context &c;
    cudaStream_t st;
    std::vector<EvSpan> pending;
    std::vector<cudaEvent_t> owned;
    explicit EvClock(Context &ctx) : c(ctx), st(ctx.stream) {}
    ~EvClock() {
        for (auto e : owned) cudaEventDestroy(e);
    }
    cudaEvent_t mark() {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        owned.push_back(e);
        CK(cudaEventRecord(e, st));
        return e;
    }
    void span(cudaEvent_t a, cudaEvent_t b, double *acc) { pending.push_back({a, b, acc}); }
    void collect() {
        stream_sync(c);
        for (auto &p : pending) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, p.a, p.b));
            *p.acc += ms * 1e-3;
        }
        pending.clear();
    }
};
} // namespace

Solver::Solver(Context &ctx, const Param &p) : c(ctx), param(p) {}

// Phase::updateCheck (sdpa_parts.cpp:875-954)
bool Solver::phase_update_check() {
    const dd_t NONZERO = dd_from(1.0e-6);
    const dd_t accuracy = dd_from(param.epsilonDash);
    phase = noINFO;
    if (dd_le(normPrimalVec, accuracy)) {
        if (dd_le(normDualMat, accuracy))
            phase = pdFEAS;
        else
            phase = pFEAS;
    }
    if (phase == noINFO && dd_le(normDualMat, accuracy)) phase = dFEAS;
    if (phase == pdFEAS) {
        dd_t mean = dd_div_d(dd_add(dd_abs(objValPrimal), dd_abs(objValDual)), 2.0);
        dd_t PDgap = dd_abs(dd_sub(objValPrimal, objValDual));
        dd_t dominator = dd_lt_d(mean, 1.0) ? ONE : mean;
        if (dd_le_d(dd_div(PDgap, dominator), param.epsilonStar)) {
            phase = pdOPT;
            return false;
        }
    }
    const dd_t onePlus = dd_add_d(NONZERO, 1.0);
    if (phase == noINFO && dd_gt(rho, onePlus)) {
        phase = pdINF;
        return false;
    }
    if (phase == pFEAS) {
        if (dd_le_d(objValPrimal, -param.upperBound)) {
            phase = pUNBD;
            return false;
        }
        if (dd_gt(rho, onePlus)) {
            phase = pFEAS_dINF;
            return false;
        }
    }
    if (phase == dFEAS) {
        if (dd_ge_d(objValDual, -param.lowerBound)) {
            phase = dUNBD;
            return false;
        }
        if (dd_gt(rho, onePlus)) {
            phase = pINF_dFEAS;
            return false;
        }
    }
    return true;
}

// Phase::reverse (sdpa_parts.cpp:956-992)
void Solver::phase_reverse() {
    switch (phase) {
    case pFEAS: phase = dFEAS; break;
    case dFEAS: phase = pFEAS; break;
    case pFEAS_dINF: phase = pINF_dFEAS; break;
    case pINF_dFEAS: phase = pFEAS_dINF; break;
    case pUNBD: phase = dUNBD; break;
    case dUNBD: phase = pUNBD; break;
    default: break;
    }
}

const char *phase_name(PhaseType p) {
    static const char *names[] = {"noINFO    ", "pFEAS     ", "dFEAS     ", "pdFEAS    ", "pdINF     ", "pFEAS_dINF", "pINF_dFEAS", "pdOPT     ", "pUNBD     ", "dUNBD     "};
    if (p < 0 || p > dUNBD) return "phase error";
    return names[p];
}

// Solutions::initialize + Residuals + the scalar objects of pinpal
// (sdpa_main.cpp:229-282)
void Solver::start() {
    const dd_t lambda = dd_from(param.lambdaStar);
    if (c.has_init) {
        // an initial point file (sdpa_main.cpp:237-251, 276-278):
        // computeInverse, then AverageComplementarity::initialize(Solutions)
        const size_t bytes = sizeof(dd_t) * c.space_len;
        CK(cudaMemcpyAsync(c.X.buf.p, c.init_X.buf.p, bytes, cudaMemcpyDeviceToDevice, c.stream));
        CK(cudaMemcpyAsync(c.Z.buf.p, c.init_Z.buf.p, bytes, cudaMemcpyDeviceToDevice, c.stream));
        CK(cudaMemcpyAsync(c.y.p, c.init_y.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToDevice, c.stream));
        if (!compute_inverse(c)) throw Error(ERR_ARG, "the initial point is not positive definite (cholesky of X or Z failed)");
        mu_initial = dd_div_d(inner_space(c, c.X, c.Z), (double)c.nDim);
    } else {
        init_point(c, lambda);
        mu_initial = dd_mul(lambda, lambda);
    }
    residuals(c, normPrimalVec, normDualMat);
    initNormPrimalVec = normPrimalVec;
    initNormDualMat = normDualMat;
    alpha_primal = alpha_dual = ZERO;
    beta_value = dd_from(param.betaStar);
    reduction_on = true;
    mu_current = mu_initial;
    // RatioInitResCurrentRes::initialize (sdpa_parts.cpp:621-634)
    const dd_t accuracy = dd_from(param.epsilonDash);
    theta_primal = dd_lt(initNormPrimalVec, accuracy) ? ZERO : ONE;
    theta_dual = dd_lt(initNormDualMat, accuracy) ? ZERO : ONE;
    // SolveInfo::initialize (sdpa_parts.cpp:671-681)
    rho = ONE;
    const dd_t omega = dd_from(param.omegaStar);
    etaPrimal = dd_mul(dd_mul_d(omega, (double)c.nDim), mu_initial);
    etaDual = etaPrimal;
    objValPrimal = inner_C(c, c.X);
    objValDual = inner_b(c, c.y.p);
    phase_update_check();
    pIteration = 0;
}

// StepLength clamps shared by MehrotraPredictor / MehrotraCorrector
// (sdpa_parts.cpp:311-354, 372-408)
static void clamp_steps(Solver &s, dd_t &primal, dd_t &dual) {
    if (s.phase == noINFO || s.phase == dFEAS) {
        if (dd_gt_d(primal, 1.0)) primal = ONE;
    } else {
        dd_t incPrimalObj = inner_C(s.c, s.c.Dx);
        if (dd_gt_d(incPrimalObj, 0.0)) {
            if (dd_gt(primal, dual)) primal = dual;
            if (dd_gt_d(primal, 1.0)) primal = ONE;
        }
    }
    if (s.phase == noINFO || s.phase == pFEAS) {
        if (dd_gt_d(dual, 1.0)) dual = ONE;
    } else {
        dd_t incDualObj = inner_b(s.c, s.c.Dy.p);
        if (dd_lt_d(incDualObj, 0.0)) {
            if (dd_gt(dual, primal)) dual = primal;
            if (dd_gt_d(dual, 1.0)) dual = ONE;
        }
    }
}

// mu + (aP uz + aD xv + aP aD uv) / nDim  (sdpa_parts.cpp:419, 510)
static dd_t mu_after(const dd_t &mu, const dd_t &aP, const dd_t &aD, const dd_t &uz, const dd_t &xv, const dd_t &uv, long nDim) {
    dd_t s = dd_add(dd_add(dd_mul(aP, uz), dd_mul(aD, xv)), dd_mul(dd_mul(aP, aD), uv));
    return dd_add(mu, dd_div_d(s, (double)nDim));
}

int Solver::step(FILE *display, FILE *out) {
    if (!(phase_update_check() && pIteration < param.maxIteration)) return 1;
    EvClock clk(c);
    const auto t_iter0 = std::chrono::steady_clock::now();
    // Switch::MehrotraPredictor, DirectionParameter::MehrotraPredictor
    // (sdpa_parts.cpp:487-496, 542-556)
    reduction_on = (phase == noINFO || phase == pFEAS || phase == dFEAS);
    if (phase == pdFEAS) {
        beta_value = ZERO;
    } else {
        beta_value = dd_from(param.betaBar);
        if (!reduction_on) beta_value = dd_from(2.0);
    }
    last_betaPred = beta_value;
    const bool dinf = (phase == pFEAS || phase == noINFO);
    // Newton::Mehrotra(PREDICTOR) (sdpa_newton.cpp:1345-1384)
    cudaEvent_t e0 = clk.mark();
    make_rhs(c, false, dd_mul(beta_value, mu_current), dinf);
    cudaEvent_t e1 = clk.mark();
    int info = 0;
    if (c.core && core_eligible(c)) {
        // a batch worker: the Schur build and Cholesky run batched with the
        // other workers' problems (the same operations, entry by entry)
        clk.span(e0, e1, &tm.makegVec);
        const auto th0 = std::chrono::steady_clock::now();
        info = c.core->schur_factor(c);
        tm.choleskybMat += std::chrono::duration<double>(std::chrono::steady_clock::now() - th0).count();
    } else {
        schur_build(c);
        cudaEvent_t e2 = clk.mark();
        clk.span(e0, e1, &tm.makegVec);
        clk.span(e1, e2, &tm.makebMat);
        const auto th0 = std::chrono::steady_clock::now();
        info = schur_factor(c);
        tm.choleskybMat += std::chrono::duration<double>(std::chrono::steady_clock::now() - th0).count();
    }
    last_cholesky_info = info;
    if (info != 0) {
        if (display) std::fprintf(display, "cholesky miss condition :: not positive definite :: info = %d\n", info);
        clk.collect();
        return 2;
    }
    cudaEvent_t e3 = clk.mark();
    solve_dy(c);
    cudaEvent_t e4 = clk.mark();
    make_dz_dx(c, dinf);
    cudaEvent_t e5 = clk.mark();
    clk.span(e3, e4, &tm.solve);
    clk.span(e4, e5, &tm.makedXdZ);
    // StepLength::MehrotraPredictor (sdpa_parts.cpp:307-354)
    alpha_primal = alpha_dual = dd_from(0.9);
    clamp_steps(*this, alpha_primal, alpha_dual);
    last_alphaPredP = alpha_primal;
    last_alphaPredD = alpha_dual;
    // DirectionParameter::MehrotraCorrector (sdpa_parts.cpp:498-529)
    {
        ScalarBatch sb(c);
        const int gxv = sb.inner_space(c.X, c.Dz), guz = sb.inner_space(c.Dx, c.Z), guv = sb.inner_space(c.Dx, c.Dz);
        sb.fetch();
        dd_t xv = sb.sum(gxv), uz = sb.sum(guz), uv = sb.sum(guv);
        dd_t muTarget = mu_after(mu_current, alpha_primal, alpha_dual, uz, xv, uv, c.nDim);
        dd_t v = dd_div(muTarget, mu_current);
        if (dd_lt_d(v, 1.0)) v = dd_mul(v, v);
        if (phase == pdFEAS) {
            if (dd_lt_d(v, param.betaStar)) v = dd_from(param.betaStar);
            if (dd_gt_d(v, 1.0)) v = ONE;
        } else {
            if (dd_lt_d(v, param.betaBar)) v = dd_from(param.betaBar);
        }
        beta_value = v;
    }
    // early stop (sdpa_main.cpp:333-335)
    if (phase == pdFEAS && (dd_gt_d(beta_value, 5.0) || dd_lt(objValPrimal, objValDual))) {
        clk.collect();
        return 3;
    }
    // Newton::Mehrotra(CORRECTOR)
    cudaEvent_t c0 = clk.mark();
    make_rhs(c, true, dd_mul(beta_value, mu_current), dinf);
    cudaEvent_t c1 = clk.mark();
    solve_dy(c);
    cudaEvent_t c2 = clk.mark();
    make_dz_dx(c, dinf);
    cudaEvent_t c3 = clk.mark();
    clk.span(c0, c1, &tm.makegVec);
    clk.span(c1, c2, &tm.solve);
    clk.span(c2, c3, &tm.makedXdZ);
    // StepLength::MehrotraCorrector (sdpa_parts.cpp:244-305, 356-466)
    {
        const dd_t alphaBD = dd_from(100.0);
        const dd_t lim = dd_div(ONE, alphaBD);
        // both eigenvalues in one pass over the blocks (their Lanczos side
        // by side); the span is booked half to each
        cudaEvent_t g0 = clk.mark();
        dd_t minx, minz;
        min_eig_pair(c, c.invCholX, c.Dx, c.invCholZ, c.Dz, minx, minz);
        cudaEvent_t g1 = clk.mark();
        clk.span(g0, g1, &tm.eigBoth);
        last_minEigX = minx;
        last_minEigZ = minz;
        dd_t primal = dd_gt(dd_neg(minx), lim) ? dd_div(dd_from(-1.0), minx) : alphaBD;
        dd_t dual = dd_gt(dd_neg(minz), lim) ? dd_div(dd_from(-1.0), minz) : alphaBD;
        primal = dd_mul_d(primal, param.gammaStar);
        dual = dd_mul_d(dual, param.gammaStar);
        clamp_steps(*this, primal, dual);
        if (reduction_on && (phase == noINFO || phase == pFEAS || phase == dFEAS)) {
            const dd_t xi = dd_from(3.0);
            ScalarBatch sb(c);
            const int gxv = sb.inner_space(c.X, c.Dz), guz = sb.inner_space(c.Dx, c.Z), guv = sb.inner_space(c.Dx, c.Dz);
            sb.fetch();
            dd_t xv = sb.sum(gxv), uz = sb.sum(guz), uv = sb.sum(guv);
            dd_t thetaMax = smax(dd_mul(d_sub_dd(1.0, primal), theta_primal), dd_mul(d_sub_dd(1.0, dual), theta_dual));
            dd_t muNew = mu_after(mu_current, primal, dual, uz, xv, uv, c.nDim);
            while (dd_gt(dd_mul(dd_mul(thetaMax, thetaMax), mu_initial), dd_mul(xi, muNew))) {
                dd_t alphaMax = dd_mul_d(smax(primal, dual), 0.95);
                primal = smin(primal, alphaMax);
                dual = smin(dual, alphaMax);
                thetaMax = smax(dd_mul(d_sub_dd(1.0, primal), theta_primal), dd_mul(d_sub_dd(1.0, dual), theta_dual));
                muNew = mu_after(mu_current, primal, dual, uz, xv, uv, c.nDim);
                if (dd_lt_d(primal, 1.0e-6) && dd_lt_d(dual, 1.0e-6)) break;
            }
        }
        if (phase == pdFEAS) {
            ScalarBatch sb(c);
            const int goD = sb.inner_b(c.y.p), goP = sb.inner_C(c.X), giD = sb.inner_b(c.Dy.p), giP = sb.inner_C(c.Dx);
            sb.fetch();
            dd_t oD = sb.sum(goD), oP = sb.sum(goP);
            dd_t incD = dd_muleq(sb.sum(giD), dual);
            dd_t incP = dd_muleq(sb.sum(giP), primal);
            dd_t maxRatio = dd_div(dd_sub(oD, oP), dd_sub(incP, incD));
            if (dd_gt_d(maxRatio, 0.0) && dd_lt_d(maxRatio, 1.0)) {
                primal = dd_muleq(primal, maxRatio);
                dual = dd_muleq(dual, maxRatio);
            }
        }
        alpha_primal = primal;
        alpha_dual = dual;
    }
    print_one_iteration(display);
    print_one_iteration(out);
    // Solutions::update (sdpa_dataset.cpp:120-143)
    update_point(c, alpha_primal, alpha_dual);
    const dd_t cannot_move = dd_from(1.0e-4);
    if (dd_lt(alpha_primal, cannot_move) && dd_lt(alpha_dual, cannot_move)) {
        if (display) std::fprintf(display, "Step length is too small. \ncannot move\n");
        clk.collect();
        return 4;
    }
    // Solutions::computeInverse, then everything the loop tail reads from
    // the new point (mu, the residual norms, the objectives and the
    // SolveInfo traces), read back together
    cudaEvent_t u0 = clk.mark();
    compute_inverse_async(c);
    cudaEvent_t u1 = clk.mark();
    clk.span(u0, u1, &tm.zMatTime);
    ScalarBatch tail(c);
    const int g_inv = tail.inverse_info();
    const int g_mu = tail.inner_space(c.X, c.Z);
    cudaEvent_t r0 = clk.mark();
    int g_np, g_nd;
    tail.residuals(g_np, g_nd);
    cudaEvent_t r1 = clk.mark();
    clk.span(r0, r1, &tm.updateRes);
    const int g_oP = tail.inner_C(c.X), g_oD = tail.inner_b(c.y.p);
    const int g_x0z = c.has_init ? tail.inner_space(c.init_X, c.Z) : tail.lambda_trace(c.Z, param.lambdaStar);
    const int g_xz0 = c.has_init ? tail.inner_space(c.X, c.init_Z) : tail.lambda_trace(c.X, param.lambdaStar);
    tail.fetch();
    if (!tail.inverse_ok(g_inv)) {
        if (display) std::fprintf(display, "cannot cholesky decomposition\nCould you try with smaller gammaStar?\ncannot move\n");
        clk.collect();
        return 4;
    }
    // RatioInitResCurrentRes::update (sdpa_parts.cpp:636-642)
    if (reduction_on) {
        theta_primal = dd_abs(dd_mul(d_sub_dd(1.0, alpha_primal), theta_primal));
        theta_dual = dd_abs(dd_mul(d_sub_dd(1.0, alpha_dual), theta_dual));
    }
    // AverageComplementarity::update (sdpa_parts.cpp:585-589)
    mu_current = dd_div_d(tail.sum(g_mu), (double)c.nDim);
    // Residuals::update
    normPrimalVec = tail.value(g_np);
    normDualMat = tail.value(g_nd);
    // RatioInitResCurrentRes::update_exact (sdpa_parts.cpp:644-655)
    theta_primal = dd_gt_d(initNormPrimalVec, 1.0e-10) ? dd_div(normPrimalVec, initNormPrimalVec) : ZERO;
    theta_dual = dd_gt_d(initNormDualMat, 1.0e-10) ? dd_div(normDualMat, initNormDualMat) : ZERO;
    // SolveInfo::update (sdpa_parts.cpp:690-739 with an initial point file,
    // :741-770 with lambda I)
    {
        objValPrimal = tail.sum(g_oP);
        objValDual = tail.sum(g_oD);
        const dd_t primal = theta_primal, dual = theta_dual, omega = dd_from(param.omegaStar);
        rho = ZERO;
        const dd_t x0z0 = dd_mul_d(mu_initial, (double)c.nDim);
        const dd_t xMatzMat = dd_mul_d(mu_current, (double)c.nDim);
        const dd_t x0zMat = tail.sum(g_x0z);
        const dd_t xMatz0 = tail.sum(g_xz0);
        const dd_t accuracy = dd_from(param.epsilonDash);
        if (dd_le(normPrimalVec, accuracy))
            if (dd_lt(xMatz0, etaPrimal)) etaPrimal = xMatz0;
        if (dd_le(normDualMat, accuracy))
            if (dd_lt(x0zMat, etaDual)) etaDual = x0zMat;
        const bool pinf = dd_gt(normPrimalVec, accuracy), dinf2 = dd_gt(normDualMat, accuracy);
        if (pinf && !dinf2)
            rho = dd_div(dd_mul(primal, x0zMat), dd_add(dd_mul(dd_add(primal, dd_mul(d_sub_dd(1.0, primal), omega)), etaDual), xMatzMat));
        if (!pinf && dinf2)
            rho = dd_div(dd_mul(dual, xMatz0), dd_add(dd_mul(dd_add(dual, dd_mul(d_sub_dd(1.0, dual), omega)), etaPrimal), xMatzMat));
        if (pinf && dinf2) {
            dd_t num = dd_add(dd_mul(dual, xMatz0), dd_mul(primal, x0zMat));
            dd_t mix = dd_add(dd_mul(primal, d_sub_dd(1.0, dual)), dd_mul(d_sub_dd(1.0, primal), dual));
            dd_t den = dd_add(dd_mul(dd_add(dd_mul(primal, dual), dd_mul(omega, mix)), x0z0), xMatzMat);
            rho = dd_div(num, den);
        }
    }
    clk.collect();
    tm.mainLoop += std::chrono::duration<double>(std::chrono::steady_clock::now() - t_iter0).count();
    pIteration++;
    return 0;
}

void Solver::finish() {
    residuals(c, normPrimalVec, normDualMat);
    phase_reverse();
}

// IO::printOneIteration with REVERSE_PRIMAL_DUAL (sdpa_io.cpp:799-816)
void Solver::print_one_iteration(FILE *fp) {
    if (!fp) return;
    dd_t m1 = dd_neg(objValDual), m2 = dd_neg(objValPrimal);
    std::fprintf(fp, "%2d %4.1e %4.1e %4.1e %+7.2e %+7.2e %4.1e %4.1e %4.2e\n", pIteration, mu_current.hi, theta_dual.hi, theta_primal.hi, m1.hi, m2.hi,
                 alpha_dual.hi, alpha_primal.hi, beta_value.hi);
}

// -------------------------------------------------------- QD decimal output
// The reference prints dd values with QD 2.3.23's dd_real::to_digits /
// to_string (src/dd_real.cpp; Copyright (c) 2003-2009 The Regents of the
// University of California, through Lawrence Berkeley National Laboratory,
// modified BSD licence).  Identical digits need its steps: scale by a power
// of ten into [1, 10), peel precision + 1 digits by truncation and *10,
// settle digits outside 0..9 by borrow and carry, round on the last digit.
static dd_t npwr10(int e) { return dd_pow10(e); }

static void to_digits(dd_t a, char *s, int &expn, int precision) {
    const int D = precision + 1;
    dd_t r = dd_abs(a);
    if (a.hi == 0.0) {
        expn = 0;
        for (int i = 0; i < precision; ++i) s[i] = '0';
        return;
    }
    int e = (int)std::floor(std::log10(std::fabs(a.hi)));
    if (e < -300) {
        r = dd_muleq(r, npwr10(300));
        r = dd_div(r, npwr10(e + 300));
    } else if (e > 300) {
        r = dd_make(std::ldexp(r.hi, -53), std::ldexp(r.lo, -53));
        r = dd_div(r, npwr10(e));
        r = dd_make(std::ldexp(r.hi, 53), std::ldexp(r.lo, 53));
    } else {
        r = dd_div(r, npwr10(e));
    }
    if (dd_ge_d(r, 10.0)) {
        r = dd_div_d(r, 10.0);
        e++;
    } else if (dd_lt_d(r, 1.0)) {
        r = dd_mul_d(r, 10.0);
        e--;
    }
    std::vector<int> dig(D);
    for (int i = 0; i < D; ++i) {
        int d = (int)r.hi;
        r = dd_sub_d(r, (double)d);
        r = dd_mul_d(r, 10.0);
        dig[i] = d;
    }
    for (int i = D - 1; i > 0; --i) {
        if (dig[i] < 0) {
            dig[i - 1]--;
            dig[i] += 10;
        } else if (dig[i] > 9) {
            dig[i - 1]++;
            dig[i] -= 10;
        }
    }
    if (dig[D - 1] >= 5) {
        dig[D - 2]++;
        int i = D - 2;
        while (i > 0 && dig[i] > 9) {
            dig[i] -= 10;
            dig[--i]++;
        }
    }
    if (dig[0] > 9) {
        e++;
        for (int i = precision; i >= 2; --i) dig[i] = dig[i - 1];
        dig[0] = 1;
        dig[1] = 0;
    }
    for (int i = 0; i < precision; ++i) s[i] = (char)('0' + dig[i]);
    s[precision] = 0;
    expn = e;
}

std::string dd_to_string(dd_t a, int precision) {
    std::string s;
    if (dd_isnan(a)) return "nan";
    if (dd_lt_d(a, 0.0)) s += '-';
    if (std::isinf(a.hi)) return s + "inf";
    if (a.hi == 0.0 && a.lo == 0.0) {
        s += '0';
        if (precision > 0) {
            s += '.';
            s.append(precision, '0');
        }
        return s + "e+00";
    }
    const int d = precision + 1;
    std::vector<char> t(d + 2);
    int e = 0;
    to_digits(a, t.data(), e, d);
    s += t[0];
    if (precision > 0) s += '.';
    for (int i = 1; i <= precision; ++i) s += t[i];
    s += 'e';
    s += (e < 0 ? '-' : '+');
    int x = std::abs(e);
    if (x >= 100) {
        s += (char)('0' + x / 100);
        x %= 100;
    }
    s += (char)('0' + x / 10);
    s += (char)('0' + x % 10);
    return s;
}

static void param_display(FILE *fp, const Param &p) {
    std::fprintf(fp, "maxIteration =    %d\n", p.maxIteration);
    std::fprintf(fp, "epsilonStar  = %8.3e\n", p.epsilonStar);
    std::fprintf(fp, "lambdaStar   = %8.3e\n", p.lambdaStar);
    std::fprintf(fp, "omegaStar    = %8.3e\n", p.omegaStar);
    std::fprintf(fp, "lowerBound   = %8.3e\n", p.lowerBound);
    std::fprintf(fp, "upperBound   = %8.3e\n", p.upperBound);
    std::fprintf(fp, "betaStar     = %8.3e\n", p.betaStar);
    std::fprintf(fp, "betaBar      = %8.3e\n", p.betaBar);
    std::fprintf(fp, "gammaStar    = %8.3e\n", p.gammaStar);
    std::fprintf(fp, "epsilonDash  = %8.3e\n", p.epsilonDash);
}

// ComputeTime::display (sdpa_parts.cpp:72-123): the rows this path measures
// carry values, the others read 0.
static void com_display(FILE *fp, const Timers &t) {
    const double ML = t.mainLoop > 0 ? t.mainLoop : 1.0;
    auto row = [&](const char *name, double v) { std::fprintf(fp, " %s=       %f,  %f\n", name, v, v / ML * 100.0); };
    std::fprintf(fp, "\n");
    std::fprintf(fp, "                         Time(sec) ");
    std::fprintf(fp, " Ratio(%% : MainLoop) \n");
    row("Predictor time  ", t.predictor);
    row("Corrector time  ", t.corrector);
    row("Make bMat time  ", t.makebMat);
    row("Make bDia time  ", 0.0);
    row("Make bF1  time  ", 0.0);
    row("Make bF2  time  ", 0.0);
    row("Make bF3  time  ", 0.0);
    row("Make bPRE time  ", 0.0);
    row("Make rMat time  ", 0.0);
    row("Make gVec Mul   ", 0.0);
    row("Make gVec time  ", t.makegVec);
    row("Cholesky bMat   ", t.choleskybMat);
    row("Ste Pre time    ", t.stepPred);
    row("Ste Cor time    ", t.stepCorr);
    row("solve           ", t.solve);
    row("sumDz           ", 0.0);
    row("makedX          ", 0.0);
    row("symmetriseDx    ", 0.0);
    row("makedXdZ        ", t.makedXdZ);
    row("xMatTime        ", t.xMatTime);
    row("zMatTime        ", t.zMatTime);
    row("invzMatTime     ", 0.0);
    row("xMatzMatTime    ", 0.0);
    row("EigxMatTime     ", t.eigX + 0.5 * t.eigBoth);
    row("EigzMatTime     ", t.eigZ + 0.5 * t.eigBoth);
    row("EigxMatzMatTime ", 0.0);
    row("updateRes       ", t.updateRes);
    row("EigTime         ", t.eigX + t.eigZ + t.eigBoth);
    row("sub_total_bMat  ", t.mainLoop - t.makebMat);
    row("Main Loop       ", t.mainLoop);
    row("File Check      ", 0.0);
    row("File Change     ", 0.0);
    row("File Read       ", t.fileRead);
    row("Total           ", t.total);
    std::fprintf(fp, "\n");
}

static void display_space_last(FILE *fp, Context &c, const Space &s) {
    // IO::displayDenseLinarSpaceLast (sdpa_io.cpp:1205-1234), hi parts "%+18.12e",
    // the data's blocks in their order: an SDP block as a matrix, an LP block
    // as one list (its entries are the order-1 blocks from nSDPdata on)
    std::vector<dd_t> h(c.space_len);
    space_to_host(c, s, h.data());
    const Problem &P = c.prob;
    std::fprintf(fp, "{\n");
    for (int b = 0; b < P.nBlock; ++b) {
        if (P.blockType[b] != 1) {
            const int n = P.blockStruct[b], base = P.nSDPdata + P.blockNumber[b];
            std::fprintf(fp, "{");
            for (int t = 0; t < n - 1; ++t) std::fprintf(fp, "%+18.12e,", h[c.off[base + t]].hi);
            if (n > 0)
                std::fprintf(fp, "%+18.12e}\n", h[c.off[base + n - 1]].hi);
            else
                std::fprintf(fp, "  }\n");
            continue;
        }
        const int l = P.blockNumber[b];
        const int n = c.sizes[l];
        const dd_t *M = h.data() + c.off[l];
        // DenseMatrix::display (sdpa_struct.cpp:684-713)
        std::fprintf(fp, "{");
        for (int i = 0; i < n - 1; ++i) {
            std::fprintf(fp, i == 0 ? " " : "  ");
            std::fprintf(fp, "{");
            for (int j = 0; j < n - 1; ++j) std::fprintf(fp, "%+18.12e,", M[i + (long)n * j].hi);
            std::fprintf(fp, "%+18.12e },\n", M[i + (long)n * (n - 1)].hi);
        }
        if (n > 1) std::fprintf(fp, "  {");
        for (int j = 0; j < n - 1; ++j) std::fprintf(fp, "%+18.12e,", M[(n - 1) + (long)n * j].hi);
        std::fprintf(fp, "%+18.12e }", M[(n - 1) + (long)n * (n - 1)].hi);
        if (n > 1)
            std::fprintf(fp, "   }\n");
        else
            std::fprintf(fp, "\n");
    }
    std::fprintf(fp, "}\n");
}

// IO::printLastInfo (pinpal's overload, sdpa_io.cpp:1015-1203)
void Solver::print_last_info(FILE *display, FILE *out, double cputime, const std::string &) {
    print_one_iteration(display);
    print_one_iteration(out);
    dd_t mean = dd_div_d(dd_add(dd_abs(objValPrimal), dd_abs(objValDual)), 2.0);
    dd_t PDgap = dd_abs(dd_sub(objValPrimal, objValDual));
    dd_t relgap = dd_lt_d(mean, 1.0) ? PDgap : dd_div(PDgap, mean);
    dd_t gap = dd_mul_d(mu_current, (double)c.nDim);
    // -log10(|PDgap / mean|): evaluated in extended precision and rounded,
    // which matches the hi part of QD's dd log10 for printing.
    dd_t q = dd_abs(dd_div(PDgap, mean));
    long double lq = (long double)q.hi + (long double)q.lo;
    double digits = (double)(-log10l(lq));
    dd_t m1 = dd_neg(objValDual), m2 = dd_neg(objValPrimal);
    const double eps = 4.93038065763132e-32; // dd_real::_eps (Rlamch_dd("E"))
    for (int which = 0; which < 2; ++which) {
        FILE *fp = which == 0 ? display : out;
        if (!fp) continue;
        std::fprintf(fp, "\n");
        std::fprintf(fp, "phase.value = %s\n", phase_name(phase));
        std::fprintf(fp, "   Iteration = %d\n", pIteration);
        std::fprintf(fp, "          mu = %4.16e\n", mu_current.hi);
        std::fprintf(fp, "relative gap = %4.16e\n", relgap.hi);
        std::fprintf(fp, "         gap = %4.16e\n", gap.hi);
        std::fprintf(fp, "      digits = %4.16e\n", digits);
        if (which == 0) {
            std::fprintf(fp, "objValPrimal = %s\n", dd_to_string(m1, 32).c_str());
            std::fprintf(fp, "objValDual   = %s\n", dd_to_string(m2, 32).c_str());
        } else {
            std::fprintf(fp, "objValPrimal = %10.16e\n", m1.hi);
            std::fprintf(fp, "objValDual   = %10.16e\n", m2.hi);
        }
        std::fprintf(fp, "p.feas.error = %10.16e\n", normDualMat.hi);
        std::fprintf(fp, "d.feas.error = %10.16e\n", normPrimalVec.hi);
        std::fprintf(fp, "relative eps = %10.16e\n", eps);
        std::fprintf(fp, "total time   = %.3f\n", cputime);
    }
    if (out) {
        std::fprintf(out, "\n\nParameters are\n");
        param_display(out, param);
        com_display(out, tm);
        // xVec = -y, xMat = Z, yMat = X (REVERSE_PRIMAL_DUAL)
        std::vector<dd_t> y(c.m);
        CK(cudaMemcpy(y.data(), c.y.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToHost));
        std::fprintf(out, "xVec = \n{");
        for (int j = 0; j < c.m - 1; ++j) std::fprintf(out, "%+18.12e,", dd_mul(y[j], dd_from(-1.0)).hi);
        std::fprintf(out, "%+18.12e}\n", dd_mul(y[c.m - 1], dd_from(-1.0)).hi);
        std::fprintf(out, "xMat = \n");
        display_space_last(out, c, c.Z);
        std::fprintf(out, "yMat = \n");
        display_space_last(out, c, c.X);
    }
}

} // namespace sddd
