// Host driver of the interior-point method (the reference's pinpal,
// sdpa_main.cpp:43-453) and its scalar control (sdpa_parts.cpp): step
// lengths, direction parameter, phase, stopping tests.  All vector and
// matrix work goes to the device through newton.h; only dd scalars live on
// the host.
#pragma once

#include <cstdio>
#include <string>

#include "context.h"

namespace sddd {

enum PhaseType { noINFO = 0, pFEAS, dFEAS, pdFEAS, pdINF, pFEAS_dINF, pINF_dFEAS, pdOPT, pUNBD, dUNBD };

// ComputeTime rows the device path measures (seconds).
struct Timers {
    double predictor = 0, corrector = 0, makebMat = 0, choleskybMat = 0, solve = 0, makedXdZ = 0, makegVec = 0, stepPred = 0, stepCorr = 0,
           eigX = 0, eigZ = 0, eigBoth = 0, xMatTime = 0, zMatTime = 0, updateRes = 0, mainLoop = 0, fileRead = 0, total = 0;
};

class Solver {
  public:
    Solver(Context &c, const Param &p);
    // Solutions::initialize .. Phase (sdpa_main.cpp:229-282)
    void start();
    // One pass of the main loop (sdpa_main.cpp:294-376).  Returns 0 when
    // the loop goes on, 1 when its condition ended it before this pass,
    // 2 on Cholesky failure of B, 3 on the pdFEAS early stop, 4 when the
    // point cannot move.
    int step(FILE *display, FILE *out);
    // Residuals::compute + phase reversal after the loop (:379-385)
    void finish();

    Context &c;
    Param param;
    // scalar state
    dd_t mu_initial, mu_current;
    dd_t theta_primal, theta_dual;
    dd_t alpha_primal, alpha_dual;
    dd_t beta_value;
    bool reduction_on = true;
    PhaseType phase = noINFO;
    dd_t rho, etaPrimal, etaDual, objValPrimal, objValDual;
    dd_t normPrimalVec, normDualMat, initNormPrimalVec, initNormDualMat;
    int pIteration = 0;
    Timers tm;
    // last pass, for tests and benchmarks
    dd_t last_minEigX, last_minEigZ, last_alphaPredP, last_alphaPredD, last_betaPred;
    int last_cholesky_info = 0;

    bool phase_update_check();
    void phase_reverse();
    void print_one_iteration(FILE *fp);
    void print_last_info(FILE *display, FILE *out, double cputime, const std::string &header_out);
};

// QD's operator<< for dd_real with precision p and default flags
// (dd_real::to_string / to_digits, dd_real.cpp:904-1190).
std::string dd_to_string(dd_t a, int precision);
const char *phase_name(PhaseType p);

} // namespace sddd
