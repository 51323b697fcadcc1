// C++-linkage helpers shared by the C ABI and the command-line driver.
#pragma once
#include <cstdio>

#include "../../include/sddd.h"
#include "problem.h"

void sddd_attach_problem(sddd_ctx *ctx, sddd::Problem &&p);
int sddd_solve_stream(sddd_ctx *ctx, const sddd_param *param, FILE *disp, FILE *fo, double fileRead, double *mainLoop);
// Records the message that sddd_last_error(NULL) returns on this thread
// (for entry points that take no context).
void sddd_set_thread_error(const char *msg);
namespace sddd {
class Solver;
}
// The numbers sddd_solve reports, from a finished solver.
void sddd_fill_result(const sddd::Solver &s, int stop_reason, sddd_result *out);
