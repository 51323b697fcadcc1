// Batches of independent SDPs (the sddd_batch_* entry points of sddd.h; the
// reference solves one problem per process and has no counterpart).
//
// A batch keeps its problems on the host in the reference's storage model
// (read and finalised exactly as a single solve reads them) and solves them
// on one GPU with a pool of host workers.  Each worker owns one device
// context (its own CUDA stream and device buffers, grown to the largest
// problem it has taken and then reused, so uploads neither allocate nor
// free) and runs the ordinary solver on it, so every problem's iterates,
// phase, iteration count and objectives are bit for bit those of a single
// sddd_solve of that problem.  Problems are handed out largest first
// (m^3/3 + m^2 n^2 + 4 n^3 m per iteration) from an atomic counter; many
// small problems keep many streams of small kernels in flight at once.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sddd.h"
#include "adjoint.h"
#include "batched.h"
#include "capi_internal.h"
#include "context.h"
#include "newton.h"
#include "solver.h"

struct sddd_batch {
    int device = 0;
    int workers = 0;
    bool blocking_waits = false; // more workers than host cores: block instead of spin
    bool use_core = true;        // eligible problems take the batched Newton core
    std::string tuning;          // the core's autotuned tile shapes, after a solve
    std::vector<sddd::Problem> probs;
    // per problem, from the last sddd_batch_solve
    std::vector<sddd_result> results;
    std::vector<int> status;
    std::vector<std::string> errors;
    std::vector<std::vector<dd_t>> X, y, Z, grad_c;
    std::string err;
};

namespace {

double work_estimate(const sddd::Problem &p) {
    double w = (double)p.m * p.m * p.m / 3.0;
    for (int n : p.sdpSize) w += (double)p.m * p.m * n * n + 4.0 * n * (double)n * n * p.m;
    return w;
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

template <class F>
int guarded(sddd_batch *b, F &&f) {
    try {
        return f();
    } catch (const sddd::Error &e) {
        if (b) b->err = e.what();
        sddd_set_thread_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        if (b) b->err = e.what();
        sddd_set_thread_error(e.what());
        return SDDD_ERR_STATE;
    }
}

// A worker's context, set up for the batch (and for the batched core).
sddd::Context *worker_context(sddd_batch &B, sddd::CoreEngine *core) {
    std::unique_ptr<sddd::Context> c(sddd::create_context(B.device));
    sddd::set_shared_gpu(*c, B.blocking_waits);
    if (core) {
        CK(cudaEventCreateWithFlags(&c->core_ready, cudaEventDisableTiming));
        c->core = core;
    }
    return c.release();
}

// The engine counts a worker as active for the span of one solve.
struct CoreSpan {
    sddd::CoreEngine *e;
    bool on = false;
    explicit CoreSpan(sddd::CoreEngine *x) : e(x) {
        if (e) {
            e->enter();
            on = true;
        }
    }
    void end() {
        if (on) e->leave();
        on = false;
    }
    ~CoreSpan() { end(); }
};

// One worker: its own context; problems by index from `next` in `order`.
void batch_worker(sddd_batch &B, const std::vector<int> &order, std::atomic<int> &next, const sddd::Param &par, bool with_grad,
                  sddd::CoreEngine *core) {
    std::unique_ptr<sddd::Context> ctx;
    try {
        ctx.reset(worker_context(B, core));
    } catch (const sddd::Error &e) {
        // no context: leave this worker's share to the others
        return;
    }
    for (;;) {
        const int q = next.fetch_add(1);
        if (q >= (int)order.size()) break;
        const int idx = order[q];
        sddd::Context &c = *ctx;
        try {
            sddd::Problem p = B.probs[idx];
            sddd::upload_problem(c, std::move(p));
            sddd::Solver s(c, par);
            CoreSpan span(core);
            s.start();
            int rc = 0;
            while ((rc = s.step(nullptr, nullptr)) == 0) {
            }
            span.end();
            s.finish();
            sddd_fill_result(s, rc, &B.results[idx]);
            B.X[idx].resize(c.space_len);
            B.Z[idx].resize(c.space_len);
            B.y[idx].resize(c.m);
            sddd::d2h(c, B.X[idx].data(), c.X.buf.p, sizeof(dd_t) * c.space_len);
            sddd::d2h(c, B.Z[idx].data(), c.Z.buf.p, sizeof(dd_t) * c.space_len);
            sddd::d2h(c, B.y[idx].data(), c.y.p, sizeof(dd_t) * c.m);
            int st = 0;
            if (with_grad) {
                const dd_t one = dd_make(1.0, 0.0);
                st = sddd::adjoint_combined(c, nullptr, nullptr, nullptr, one);
                if (st == 0) {
                    sddd::adjoint_grad_c(c, one, c.adj_v.p);
                    B.grad_c[idx].resize(c.m);
                    sddd::d2h(c, B.grad_c[idx].data(), c.adj_v.p, sizeof(dd_t) * c.m);
                } else {
                    B.errors[idx] = "adjoint: the Schur matrix at the final iterate is not positive definite";
                }
            }
            B.status[idx] = st;
        } catch (const sddd::Error &e) {
            B.status[idx] = e.code;
            B.errors[idx] = e.what();
            if (e.code == SDDD_ERR_CUDA) {
                // the context may be unusable: start a fresh one
                try {
                    ctx.reset(worker_context(B, core));
                } catch (const sddd::Error &) {
                    return;
                }
            }
        } catch (const std::exception &e) {
            B.status[idx] = SDDD_ERR_STATE;
            B.errors[idx] = e.what();
        }
    }
}

} // namespace

extern "C" {

int sddd_batch_create(int device, int workers, sddd_batch **out) {
    if (!out) return SDDD_ERR_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        int count = 0;
        CK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) throw sddd::Error(SDDD_ERR_ARG, "no such CUDA device");
        auto *b = new sddd_batch();
        b->device = device;
        const int cores = (int)std::max(1u, std::thread::hardware_concurrency());
        b->workers = workers > 0 ? workers : std::min(8, cores);
        b->blocking_waits = b->workers > cores;
        *out = b;
        return SDDD_OK;
    });
}

int sddd_batch_destroy(sddd_batch *b) {
    delete b;
    return SDDD_OK;
}

const char *sddd_batch_last_error(const sddd_batch *b) { return b ? b->err.c_str() : ""; }

int sddd_batch_add_file(sddd_batch *b, const char *path, int sparse, double kappa) {
    if (!b || !path) return SDDD_ERR_ARG;
    return guarded(b, [&] {
        sddd::Problem p = sddd::read_problem(path, sparse != 0);
        sddd::finalize_problem(p, kappa);
        b->probs.push_back(std::move(p));
        return (int)b->probs.size() - 1;
    });
}

int sddd_batch_add_problem(sddd_batch *b, int m, int nblock, const int *block_struct, const sddd_dd *bvec, long nnz, const int *k, const int *blk,
                           const int *i, const int *j, const sddd_dd *val, double kappa) {
    if (!b || !block_struct || !bvec || (nnz > 0 && (!k || !blk || !i || !j || !val))) return SDDD_ERR_ARG;
    return guarded(b, [&] {
        sddd::Problem p = sddd::make_problem(m, nblock, block_struct, reinterpret_cast<const dd_t *>(bvec), nnz, k, blk, i, j,
                                             reinterpret_cast<const dd_t *>(val));
        sddd::finalize_problem(p, kappa);
        b->probs.push_back(std::move(p));
        return (int)b->probs.size() - 1;
    });
}

int sddd_batch_count(const sddd_batch *b) { return b ? (int)b->probs.size() : SDDD_ERR_ARG; }

int sddd_batch_solve(sddd_batch *b, const sddd_param *param, int with_grad, sddd_result *results) {
    if (!b || !param) return SDDD_ERR_ARG;
    return guarded(b, [&] {
        const int P = (int)b->probs.size();
        b->results.assign(P, sddd_result{});
        b->status.assign(P, SDDD_ERR_STATE);
        b->errors.assign(P, "not solved: no worker could create a device context");
        b->X.assign(P, {});
        b->y.assign(P, {});
        b->Z.assign(P, {});
        b->grad_c.assign(P, {});
        std::vector<int> order(P);
        std::vector<double> w(P);
        for (int p = 0; p < P; ++p) {
            order[p] = p;
            w[p] = work_estimate(b->probs[p]);
        }
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return w[a] > w[c]; });
        const sddd::Param par = to_param(param);
        std::atomic<int> next{0};
        const int nw = std::max(1, std::min(b->workers, P));
        std::unique_ptr<sddd::CoreEngine> core;
        if (b->use_core) core.reset(new sddd::CoreEngine(b->device));
        std::vector<std::thread> pool;
        pool.reserve(nw);
        for (int t = 0; t < nw; ++t) pool.emplace_back([&] { batch_worker(*b, order, next, par, with_grad != 0, core.get()); });
        for (auto &th : pool) th.join();
        if (core) b->tuning = core->tuning();
        if (results) std::memcpy(results, b->results.data(), sizeof(sddd_result) * P);
        for (int p = 0; p < P; ++p)
            if (b->status[p] < 0) throw sddd::Error(b->status[p], "problem " + std::to_string(p) + ": " + b->errors[p]);
        return SDDD_OK;
    });
}

int sddd_batch_set_core(sddd_batch *b, int on) {
    if (!b) return SDDD_ERR_ARG;
    b->use_core = on != 0;
    return SDDD_OK;
}

const char *sddd_batch_tuning(const sddd_batch *b) { return b ? b->tuning.c_str() : ""; }

int sddd_batch_status(const sddd_batch *b, int index) {
    if (!b || index < 0 || index >= (int)b->status.size()) return SDDD_ERR_ARG;
    return b->status[index];
}

int sddd_batch_get_point(const sddd_batch *b, int index, sddd_dd *X, sddd_dd *y, sddd_dd *Z) {
    if (!b || index < 0 || index >= (int)b->X.size()) return SDDD_ERR_ARG;
    if (b->X[index].empty()) return SDDD_ERR_STATE;
    if (X) std::memcpy(X, b->X[index].data(), sizeof(dd_t) * b->X[index].size());
    if (y) std::memcpy(y, b->y[index].data(), sizeof(dd_t) * b->y[index].size());
    if (Z) std::memcpy(Z, b->Z[index].data(), sizeof(dd_t) * b->Z[index].size());
    return SDDD_OK;
}

int sddd_batch_grad_c(const sddd_batch *b, int index, sddd_dd *grad_c) {
    if (!b || !grad_c || index < 0 || index >= (int)b->grad_c.size()) return SDDD_ERR_ARG;
    if (b->grad_c[index].empty()) return SDDD_ERR_STATE;
    std::memcpy(grad_c, b->grad_c[index].data(), sizeof(dd_t) * b->grad_c[index].size());
    return SDDD_OK;
}

} // extern "C"
