// Opt-in per-kernel timing with CUDA events on the launching stream.
// When a profiler is installed for the calling thread, PROF_SCOPE records
// an event pair around the enclosed launches; collect() reads the elapsed
// times after a stream synchronisation.  Off by default: no events, no
// synchronisation.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

namespace sddd {

struct Profiler {
    struct Rec {
        const char *name;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    std::map<std::string, std::pair<double, long>> totals; // ms, launches
    cudaEvent_t get();
    void collect(cudaStream_t st);
    ~Profiler();
};

extern thread_local Profiler *g_prof;

struct ProfScope {
    Profiler *p;
    const char *name;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    ProfScope(const char *n, cudaStream_t s) : p(g_prof), name(n), st(s) {
        if (p) {
            a = p->get();
            cudaEventRecord(a, st);
        }
    }
    ~ProfScope() {
        if (p) {
            cudaEvent_t b = p->get();
            cudaEventRecord(b, st);
            p->pending.push_back({name, a, b});
        }
    }
};

#define SDDD_CAT2(a, b) a##b
#define SDDD_CAT(a, b) SDDD_CAT2(a, b)
#define PROF_SCOPE(name, st) ::sddd::ProfScope SDDD_CAT(_prof_scope_, __LINE__)(name, st)

} // namespace sddd
