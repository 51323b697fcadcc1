#include "prof.h"
#include "common.cuh"

namespace sddd {

thread_local Profiler *g_prof = nullptr;
std::atomic<unsigned long long> g_launches{0};

cudaEvent_t Profiler::get() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void Profiler::collect(cudaStream_t st) {
    cudaStreamSynchronize(st);
    for (auto &r : pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        auto &t = totals[r.name];
        t.first += ms;
        t.second += 1;
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    pending.clear();
}

Profiler::~Profiler() {
    for (auto &r : pending) {
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
}

} // namespace sddd
