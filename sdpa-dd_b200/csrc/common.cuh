// Shared device/host helpers for the sm_100a dd kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "dd.h"

namespace sddd {

// Failures inside the library are thrown as sddd::Error and turned into
// status codes at the C-ABI boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

enum Status {
    OK = 0,
    ERR_ARG = -1,
    ERR_CUDA = -2,
    ERR_NOCONV = -3,
    ERR_STATE = -4,
    ERR_NOMEM = -5,
    ERR_IO = -6,
    ERR_UNSUPPORTED = -7,
};

inline void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
        throw Error(e == cudaErrorMemoryAllocation ? ERR_NOMEM : ERR_CUDA, buf);
    }
}
// Kernels launched by this library in this process (every launch site
// goes through CK_LAUNCH).
extern std::atomic<unsigned long long> g_launches;
#define CK(call) ::sddd::cuda_check((call), #call, __FILE__, __LINE__)
#define CK_LAUNCH()                                                                                                                                  \
    do {                                                                                                                                             \
        ++::sddd::g_launches;                                                                                                                        \
        ::sddd::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__);                                                                 \
    } while (0)

inline unsigned ceil_div(long a, long b) { return (unsigned)((a + b - 1) / b); }

// Device-resident matrix view: column-major dd, leading dimension ld.
struct Mat {
    dd_t *p = nullptr;
    long ld = 0;
    __host__ __device__ dd_t &operator()(long i, long j) const { return p[i + ld * j]; }
};

__device__ __forceinline__ dd_t ld_dd(const dd_t *p) {
    double2 v = *reinterpret_cast<const double2 *>(p);
    return dd_make(v.x, v.y);
}
__device__ __forceinline__ void st_dd(dd_t *p, dd_t v) { *reinterpret_cast<double2 *>(p) = make_double2(v.hi, v.lo); }

} // namespace sddd
