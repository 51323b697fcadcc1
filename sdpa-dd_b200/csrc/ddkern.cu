// Elementwise dd arithmetic on the device, one operation per element (the
// operation numbering of the arithmetic tests).  Used to check the device
// rounding of every dd shape against QD.
#include "../../include/sddd.h"
#include "common.cuh"

namespace sddd {

__global__ void dd_op_kernel(int op, long n, const dd_t *a, const dd_t *b, dd_t *out) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    dd_t x = a[i], y = b[i], r;
    switch (op) {
    case 0: r = dd_add(x, y); break;
    case 1: r = dd_acc(x, y); break;
    case 2:
    case 3: r = dd_sub(x, y); break;
    case 4: r = dd_mul(x, y); break;
    case 5: r = dd_muleq(x, y); break;
    case 6: r = dd_div(x, y); break;
    case 7: r = dd_sqrt(x); break;
    case 8: r = dd_mul_d(x, y.hi); break;
    case 9: r = dd_add_d(x, y.hi); break;
    case 10: r = dd_sub_d(x, y.hi); break;
    case 11: r = d_sub_dd(x.hi, y); break;
    case 12: r = dd_div_d(x, y.hi); break;
    case 13: r = dd_div(dd_from(x.hi), y); break;
    case 14: r = dd_neg(x); break;
    case 15: r = dd_abs(x); break;
    case 16: r = dd_sqr(x); break;
    case 17: r = dd_add_dd_exact(x.hi, y.hi); break;
    default: r = dd_zero(); break;
    }
    out[i] = r;
}

// FP64 issue-rate probe: 8 independent FMA chains per thread, full
// occupancy; the FP64-pipe ceiling the dd kernels are measured against.
__global__ void fp64_probe_kernel(double *out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = threadIdx.x * 1e-3 + j;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = __fma_rn(x[j], a, b);
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += x[j];
    if (s == 1.2345) out[0] = s; // keeps the chains live
}

} // namespace sddd

extern "C" int sddd_fp64_peak(sddd_ctx *, double *gflops) {
    if (!gflops) return SDDD_ERR_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return SDDD_ERR_CUDA;
    const int iters = 4096, threads = 256, blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    sddd::fp64_probe_kernel<<<blocks, threads>>>(d, iters, 0.999999, 1e-9);
    cudaEventRecord(a);
    sddd::fp64_probe_kernel<<<blocks, threads>>>(d, iters, 0.999999, 1e-9);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (cudaGetLastError() != cudaSuccess || ms <= 0) return SDDD_ERR_CUDA;
    *gflops = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e9;
    return SDDD_OK;
}

extern "C" int sddd_dd_op(sddd_ctx *, int op, long n, const sddd_dd *a, const sddd_dd *b, sddd_dd *out) {
    if (n <= 0) return SDDD_OK;
    if (!a || !b || !out || op < 0 || op > 17) return SDDD_ERR_ARG;
    sddd::dd_op_kernel<<<sddd::ceil_div(n, 256), 256>>>(op, n, reinterpret_cast<const dd_t *>(a), reinterpret_cast<const dd_t *>(b),
                                                       reinterpret_cast<dd_t *>(out));
    if (cudaGetLastError() != cudaSuccess) return SDDD_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return SDDD_ERR_CUDA;
    return SDDD_OK;
}

// ------------------------------------------------------- host-side checks
// The same dd shapes compiled for the host (the solver's scalar control
// runs on these), the QD-compatible decimal reader and QD's 32-digit output.
#include "problem.h"
#include "solver.h"
#include <cstring>

extern "C" int sddd_host_dd_op(int op, long n, const sddd_dd *a, const sddd_dd *b, sddd_dd *out) {
    if (op < 0 || op > 17) return SDDD_ERR_ARG;
    for (long i = 0; i < n; ++i) {
        dd_t x = dd_make(a[i].hi, a[i].lo), y = dd_make(b[i].hi, b[i].lo), r;
        switch (op) {
        case 0: r = dd_add(x, y); break;
        case 1: r = dd_acc(x, y); break;
        case 2:
        case 3: r = dd_sub(x, y); break;
        case 4: r = dd_mul(x, y); break;
        case 5: r = dd_muleq(x, y); break;
        case 6: r = dd_div(x, y); break;
        case 7: r = dd_sqrt(x); break;
        case 8: r = dd_mul_d(x, y.hi); break;
        case 9: r = dd_add_d(x, y.hi); break;
        case 10: r = dd_sub_d(x, y.hi); break;
        case 11: r = d_sub_dd(x.hi, y); break;
        case 12: r = dd_div_d(x, y.hi); break;
        case 13: r = dd_div(dd_from(x.hi), y); break;
        case 14: r = dd_neg(x); break;
        case 15: r = dd_abs(x); break;
        case 16: r = dd_sqr(x); break;
        default: r = dd_add_dd_exact(x.hi, y.hi); break;
        }
        out[i].hi = r.hi;
        out[i].lo = r.lo;
    }
    return SDDD_OK;
}

extern "C" int sddd_host_dd_read(const char *s, sddd_dd *out) {
    dd_t v;
    int rc = sddd::dd_read(s, &v);
    out->hi = v.hi;
    out->lo = v.lo;
    return rc;
}

extern "C" int sddd_host_dd_to_string(sddd_dd a, int precision, char *buf, int buflen) {
    std::string s = sddd::dd_to_string(dd_make(a.hi, a.lo), precision);
    if ((int)s.size() + 1 > buflen) return SDDD_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)s.size();
}
