// sddd_min_eig_noalloc: the step-length eigenvalue lambda_min(L D L^T) of
// one block, computed with no device allocation at all.
//
// Who needs it: a caller that owns every byte of device memory through its
// own pool (a caching allocator that already holds the GPU, a serving
// process with a fixed memory budget) cannot let a library call cudaMalloc,
// which fails once the pool holds the memory, or cudaFree, which
// synchronises the whole device and stalls that caller's other streams.
// sddd_min_eig keeps its block list and Lanczos vectors in context buffers
// that grow on demand, so it allocates on a context's first call and on any
// call with a larger block, and it needs a context (whose creation
// allocates) at all; this entry point runs the same kernels on a scratch
// array that is part of the library image instead.
//
// Scratch: one file-scope __device__ array of NOALLOC_SCRATCH_DD dd values
// (about 320 KiB), which every GPU that loads the library holds until the
// process exits.  Host code cannot use the array's name as a device address;
// the first call on each device looks the address up once, with that device
// current, and caches it.  Every call shares the array and the array keeps
// the previous call's contents: the header is rewritten by every call and
// the Lanczos kernel initialises its own vectors, so nothing stale is read,
// but two calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on the array.
#include <mutex>

#include "../../include/sddd.h"
#include "blas.h"
#include "capi_internal.h"
#include "common.cuh"
#include "eig_kernels.cuh"

namespace sddd {
namespace {

constexpr long NOALLOC_MAX_N = SDDD_MIN_EIG_NOALLOC_MAX_N;
// Order up to which the block takes the dense path (two GEMMs and a
// tridiagonal eigenvalue), as Jal::getMinEigen (sdpa_jordan.cpp:55-88).
constexpr long SMALL_N = 20;
// Header (block id, order, offset) in the first 256 bytes, then five Lanczos
// vectors of the largest order; the dense path's two n x n products fit in
// the same region.
constexpr long HEADER_DD = 16;
constexpr long NOALLOC_SCRATCH_DD = HEADER_DD + 5 * NOALLOC_MAX_N;
static_assert(2 * SMALL_N * SMALL_N <= 5 * NOALLOC_MAX_N, "dense path fits the Lanczos region");

static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_SCRATCH_DD];

// Block list of one block of order n at offset 0.
__global__ void noalloc_header_kernel(int *ids, int *sizes, long *off, int n) {
    ids[0] = 0;
    sizes[0] = n;
    off[0] = 0;
}

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
double2 *g_scratch_addr[MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on the current device (looked up on
// the first call per device).
int scratch_address(double2 **out, char *msg, size_t msglen) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        std::snprintf(msg, msglen, "sddd_min_eig_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
        return SDDD_ERR_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) {
        std::snprintf(msg, msglen, "sddd_min_eig_noalloc: device %d is beyond the %d devices it supports", dev, MAX_DEVICES);
        return SDDD_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::snprintf(msg, msglen, "sddd_min_eig_noalloc: cudaGetSymbolAddress of the scratch array failed on device %d: %s", dev,
                          cudaGetErrorString(e));
            return SDDD_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double2 *>(p);
    }
    *out = g_scratch_addr[dev];
    return SDDD_OK;
}

} // namespace
} // namespace sddd

extern "C" int sddd_min_eig_noalloc(void *stream, long n, const sddd_dd *L, const sddd_dd *D, sddd_dd *out) {
    using namespace sddd;
    char msg[256];
    if (n < 1 || n > NOALLOC_MAX_N) {
        std::snprintf(msg, sizeof msg, "sddd_min_eig_noalloc: block order n = %ld is outside 1..%ld (the size of its static scratch array)", n,
                      NOALLOC_MAX_N);
        sddd_set_thread_error(msg);
        return SDDD_ERR_ARG;
    }
    if (!L || !D || !out) {
        sddd_set_thread_error("sddd_min_eig_noalloc: L, D and out must be device pointers");
        return SDDD_ERR_ARG;
    }
    double2 *base = nullptr;
    int rc = scratch_address(&base, msg, sizeof msg);
    if (rc != SDDD_OK) {
        sddd_set_thread_error(msg);
        return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *ids = reinterpret_cast<int *>(base);
    int *sizes = ids + 4;
    long *off = reinterpret_cast<long *>(base + 2);
    dd_t *work = reinterpret_cast<dd_t *>(base + HEADER_DD);
    const dd_t *Ld = reinterpret_cast<const dd_t *>(L), *Dd = reinterpret_cast<const dd_t *>(D);
    dd_t *o = reinterpret_cast<dd_t *>(out);
    try {
        noalloc_header_kernel<<<1, 1, 0, st>>>(ids, sizes, off, (int)n);
        CK_LAUNCH();
        if (n > SMALL_N) {
            lanczos_kernel<<<1, LZ_THREADS, 0, st>>>(ids, 1, sizes, off, Ld, Dd, Ld, Dd, work, 5 * n, o);
            CK_LAUNCH();
        } else {
            // W2 = D L^T (Rgemm "N","T"), W1 = L W2 (Rgemm "N","N")
            const int m = (int)n;
            dd_t *W2 = work, *W1 = work + n * n;
            gemm(st, 'N', 'T', GEMM_STORE, m, m, m, Dd, n, 0, Ld, n, 0, W2, n, 0, 1, false);
            gemm(st, 'N', 'N', GEMM_STORE, m, m, m, Ld, n, 0, W2, n, 0, W1, n, 0, 1, false);
            small_min_eig_kernel<<<1, 32, 0, st>>>(ids, sizes, off, W1, o);
            CK_LAUNCH();
        }
    } catch (const Error &e) {
        sddd_set_thread_error(e.what());
        return e.code;
    }
    return SDDD_OK;
}
