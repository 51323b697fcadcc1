// The MPLAPACK seam of SDPA-DD bound to libsddd: Rgemm, Rpotrf and Rtrsv
// with the C++ signatures of the reference's mplapack/mpblas_dd.h:47,54 and
// mplapack/mplapack_dd.h:41, forwarding to sddd_Rgemm, sddd_Rpotrf and
// sddd_Rtrsv on the GPU.
//
// A maintainer links this file into the reference's sdpa_dd in place of
// mplapack/Rgemm_omp.cpp (with Rgemm_{NN,NT,TN,TT}_omp.cpp), Rpotrf.cpp and
// Rtrsv.cpp, and adds -lsddd -lcudart; everything else stays as it is.
// Every call copies its operands to device buffers (grown on demand, kept
// for the process), runs the kernel and copies the result back, so the
// binary's results are the reference's own, bit for bit (the kernels keep
// MPLAPACK's per-entry operation order).  Bad arguments go to the
// reference's Mxerbla_dd with the position it reports; a forwarding error
// (no GPU, a form SDPA never calls) prints the library's message and
// aborts, as Mxerbla does for its own errors.
#include <mpblas_dd.h>
#include <mplapack_dd.h>

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "sddd.h"

namespace {

static_assert(sizeof(dd_real) == sizeof(sddd_dd), "dd_real and sddd_dd must share a layout");

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    void *get(size_t bytes) {
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            if (cudaMalloc(&p, bytes) != cudaSuccess) {
                std::fprintf(stderr, "mplapack_sddd: cudaMalloc of %zu bytes failed\n", bytes);
                std::abort();
            }
            cap = bytes;
        }
        return p;
    }
};

struct Gpu {
    sddd_ctx *ctx = nullptr;
    DevBuf a, b, c;
    std::mutex mu; // the reference calls these from OpenMP regions too
    Gpu() {
        if (sddd_create(0, &ctx) != SDDD_OK) {
            std::fprintf(stderr, "mplapack_sddd: %s\n", sddd_last_error(nullptr));
            std::abort();
        }
    }
};

Gpu &gpu() {
    static Gpu g;
    return g;
}

void fail(const char *routine, int rc) {
    if (rc == SDDD_ERR_ARG) {
        // sddd's message names the 1-based position, as Mxerbla reports it
        std::fprintf(stderr, "mplapack_sddd: %s\n", sddd_last_error(gpu().ctx));
        std::abort();
    }
    std::fprintf(stderr, "mplapack_sddd: %s failed (%d): %s\n", routine, rc, sddd_last_error(gpu().ctx));
    std::abort();
}

// A copy from pageable memory may still be in flight when cudaMemcpy
// returns, and the library's kernels run on a non-blocking stream: wait for
// the device before the call that reads the data.
void h2d(void *d, const void *h, size_t bytes) {
    if (bytes && cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) fail("cudaMemcpy", SDDD_ERR_CUDA);
}
void h2d_done() {
    if (cudaDeviceSynchronize() != cudaSuccess) fail("cudaDeviceSynchronize", SDDD_ERR_CUDA);
}
void d2h(void *h, const void *d, size_t bytes) {
    if (bytes && cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) fail("cudaMemcpy", SDDD_ERR_CUDA);
}

inline bool is(const char *s, char c) { return s && (s[0] == c || s[0] == c + ('a' - 'A')); }

// Bytes of a column-major rows x cols operand with leading dimension ld,
// up to its last entry (a caller may pass a pointer into a larger array:
// nothing past the operand's last entry is read or written).
// An invalid ld (< rows) copies nothing; the library then reports it.
inline size_t extent(long ld, long rows, long cols) {
    return rows > 0 && cols > 0 && ld >= rows ? sizeof(dd_real) * (size_t)(ld * (cols - 1) + rows) : 0;
}

} // namespace

void Rgemm(const char *transa, const char *transb, mplapackint const m, mplapackint const n, mplapackint const k, dd_real const alpha, dd_real *a,
           mplapackint const lda, dd_real *b, mplapackint const ldb, dd_real const beta, dd_real *c, mplapackint const ldc) {
    Gpu &g = gpu();
    std::lock_guard<std::mutex> lock(g.mu);
    const bool nota = is(transa, 'N'), notb = is(transb, 'N');
    // op(A) is m x k, op(B) k x n, C m x n
    const size_t ba = nota ? extent(lda, m, k) : extent(lda, k, m), bb = notb ? extent(ldb, k, n) : extent(ldb, n, k), bc = extent(ldc, m, n);
    void *da = g.a.get(ba + 16), *db = g.b.get(bb + 16), *dc = g.c.get(bc + 16);
    h2d(da, a, ba);
    h2d(db, b, bb);
    h2d(dc, c, bc);
    h2d_done();
    const sddd_dd al{alpha.x[0], alpha.x[1]}, be{beta.x[0], beta.x[1]};
    const int rc = sddd_Rgemm(g.ctx, transa ? transa[0] : '?', transb ? transb[0] : '?', m, n, k, al, (const sddd_dd *)da, lda,
                              (const sddd_dd *)db, ldb, be, (sddd_dd *)dc, ldc);
    if (rc != SDDD_OK) fail("Rgemm", rc);
    d2h(c, dc, bc);
}

void Rpotrf(const char *uplo, mplapackint const n, dd_real *a, mplapackint const lda, mplapackint &info) {
    Gpu &g = gpu();
    std::lock_guard<std::mutex> lock(g.mu);
    const size_t bytes = extent(lda, n, n);
    void *da = g.a.get(bytes + 16);
    h2d(da, a, bytes);
    h2d_done();
    const int rc = sddd_Rpotrf(g.ctx, uplo ? uplo[0] : '?', n, (sddd_dd *)da, lda);
    if (rc < 0) fail("Rpotrf", rc);
    d2h(a, da, bytes);
    info = rc;
}

void Rtrsv(const char *uplo, const char *trans, const char *diag, mplapackint const n, dd_real *a, mplapackint const lda, dd_real *x,
           mplapackint const incx) {
    Gpu &g = gpu();
    std::lock_guard<std::mutex> lock(g.mu);
    const size_t ba = extent(lda, n, n), bx = n > 0 ? sizeof(dd_real) * (size_t)n : 0;
    void *da = g.a.get(ba + 16), *dx = g.b.get(bx + 16);
    h2d(da, a, ba);
    if (incx == 1) h2d(dx, x, bx);
    h2d_done();
    const int rc = sddd_Rtrsv(g.ctx, uplo ? uplo[0] : '?', trans ? trans[0] : '?', diag ? diag[0] : '?', n, (const sddd_dd *)da, lda, (sddd_dd *)dx,
                              incx);
    if (rc != SDDD_OK) fail("Rtrsv", rc);
    d2h(x, dx, bx);
}
