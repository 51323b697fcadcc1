// Adjoint of the solve at its final iterate: gradients of the optimal value
// and of the solution (x, Y, X) with respect to the data c, F_0, F_k.  The
// reference has no derivative code; this is new.
//
// In the solver's internal form (sdpa_io.cpp:692-694: C = -F_0, A_k = F_k,
// b = c; the file's x is -y, its Y is the internal X, its X the internal Z)
// the iterate satisfies
//     A_k . X = b_k,   sum_k y_k A_k + Z = C,   X Z = mu I.
// Differentiating with mu held fixed and the HKM form of the last equation
// (dX = -sym(X dZ Z^-1), the form whose Schur matrix the solver factors,
// sdpa_newton.cpp:895-1068) gives the forward map
//     R  = dC - sum_k y_k dA_k
//     B dy = db - dA(X) + A(X R Z^-1),      B_kl = A_k . (X A_l Z^-1)
//     dZ = R - A^T(dy),   dX = -sym(X dZ Z^-1).
// Its transpose, for output weights (g_X, g_y, g_Z):
//     g_Z' = g_Z - sym(X g_X Z^-1)
//     u    = B^-1 (g_y - A(g_Z'))           (the Cholesky of B at the iterate)
//     R_g  = g_Z' + sym(X A^T(u) Z^-1)
//     grad b = u,  grad C = R_g,  grad A_k = -u_k X - y_k R_g.
// As mu -> 0 this tends to the derivative of the optimal solution; for the
// optimal value it tends to the envelope gradient (x, Y, -x_k Y).
#include "adjoint.h"

#include "blas.h"
#include "newton.h"

namespace sddd {

static const dd_t MONE = {-1.0, 0.0};

static void adj_alloc(Context &c) {
    c.adj_u.alloc(c.m);
    c.adj_v.alloc(c.m);
    c.adj_x.alloc(c.m);
    c.adj_R.buf.alloc(c.space_len);
    c.adj_T.buf.alloc(c.space_len);
}

// g_y = -g_x - g_obj b   (the objective is c.x = -b.y, x = -y)
__global__ void adj_seed_y_kernel(int m, const dd_t *gx, const dd_t *b, dd_t gobj, dd_t *gy) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    dd_t v = dd_neg(dd_mul(gobj, ld_dd(b + k)));
    if (gx) v = dd_sub(v, ld_dd(gx + k));
    st_dd(gy + k, v);
}

// out = a - t (t may be null: out = a; a may be null: out = -t)
__global__ void adj_sub_kernel(long n, const dd_t *a, const dd_t *t, dd_t *out) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    dd_t v = a ? ld_dd(a + e) : dd_zero();
    if (t) v = dd_sub(v, ld_dd(t + e));
    st_dd(out + e, v);
}

// grad c = u - g_obj y
__global__ void adj_grad_c_kernel(int m, const dd_t *u, const dd_t *y, dd_t gobj, dd_t *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    st_dd(out + k, dd_sub(ld_dd(u + k), dd_mul(gobj, ld_dd(y + k))));
}

// grad F_k = -u_k X - y_k R over one block space
__global__ void adj_grad_F_kernel(long n, dd_t uk, dd_t yk, const dd_t *X, const dd_t *R, dd_t *out) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    st_dd(out + e, dd_neg(dd_add(dd_mul(uk, ld_dd(X + e)), dd_mul(yk, ld_dd(R + e)))));
}

static void sym_blocks(Context &c, Space &s) {
    for (int l = 0; l < c.nSDP; ++l) symmetrize(c.stream, s.blk(c.off, l), c.sizes[l]);
}

int adjoint(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj) {
    cudaStream_t st = c.stream;
    const long L = c.space_len;
    adj_alloc(c);
    c.adj_valid = false;
    // host weights up: g_x -> adj_x, g_Y -> Dx (the internal X weight),
    // g_X -> Dz (the internal Z weight); the Newton direction is scratch now
    if (g_x) CK(cudaMemcpyAsync(c.adj_x.p, g_x, sizeof(dd_t) * c.m, cudaMemcpyHostToDevice, st));
    if (g_Y) space_from_host(c, c.Dx, g_Y);
    if (g_X) space_from_host(c, c.Dz, g_X);
    adj_seed_y_kernel<<<ceil_div(c.m, 128), 128, 0, st>>>(c.m, g_x ? c.adj_x.p : nullptr, c.b.p, g_obj, c.adj_v.p);
    CK_LAUNCH();
    // g_Z' = g_Z - sym(X g_X Z^-1)  -> adj_R
    const dd_t *t = nullptr;
    if (g_Y) {
        triple(c, c.X, c.Dx, c.invZ, c.adj_T);
        sym_blocks(c, c.adj_T);
        t = c.adj_T.buf.p;
    }
    adj_sub_kernel<<<ceil_div(L, 256), 256, 0, st>>>(L, g_X ? c.Dz.buf.p : nullptr, t, c.adj_R.buf.p);
    CK_LAUNCH();
    // v = g_y - A(g_Z')
    constraint_inner(c, c.adj_R, c.adj_v.p, c.adj_v.p);
    // u = B^-1 v with B at this iterate
    schur_build(c);
    const int info = schur_factor(c);
    if (info != 0) return info;
    CK(cudaMemcpyAsync(c.adj_u.p, c.adj_v.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToDevice, st));
    TrsvSync &sync = trsv_sync(c, c.m);
    trsv_lower(st, 'N', c.B.p, c.m, c.m, c.adj_u.p, sync, c.shared_gpu);
    trsv_lower(st, 'T', c.B.p, c.m, c.m, c.adj_u.p, sync, c.shared_gpu);
    trsv_check(st, sync);
    // R_g = g_Z' + sym(X A^T(u) Z^-1) = g_Z' - sym(X (-A^T(u)) Z^-1)
    sum_yA(c, c.adj_u.p, c.Dz, 0, nullptr, nullptr);
    triple(c, c.X, c.Dz, c.invZ, c.adj_T);
    sym_blocks(c, c.adj_T);
    adj_sub_kernel<<<ceil_div(L, 256), 256, 0, st>>>(L, c.adj_R.buf.p, c.adj_T.buf.p, c.adj_R.buf.p);
    CK_LAUNCH();
    stream_sync(c);
    c.adj_valid = true;
    return 0;
}

void adjoint_grad_c(Context &c, dd_t g_obj, dd_t *out_dev) {
    adj_grad_c_kernel<<<ceil_div(c.m, 128), 128, 0, c.stream>>>(c.m, c.adj_u.p, c.y.p, g_obj, out_dev);
    CK_LAUNCH();
}

void adjoint_grad_F0(Context &c, dd_t *out_dev) {
    adj_sub_kernel<<<ceil_div(c.space_len, 256), 256, 0, c.stream>>>(c.space_len, nullptr, c.adj_R.buf.p, out_dev);
    CK_LAUNCH();
}

void adjoint_grad_F(Context &c, int k, dd_t *out_dev) {
    dd_t uy[2];
    d2h(c, &uy[0], c.adj_u.p + k, sizeof(dd_t));
    d2h(c, &uy[1], c.y.p + k, sizeof(dd_t));
    adj_grad_F_kernel<<<ceil_div(c.space_len, 256), 256, 0, c.stream>>>(c.space_len, uy[0], uy[1], c.X.buf.p, c.adj_R.buf.p, out_dev);
    CK_LAUNCH();
}

} // namespace sddd
