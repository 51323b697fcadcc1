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

#include <algorithm>
#include <cmath>
#include <vector>

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
    solve_B(c, c.adj_u.p);
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

// ------------------------------------------------ the limit at the optimum
// The iterate the solver stops at is off the central path, and there the
// HKM form couples the range R and null space N of X by the average of
// lambda_R/omega_N and lambda_N/omega_R, which agree only on the path: the
// solution gradients come out wrong by O(1) (the optimal value's gradient
// is unaffected).  adjoint_limit linearises at exactly central points built
// from the iterate's spectral data instead.  With X = Q diag(Lambda) Q^T
// (cyclic Jacobi in dd), R = {lambda > 1e-12 max lambda}, Q = [Q_R Q_N] and
// K = (Q_N^T Z Q_N)^-1:
//     X_c = Q diag(Lambda_R, mu K) Q^T,   Z_c^-1 = Q diag(Lambda_R / mu, K) Q^T,
// so X_c Z_c = mu I exactly; the HKM adjoint there is exact for the
// central path through (X_c, Z_c), and as mu -> 0 it tends to the
// derivative at the optimum (the RR block becomes a constraint, the RN
// coupling lambda_R / omega_N).  It is evaluated at mu = h, 2h, 4h
// (h = 1e-8 max lambda) and extrapolated, (8 g(h) - 6 g(2h) + g(4h)) / 3,
// which removes the h and h^2 terms; the 1/mu scale of the RR block costs
// ~1e-32 / h of rounding.

constexpr int JAC_THREADS = 256;
constexpr int JAC_MAX_N = 1024;
constexpr int JAC_MAX_SWEEPS = 40;

__device__ __forceinline__ int jac_elem(int pos, int r, int np) { return pos == 0 ? 0 : 1 + (pos - 1 + r) % (np - 1); }

// Cyclic Jacobi with the round-robin ordering (n/2 disjoint rotations per
// round, every pair once per sweep; Golub & Van Loan, Matrix Computations,
// the parallel Jacobi method): A (one symmetric block per CTA, overwritten)
// -> diagonal, Q -> eigenvectors (A_0 = Q diag Q^T).  Rotation for (p, q):
// tau = (a_qq - a_pp) / (2 a_pq), t = sign(tau) / (|tau| + sqrt(1 + tau^2)),
// c = 1 / sqrt(1 + t^2), s = t c; A <- J^T A J, Q <- Q J.  Stops when the
// off-diagonal mass is below 1e-56 of the diagonal's (in squares: 1e-28 in
// norm, above the dd rounding floor of ~n 1e-32) or after JAC_MAX_SWEEPS
// sweeps; sweeps[block] gets the count used.
__global__ void __launch_bounds__(JAC_THREADS) jacobi_kernel(const int *sizes, const long *off, dd_t *A, dd_t *Q, int *sweeps, double *offr) {
    const int l = blockIdx.x, n = sizes[l], tid = threadIdx.x, nt = blockDim.x;
    dd_t *a = A + off[l], *q = Q + off[l];
    __shared__ double2 cs_c[JAC_MAX_N / 2], cs_s[JAC_MAX_N / 2];
    __shared__ double red0[JAC_THREADS], red1[JAC_THREADS];
    for (long e = tid; e < (long)n * n; e += nt) st_dd(q + e, (e % n == e / n) ? dd_from(1.0) : dd_zero());
    const int np = (n + 1) & ~1, half = np / 2;
    int sweep = 0;
    __syncthreads();
    for (; sweep < JAC_MAX_SWEEPS; ++sweep) {
        double o = 0.0, d = 0.0;
        for (long e = tid; e < (long)n * n; e += nt) {
            const double v = a[e].hi;
            if (e % n == e / n) d += v * v;
            else o += v * v;
        }
        red0[tid] = o;
        red1[tid] = d;
        __syncthreads();
        for (int w = nt / 2; w > 0; w >>= 1) {
            if (tid < w) {
                red0[tid] += red0[tid + w];
                red1[tid] += red1[tid + w];
            }
            __syncthreads();
        }
        const bool done = red0[0] <= 1e-56 * red1[0];
        if (tid == 0) offr[l] = red1[0] > 0.0 ? red0[0] / red1[0] : red0[0];
        __syncthreads();
        if (done || n < 2) break;
        for (int r = 0; r < np - 1; ++r) {
            for (int k = tid; k < half; k += nt) {
                const int p = jac_elem(k, r, np), qq = jac_elem(np - 1 - k, r, np);
                dd_t c = dd_from(1.0), sn = dd_zero();
                if (p < n && qq < n) {
                    const dd_t apq = ld_dd(a + p + (long)n * qq), app = ld_dd(a + p + (long)n * p), aqq = ld_dd(a + qq + (long)n * qq);
                    // a_pq below 1e-36 of sqrt(|a_pp a_qq|) is already zero
                    // at dd precision: no rotation (entries deep in a
                    // near-null space would otherwise shrink into the
                    // denormals, where tau^2 overflows)
                    if (fabs(apq.hi) > 1e-36 * sqrt(fabs(app.hi) * fabs(aqq.hi)) && fabs(apq.hi) > 1e-250) {
                        const dd_t tau = dd_div(dd_sub(aqq, app), dd_mul_d(apq, 2.0));
                        dd_t t;
                        if (fabs(tau.hi) < 1e100) {
                            const dd_t root = dd_sqrt(dd_add(dd_from(1.0), dd_sqr(tau)));
                            t = dd_div(dd_from(1.0), dd_add(dd_abs(tau), root));
                        } else {
                            t = dd_div(dd_from(0.5), dd_abs(tau)); // 1 / (|tau| + sqrt(1 + tau^2)) to dd precision
                        }
                        if (tau.hi < 0.0) t = dd_neg(t);
                        c = dd_div(dd_from(1.0), dd_sqrt(dd_add(dd_from(1.0), dd_sqr(t))));
                        sn = dd_mul(t, c);
                    }
                }
                cs_c[k] = make_double2(c.hi, c.lo);
                cs_s[k] = make_double2(sn.hi, sn.lo);
            }
            __syncthreads();
            // columns p, q of A and Q: (x_p, x_q) <- (c x_p - s x_q, s x_p + c x_q)
            for (long w = tid; w < (long)half * n; w += nt) {
                const int k = (int)(w / n), i = (int)(w % n);
                const int p = jac_elem(k, r, np), qq = jac_elem(np - 1 - k, r, np);
                if (p >= n || qq >= n) continue;
                const dd_t c = dd_make(cs_c[k].x, cs_c[k].y), sn = dd_make(cs_s[k].x, cs_s[k].y);
                for (int mtx = 0; mtx < 2; ++mtx) {
                    dd_t *m = mtx ? q : a;
                    const dd_t xp = ld_dd(m + i + (long)n * p), xq = ld_dd(m + i + (long)n * qq);
                    st_dd(m + i + (long)n * p, dd_sub(dd_mul(c, xp), dd_mul(sn, xq)));
                    st_dd(m + i + (long)n * qq, dd_add(dd_mul(sn, xp), dd_mul(c, xq)));
                }
            }
            __syncthreads();
            // rows p, q of A
            for (long w = tid; w < (long)half * n; w += nt) {
                const int k = (int)(w / n), j = (int)(w % n);
                const int p = jac_elem(k, r, np), qq = jac_elem(np - 1 - k, r, np);
                if (p >= n || qq >= n) continue;
                const dd_t c = dd_make(cs_c[k].x, cs_c[k].y), sn = dd_make(cs_s[k].x, cs_s[k].y);
                const dd_t xp = ld_dd(a + p + (long)n * j), xq = ld_dd(a + qq + (long)n * j);
                st_dd(a + p + (long)n * j, dd_sub(dd_mul(c, xp), dd_mul(sn, xq)));
                st_dd(a + qq + (long)n * j, dd_add(dd_mul(sn, xp), dd_mul(c, xq)));
            }
            __syncthreads();
            // the pair's entry is zero after its rotation (or was negligible)
            for (int k = tid; k < half; k += nt) {
                const int p = jac_elem(k, r, np), qq = jac_elem(np - 1 - k, r, np);
                if (p < n && qq < n) {
                    st_dd(a + p + (long)n * qq, dd_zero());
                    st_dd(a + qq + (long)n * p, dd_zero());
                }
            }
            __syncthreads();
        }
    }
    if (tid == 0) sweeps[l] = sweep;
}

// Qp(:, j) = Q(:, perm[j]) per block.
__global__ void permute_cols_kernel(int n, const int *perm, const dd_t *Q, dd_t *Qp) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    st_dd(Qp + e, ld_dd(Q + i + (long)n * perm[j]));
}

// Kb (nN x nN) = T(r.., r..) of an n x n matrix.
__global__ void copy_nn_kernel(int n, int r, const dd_t *T, dd_t *Kb) {
    const int nN = n - r;
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)nN * nN) return;
    const int i = (int)(e % nN), j = (int)(e / nN);
    st_dd(Kb + e, ld_dd(T + (r + i) + (long)n * (r + j)));
}

// The middle factor: x_mode: diag(lam_R) (+) mu K;  otherwise diag(lam_R / mu) (+) K.
__global__ void central_mid_kernel(int n, int r, const dd_t *lam, const dd_t *K, dd_t mu, int x_mode, dd_t *M) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    dd_t v = dd_zero();
    if (i < r && j < r) {
        if (i == j) v = x_mode ? ld_dd(lam + i) : dd_div(ld_dd(lam + i), mu);
    } else if (i >= r && j >= r) {
        const dd_t kv = ld_dd(K + (i - r) + (long)(n - r) * (j - r));
        v = x_mode ? dd_mul(mu, kv) : kv;
    }
    st_dd(M + e, v);
}

// out = (8 a - 6 b + c) / 3: Richardson's extrapolation to mu -> 0 from
// values at h, 2h, 4h with errors c1 mu + c2 mu^2 + O(mu^3).
__global__ void richardson3_kernel(long n, const dd_t *a, const dd_t *b, const dd_t *c, dd_t *out) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const dd_t v = dd_add(dd_sub(dd_mul_d(ld_dd(a + e), 8.0), dd_mul_d(ld_dd(b + e), 6.0)), ld_dd(c + e));
    st_dd(out + e, dd_div_d(v, 3.0));
}

int adjoint_limit(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj) {
    cudaStream_t st = c.stream;
    const long L = c.space_len;
    for (int l = 0; l < c.nSDP; ++l)
        if (c.sizes[l] > JAC_MAX_N) throw Error(ERR_UNSUPPORTED, "adjoint: SDP blocks above order 1024 are not supported");
    Space *sp[] = {&c.lim_Q, &c.lim_Qp, &c.lim_T, &c.lim_M, &c.lim_Xs, &c.lim_Zs, &c.lim_R[0], &c.lim_R[1], &c.lim_R[2]};
    for (Space *x : sp) x->buf.alloc(L);
    for (auto &u : c.lim_u) u.alloc(c.m);
    c.lim_sweeps.alloc(c.nSDP);
    c.lim_offr.alloc(c.nSDP);
    // X = Q diag(lambda) Q^T, blockwise
    CK(cudaMemcpyAsync(c.lim_T.buf.p, c.X.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    jacobi_kernel<<<c.nSDP, JAC_THREADS, 0, st>>>(c.d_sizes.p, c.d_off.p, c.lim_T.buf.p, c.lim_Q.buf.p, c.lim_sweeps.p, c.lim_offr.p);
    CK_LAUNCH();
    std::vector<dd_t> T(L);
    d2h(c, T.data(), c.lim_T.buf.p, sizeof(dd_t) * L);
    std::vector<int> sweeps(c.nSDP);
    std::vector<double> offr(c.nSDP);
    d2h(c, sweeps.data(), c.lim_sweeps.p, sizeof(int) * c.nSDP);
    d2h(c, offr.data(), c.lim_offr.p, sizeof(double) * c.nSDP);
    for (int l = 0; l < c.nSDP; ++l)
        if (sweeps[l] >= JAC_MAX_SWEEPS)
            throw Error(ERR_NOCONV, "adjoint: the eigenvalues of X (block " + std::to_string(l + 1) + ", order " + std::to_string(c.sizes[l]) +
                                        ") did not converge: off-diagonal mass " + std::to_string(offr[l]) + " of the diagonal's");
    double lmax = 0.0;
    for (int l = 0; l < c.nSDP; ++l)
        for (int i = 0; i < c.sizes[l]; ++i) lmax = std::max(lmax, std::fabs(T[c.off[l] + i + (long)c.sizes[l] * i].hi));
    if (!(lmax > 0.0)) throw Error(ERR_STATE, "adjoint: X is zero");
    // per block: R first (descending lambda), the order and lambda_R
    std::vector<int> rk(c.nSDP), perm_all;
    std::vector<long> poff(c.nSDP + 1, 0), koff(c.nSDP + 1, 0);
    std::vector<dd_t> lam_all;
    for (int l = 0; l < c.nSDP; ++l) {
        const int n = c.sizes[l];
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) idx[i] = i;
        auto lam = [&](int i) { return T[c.off[l] + i + (long)n * i]; };
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return lam(a).hi > lam(b).hi; });
        int r = 0;
        while (r < n && lam(idx[r]).hi > 1e-12 * lmax) ++r;
        rk[l] = r;
        for (int i : idx) {
            perm_all.push_back(i);
            lam_all.push_back(lam(i));
        }
        poff[l + 1] = poff[l] + n;
        koff[l + 1] = koff[l] + (long)(n - r) * (n - r);
    }
    c.lim_perm.upload(perm_all, st);
    c.lim_lam.upload(lam_all, st);
    c.lim_K.alloc(std::max<long>(1, koff[c.nSDP]));
    c.lim_Kw.alloc(std::max<long>(1, koff[c.nSDP]));
    // Q_p = Q permuted; K = (Q_N^T Z Q_N)^-1 per block
    CK(cudaMemsetAsync(c.info.p, 0, sizeof(int), st));
    for (int l = 0; l < c.nSDP; ++l) {
        const int n = c.sizes[l], r = rk[l], nN = n - r;
        const long nn = (long)n * n;
        dd_t *Qp = c.lim_Qp.blk(c.off, l);
        permute_cols_kernel<<<ceil_div(nn, 256), 256, 0, st>>>(n, c.lim_perm.p + poff[l], c.lim_Q.blk(c.off, l), Qp);
        CK_LAUNCH();
        if (nN == 0) continue;
        gemm(st, 'N', 'N', GEMM_STORE, n, n, n, c.Z.blk(c.off, l), n, 0, Qp, n, 0, c.lim_M.blk(c.off, l), n, 0, 1, false);
        gemm(st, 'T', 'N', GEMM_STORE, n, n, n, Qp, n, 0, c.lim_M.blk(c.off, l), n, 0, c.lim_T.blk(c.off, l), n, 0, 1, false);
        dd_t *Kb = c.lim_Kw.p + koff[l];
        copy_nn_kernel<<<ceil_div((long)nN * nN, 256), 256, 0, st>>>(n, r, c.lim_T.blk(c.off, l), Kb);
        CK_LAUNCH();
        potrf(st, Kb, nN, nN, c.info.p, c.rdiag.p);
        zero_upper(st, Kb, nN, nN);
        inv_lower(st, Kb, nN, nN, c.lim_T.blk(c.off, l), nN);
        trmm_lt(st, c.lim_T.blk(c.off, l), nN, nN, c.lim_K.p + koff[l], nN);
    }
    int info = 0;
    d2h(c, &info, c.info.p, sizeof(int));
    if (potrf_info_check(info) != 0) throw Error(ERR_STATE, "adjoint: Z is not positive definite on the null space of X");
    // the originals, restored at the end
    CK(cudaMemcpyAsync(c.lim_Xs.buf.p, c.X.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c.lim_Zs.buf.p, c.invZ.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    const double h = 1e-8 * lmax;
    int rc = 0;
    for (int s = 0; s < 3 && rc == 0; ++s) {
        const dd_t mu = dd_from(h * (double)(1 << s));
        for (int l = 0; l < c.nSDP; ++l) {
            const int n = c.sizes[l], r = rk[l];
            const long nn = (long)n * n;
            const dd_t *Qp = c.lim_Qp.blk(c.off, l);
            for (int xm = 1; xm >= 0; --xm) {
                Space &dst = xm ? c.X : c.invZ;
                central_mid_kernel<<<ceil_div(nn, 256), 256, 0, st>>>(n, r, c.lim_lam.p + poff[l], c.lim_K.p + koff[l], mu, xm,
                                                                      c.lim_M.blk(c.off, l));
                CK_LAUNCH();
                gemm(st, 'N', 'N', GEMM_STORE, n, n, n, Qp, n, 0, c.lim_M.blk(c.off, l), n, 0, c.lim_T.blk(c.off, l), n, 0, 1, false);
                gemm(st, 'N', 'T', GEMM_STORE, n, n, n, c.lim_T.blk(c.off, l), n, 0, Qp, n, 0, dst.blk(c.off, l), n, 0, 1, false);
                symmetrize(st, dst.blk(c.off, l), n);
            }
        }
        rc = adjoint(c, g_x, g_Y, g_X, g_obj);
        if (rc == 0) {
            CK(cudaMemcpyAsync(c.lim_u[s].p, c.adj_u.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(c.lim_R[s].buf.p, c.adj_R.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
        }
    }
    CK(cudaMemcpyAsync(c.X.buf.p, c.lim_Xs.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c.invZ.buf.p, c.lim_Zs.buf.p, sizeof(dd_t) * L, cudaMemcpyDeviceToDevice, st));
    if (rc != 0) {
        c.adj_valid = false;
        stream_sync(c);
        return rc;
    }
    richardson3_kernel<<<ceil_div((long)c.m, 256), 256, 0, st>>>(c.m, c.lim_u[0].p, c.lim_u[1].p, c.lim_u[2].p, c.adj_u.p);
    CK_LAUNCH();
    richardson3_kernel<<<ceil_div(L, 256), 256, 0, st>>>(L, c.lim_R[0].buf.p, c.lim_R[1].buf.p, c.lim_R[2].buf.p, c.adj_R.buf.p);
    CK_LAUNCH();
    stream_sync(c);
    c.adj_valid = true;
    return 0;
}

// out = a + b (dd, n entries)
__global__ void add_kernel(long n, const dd_t *a, const dd_t *b, dd_t *out) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    st_dd(out + e, dd_add(ld_dd(a + e), ld_dd(b + e)));
}

int adjoint_combined(Context &c, const dd_t *g_x, const dd_t *g_Y, const dd_t *g_X, dd_t g_obj) {
    const bool sol = g_x || g_Y || g_X, val = !dd_is_zero(g_obj);
    if (!sol) return adjoint(c, nullptr, nullptr, nullptr, g_obj);
    int rc = adjoint_limit(c, g_x, g_Y, g_X, dd_zero());
    if (rc != 0 || !val) return rc;
    // the solution part (limit) kept aside while the value part runs at the iterate
    CK(cudaMemcpyAsync(c.lim_u[0].p, c.adj_u.p, sizeof(dd_t) * c.m, cudaMemcpyDeviceToDevice, c.stream));
    CK(cudaMemcpyAsync(c.lim_R[0].buf.p, c.adj_R.buf.p, sizeof(dd_t) * c.space_len, cudaMemcpyDeviceToDevice, c.stream));
    rc = adjoint(c, nullptr, nullptr, nullptr, g_obj);
    if (rc != 0) return rc;
    add_kernel<<<ceil_div((long)c.m, 256), 256, 0, c.stream>>>(c.m, c.adj_u.p, c.lim_u[0].p, c.adj_u.p);
    CK_LAUNCH();
    add_kernel<<<ceil_div(c.space_len, 256), 256, 0, c.stream>>>(c.space_len, c.adj_R.buf.p, c.lim_R[0].buf.p, c.adj_R.buf.p);
    CK_LAUNCH();
    stream_sync(c);
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
