"""Adjoint of a finished solve (sddd_adjoint) on the GPU: gradients of the
optimal value c.x and of weighted sums of the solution (x, Y) with respect
to the data c, F_0, F_k.

The reference has no derivative code, so the adjoint is checked against the
solver itself and against duality theory:

* finite differences in dd: a data entry theta moved by multiples of h
  (powers of two, so theta +- j h is exact in dd), every problem solved to
  relative gap 1e-25, combined by a central stencil;
* the envelope theorem: at the optimum d(c.x)/dc = x, d/dF_0 = Y,
  d/dF_k = -x_k Y (the primal is min c.x s.t. sum_k F_k x_k - F_0 >= 0,
  so raising F_0 shrinks the feasible set and the gradient is +Y);
* a torch.autograd.Function whose forward solves and whose backward calls
  the adjoint, as a user of the C ABI would wrap it.

Workloads: the control-shaped two-block construction (dense N(0,1)/sqrt(n)
blocks, feasible by construction): small (blocks 12 and 6, m = 60), medium
(20 and 10, m = 150) and full size (100 and 50, m = 1326), seeds on which
the reference reaches pdOPT at relative gap 1e-25.
"""
import ctypes
import importlib
import tempfile
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import DD, load_pkg

pytestmark = pytest.mark.gpu
getcontext().prec = 60

H = 2.0 ** -40    # ~9.1e-13
H6 = 2.0 ** -14   # ~6.1e-5, the step of the sixth-order stencil
# sixth-order differences vs adjoint, relative to max(1, |grad|): measured
# on B200 1.7e-23 to 1.75e-20 on the small workload (nine entries of c and
# F), up to 5.03e-20 at full size (m = 1326), with every difference point a
# pdOPT solve at relative gap 1e-25.  The differences themselves carry
# ~1e-21 of solve noise (1e-25 / h times the stencil's weights) and cannot
# be sharpened by a tighter gap: at epsilon 1e-28 and 1e-30 these problems
# end in pFEAS / noINFO with iteration counts that vary along the stencil.
FD_TOL = 1e-19
# A solve stops within ~1e-25 of the optimum, at a point that moves
# non-smoothly with the data (iteration counts and step lengths), so a
# difference quotient carries ~1e-25 / h of noise: ~1e-13 at h = 1e-12.
# The sixth-order stencil at h = 6e-5 keeps both that noise (~3e-21) and its
# truncation error (h^6 ~ 5e-26) near 1e-20.
FD2_TOL = 1e-11
# solution gradients (weights on x and Y) vs sixth-order differences:
# measured 2e-18 to 4e-14
SOL_TOL = 1e-12
# central stencils: sum_j coef_j (f(theta + j h) - f(theta - j h)) / (den h)
CENTRAL2 = ([(1, 1)], 2)                      # truncation h^2 f(3) / 6
CENTRAL6 = ([(1, 45), (2, -9), (3, 1)], 60)   # truncation h^6 f(7) / 140

PH = ["noINFO", "pFEAS", "dFEAS", "pdFEAS", "pdINF", "pFEAS_dINF", "pINF_dFEAS", "pdOPT", "pUNBD", "dUNBD"]


def _problems():
    load_pkg()
    return importlib.import_module("sdpa_dd_b200.problems")


def _dec(v):
    return Decimal(float(v["hi"])) + Decimal(float(v["lo"]))


def _two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


class Workload:
    """Dense two-block SDP of the control-shaped construction, held as the
    upload arrays of sddd_upload_problem."""

    def __init__(self, sizes, m, seed):
        P = _problems()
        rng = np.random.default_rng(seed)
        c, F0, Fs = P._dense_blocks(rng, m, list(sizes), scale_by_n=True)
        self.sizes, self.m = list(sizes), m
        ks, bs, iis, jjs, vs = [], [], [], [], []
        self.pos = {}
        base = 0
        for k in range(m + 1):
            for b, n in enumerate(sizes):
                M = F0[b] if k == 0 else Fs[b][k - 1]
                iu, ju = np.triu_indices(n)
                ks.append(np.full(len(iu), k))
                bs.append(np.full(len(iu), b + 1))
                iis.append(iu + 1)
                jjs.append(ju + 1)
                vs.append(M[iu, ju])
                self.pos[(k, b)] = (base, n)
                base += len(iu)
        self.k, self.blk = np.concatenate(ks), np.concatenate(bs)
        self.i, self.j = np.concatenate(iis), np.concatenate(jjs)
        self.val = np.zeros(len(self.k), DD)
        self.val["hi"] = np.concatenate(vs)
        self.b = np.zeros(m, DD)
        self.b["hi"] = c
        self.off = np.concatenate([[0], np.cumsum([n * n for n in sizes])])

    def entry(self, k, b, i, j):
        """Index of F_k's block-b entry (i, j), i <= j, 0-based."""
        base, n = self.pos[(k, b)]
        iu, ju = np.triu_indices(n)
        return base + int(np.nonzero((iu == i) & (ju == j))[0][0])

    def space_index(self, b, i, j):
        return int(self.off[b]) + i + self.sizes[b] * j


def _param(td):
    P = _problems()
    return load_pkg().param(P.write_param(f"{td}/p.sdpa", eps=1e-25, max_iter=200))


def _solve(ctx, w, par, b=None, val=None):
    ctx.upload(w.m, w.sizes, w.b if b is None else b, w.k, w.blk, w.i, w.j, w.val if val is None else val)
    r = ctx.solve(par)
    L = ctx.L.sddd_space_len(ctx.h)
    X, y, Z = np.zeros(L, DD), np.zeros(w.m, DD), np.zeros(L, DD)
    ctx.call("sddd_get_point", X.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p), Z.ctypes.data_as(ctypes.c_void_p))
    return r, X, y, Z


def _obj(r):
    return Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)


def _fd(ctx, w, par, which, h=H, stencil=CENTRAL2):
    """Finite-difference derivative of the optimal value for one data entry:
    which = ('c', k) or ('F', index into the upload arrays)."""
    coefs, den = stencil
    acc, iters = Decimal(0), []
    for j, coef in coefs:
        outs = []
        for sgn in (1.0, -1.0):
            b, val = w.b.copy(), w.val.copy()
            arr, idx = (b, which[1]) if which[0] == "c" else (val, which[1])
            hi, lo = _two_sum(float(arr["hi"][idx]), sgn * j * h)
            arr["hi"][idx], arr["lo"][idx] = hi, lo + float(arr["lo"][idx])
            r, X, y, Z = _solve(ctx, w, par, b, val)
            outs.append(_obj(r))
            iters.append(r.iterations)
        acc += coef * (outs[0] - outs[1])
    return acc / (Decimal(den) * Decimal(h)), iters


def _rel(a, b):
    return float(abs(a - b) / max(Decimal(1), abs(b)))


@pytest.fixture(scope="module")
def small():
    return Workload((12, 6), 60, seed=14)


def _check_envelope(ctx, w, par, tol):
    r, X, y, Z = _solve(ctx, w, par)
    assert PH[r.phase] == "pdOPT", PH[r.phase]
    assert r.relative_gap.hi < 1e-25
    gc, gF0 = ctx.adjoint(g_obj=(1.0, 0.0))
    # d(c.x)/dc = x = -y
    err_c = max(_rel(_dec(gc[k]), -_dec(y[k])) for k in range(w.m))
    # d/dF_0 = Y = X (internal)
    err_F0 = max(_rel(_dec(gF0[e]), _dec(X[e])) for e in range(len(X)))
    # d/dF_k = -x_k Y = y_k X for a few k
    err_F = 0.0
    for k in (1, w.m // 2, w.m):
        g = ctx.adjoint_grad_F(k)
        yk = _dec(y[k - 1])
        err_F = max(err_F, max(_rel(_dec(g[e]), yk * _dec(X[e])) for e in range(0, len(X), 7)))
    print(f"envelope m={w.m}: grad c {err_c:.2e}, grad F0 {err_F0:.2e}, grad F_k {err_F:.2e}; gap {r.relative_gap.hi:.2e}")
    assert err_c < tol and err_F0 < tol and err_F < tol
    return r, X, y, gc, gF0


@pytest.mark.parametrize("sizes,m", [((12, 6), 60), ((20, 10), 150)])
def test_envelope(sizes, m):
    sddd = load_pkg()
    with tempfile.TemporaryDirectory() as td, sddd.Context(0) as ctx:
        _check_envelope(ctx, Workload(sizes, m, seed=14), _param(td), 1e-19)


def _value_cases(ctx, w, gc, gF0):
    """(kind, index, adjoint gradient) for entries of c, F_0 and F_k; an
    off-diagonal entry (i, j) listed once moves F_ij and F_ji: 2 G_ij."""
    cases = [("c", 0, _dec(gc[0])), ("c", w.m - 1, _dec(gc[w.m - 1]))]
    for (b, i, j) in ((0, 3, 3), (0, 2, 9), (1, 0, 5)):
        cases.append(("F", w.entry(0, b, i, j), _dec(gF0[w.space_index(b, i, j)]) * (1 if i == j else 2)))
    for k, (b, i, j) in ((4, (0, 1, 1)), (22, (1, 2, 4))):
        gk = ctx.adjoint_grad_F(k)
        cases.append(("F", w.entry(k, b, i, j), _dec(gk[w.space_index(b, i, j)]) * (1 if i == j else 2)))
    return cases


@pytest.mark.parametrize("order", [6, 2])
def test_optimal_value_gradient_vs_differences(small, order):
    """Sixth order at h = 2^-14 to FD_TOL; second order at h = 2^-40
    (~1e-12) to its noise floor."""
    sddd = load_pkg()
    w = small
    h, stencil, tol = (H6, CENTRAL6, FD_TOL) if order == 6 else (H, CENTRAL2, FD2_TOL)
    with tempfile.TemporaryDirectory() as td, sddd.Context(0) as ctx:
        par = _param(td)
        _solve(ctx, w, par)
        gc, gF0 = ctx.adjoint(g_obj=(1.0, 0.0))
        worst = 0.0
        for kind, idx, g in _value_cases(ctx, w, gc, gF0):
            fd, iters = _fd(ctx, w, par, (kind, idx), h, stencil)
            e = _rel(fd, g)
            print(f"FD{order} {kind}[{idx}] iters {iters}: adjoint {float(g):+.16e} fd {float(fd):+.16e} rel {e:.2e}")
            worst = max(worst, e)
        assert worst < tol


def _weighted(gx, gY, y, X):
    """g_x . x + g_Y . Y with x = -y and Y the internal X, in decimals."""
    s = Decimal(0)
    for a, v in zip(gx, y):
        if a:
            s -= Decimal(float(a)) * _dec(v)
    for a, v in zip(gY, X):
        if a:
            s += Decimal(float(a)) * _dec(v)
    return s


def _fd_f(ctx, w, par, which, f, h, stencil):
    """Finite-difference derivative of f(r, X, y) of the solution."""
    coefs, den = stencil
    acc = Decimal(0)
    for j, coef in coefs:
        outs = []
        for sgn in (1.0, -1.0):
            b, val = w.b.copy(), w.val.copy()
            arr, idx = (b, which[1]) if which[0] == "c" else (val, which[1])
            hi, lo = _two_sum(float(arr["hi"][idx]), sgn * j * h)
            arr["hi"][idx], arr["lo"][idx] = hi, lo + float(arr["lo"][idx])
            r, X, y, Z = _solve(ctx, w, par, b, val)
            outs.append(f(r, X, y))
        acc += coef * (outs[0] - outs[1])
    return acc / (Decimal(den) * Decimal(h))


@pytest.mark.parametrize("sizes,m", [((12, 6), 60), ((20, 10), 150)])
def test_solution_gradient_vs_sixth_order_differences(sizes, m):
    """Weights on the solution: f = g_x . x + g_Y . Y (random dyadic g_x,
    symmetric g_Y), gradients with respect to entries of c, F_0 and F_k."""
    sddd = load_pkg()
    w = Workload(sizes, m, seed=14)
    rng = np.random.default_rng(5)
    with tempfile.TemporaryDirectory() as td, sddd.Context(0) as ctx:
        par = _param(td)
        r, X, y, Z = _solve(ctx, w, par)
        gx = np.round(rng.standard_normal(w.m) * 8) / 8
        gY = np.zeros(len(X))
        for b_, n in enumerate(w.sizes):
            S = np.round(rng.standard_normal((n, n)) * 8) / 8
            gY[int(w.off[b_]):int(w.off[b_ + 1])] = ((S + S.T) / 2).reshape(-1, order="F")
        gxd, gYd = np.zeros(w.m, DD), np.zeros(len(gY), DD)
        gxd["hi"], gYd["hi"] = gx, gY
        gc, gF0 = ctx.adjoint(g_x=gxd, g_Y=gYd)
        cases = [("c", 3, _dec(gc[3])), ("c", w.m - 1, _dec(gc[w.m - 1])),
                 ("F", w.entry(0, 0, 4, 4), _dec(gF0[w.space_index(0, 4, 4)])),
                 ("F", w.entry(0, 1, 1, 3), 2 * _dec(gF0[w.space_index(1, 1, 3)]))]
        gk = ctx.adjoint_grad_F(7)
        cases.append(("F", w.entry(7, 0, 2, 5), 2 * _dec(gk[w.space_index(0, 2, 5)])))
        worst = 0.0
        for kind, idx, g in cases:
            fd = _fd_f(ctx, w, par, (kind, idx), lambda r_, X_, y_: _weighted(gx, gY, y_, X_), H6, CENTRAL6)
            e = _rel(fd, g)
            print(f"solution FD6 m={w.m} {kind}[{idx}]: adjoint {float(g):+.16e} fd {float(fd):+.16e} rel {e:.2e}")
            worst = max(worst, e)
        assert worst < SOL_TOL


def test_torch_autograd_function(small):
    """The adjoint behind torch.autograd: gradients of c.x with respect to
    (c, F_0) from backward() equal the envelope gradient (x, Y)."""
    torch = pytest.importorskip("torch")
    sddd = load_pkg()
    w = small

    class SdpValue(torch.autograd.Function):
        @staticmethod
        def forward(fctx, c, F0_entries):
            b, val = w.b.copy(), w.val.copy()
            b["hi"] = c.detach().cpu().numpy()
            val["hi"][:F0_entries.numel()] = F0_entries.detach().cpu().numpy()
            r, X, y, Z = _solve(ctx, w, par, b, val)
            return torch.tensor(r.objValPrimal.hi, dtype=torch.float64)

        @staticmethod
        def backward(fctx, g):
            gc, gF0 = ctx.adjoint(g_obj=(float(g), 0.0))
            # F_0's upload entries are its upper triangles, block by block
            ge = []
            for b_, n in enumerate(w.sizes):
                iu, ju = np.triu_indices(n)
                G = gF0["hi"][int(w.off[b_]):int(w.off[b_ + 1])].reshape(n, n, order="F")
                ge.append(G[iu, ju] * np.where(iu == ju, 1.0, 2.0))
            return torch.from_numpy(gc["hi"].copy()), torch.from_numpy(np.concatenate(ge))

    with tempfile.TemporaryDirectory() as td, sddd.Context(0) as ctx:
        par = _param(td)
        n0 = sum(n * (n + 1) // 2 for n in w.sizes)
        c = torch.tensor(w.b["hi"], dtype=torch.float64, requires_grad=True)
        F0e = torch.tensor(w.val["hi"][:n0], dtype=torch.float64, requires_grad=True)
        v = SdpValue.apply(c, F0e)
        v.backward()
        r, X, y, Z = _solve(ctx, w, par)
        assert np.allclose(c.grad.numpy(), -y["hi"], rtol=1e-13, atol=1e-13)
        want = []
        for b_, n in enumerate(w.sizes):
            iu, ju = np.triu_indices(n)
            Y = X["hi"][int(w.off[b_]):int(w.off[b_ + 1])].reshape(n, n, order="F")
            want.append(Y[iu, ju] * np.where(iu == ju, 1.0, 2.0))
        assert np.allclose(F0e.grad.numpy(), np.concatenate(want), rtol=1e-13, atol=1e-13)


def test_control_full_size_envelope_and_differences():
    """The full control-shaped workload (blocks 100 and 50, m = 1326)."""
    sddd = load_pkg()
    w = Workload((100, 50), 1326, seed=3)
    with tempfile.TemporaryDirectory() as td, sddd.Context(0) as ctx:
        par = _param(td)
        r, X, y, gc, gF0 = _check_envelope(ctx, w, par, 2e-18)
        cases = [("c", 0, _dec(gc[0])), ("F", w.entry(0, 0, 7, 7), _dec(gF0[w.space_index(0, 7, 7)])),
                 ("F", w.entry(0, 1, 3, 20), 2 * _dec(gF0[w.space_index(1, 3, 20)]))]
        worst = 0.0
        for kind, idx, g in cases:
            fd, iters = _fd(ctx, w, par, (kind, idx), H6, CENTRAL6)
            e = _rel(fd, g)
            print(f"control FD6 {kind}[{idx}] iters {iters}: adjoint {float(g):+.16e} fd {float(fd):+.16e} rel {e:.2e}")
            worst = max(worst, e)
        assert worst < FD_TOL
