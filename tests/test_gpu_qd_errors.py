"""Errors of the GPU's dd results against a quad-double (qd_real) oracle.

The oracle (oracle/ref_capi.cpp, QD 2.3.23's qd_real, ~212 bits) computes
the same quantities from the same dd inputs, so the difference is the dd
path's own error: the Schur matrix B of the F1 formula, the Cholesky factor
of B in the plain form and in the tensor-core split form, and the solution
of B dy = g through that factor.  Errors are max |dd - qd| over max |qd|;
each test prints what it measured and holds it under a bound written here.
"""
import ctypes

import numpy as np
import pytest

from conftest import DD, load_pkg, ptr
from test_oracle import same

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).cuda()


def from_dev(t, n):
    return t.cpu().numpy().view(DD)[:n].copy()


def maxdiff(ref_lib, dd, qd, lower=0, order=0):
    out = np.zeros(2)
    ref_lib.qd_maxdiff(ctypes.c_long(len(dd)), ptr(np.ascontiguousarray(dd)), ptr(qd), ctypes.c_int(lower), ctypes.c_long(order), ptr(out))
    return out[0] / out[1]


def spd_dd(rng, n, cond):
    """n x n SPD dd matrix (column-major) with condition ~cond: Q diag Q^T
    with log-spaced eigenvalues, entries rounded to doubles (lo = 0)."""
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.logspace(0, -np.log10(cond), n)
    A = (Q * ev) @ Q.T
    A = (A + A.T) / 2
    out = np.zeros(n * n, DD)
    out["hi"] = A.T.ravel()
    return out


def test_schur_matrix_error_against_qd(ref_lib):
    sddd = load_pkg()
    rng = np.random.default_rng(8)
    n, m = 16, 40
    As = rng.standard_normal((m, n, n))
    As = (As + As.transpose(0, 2, 1)) / 2
    iu, ju = np.triu_indices(n)
    k = np.concatenate([np.full(len(iu), q + 1) for q in range(m)])
    val = np.zeros(len(k), DD)
    val["hi"] = np.concatenate([As[q][iu, ju] for q in range(m)])
    b = np.zeros(m, DD)
    b["hi"] = rng.standard_normal(m)
    G = rng.standard_normal((n, n))
    X = np.zeros(n * n, DD)
    X["hi"] = (np.eye(n) + G @ G.T / n).T.ravel()
    H = rng.standard_normal((n, n))
    Z = np.zeros(n * n, DD)
    Z["hi"] = (np.eye(n) + H @ H.T / n).T.ravel()
    with sddd.Context(0) as c:
        c.upload(m, [n], b, k, np.ones_like(k), np.tile(iu + 1, m), np.tile(ju + 1, m), val)
        assert c.set_point(X, np.zeros(m, DD), Z) == 0
        c.call("sddd_schur_build")
        B = c.get("B")
        Zi = c.get("invZ")
    Adense = np.zeros(m * n * n, DD)
    Adense["hi"] = np.concatenate([As[q].T.ravel() for q in range(m)])
    Bq = np.zeros(4 * m * m)
    ref_lib.qd_schur_dense(ctypes.c_long(n), ctypes.c_long(m), ptr(Adense), ptr(X), ptr(Zi), ptr(Bq))
    err = maxdiff(ref_lib, B, Bq)
    print(f"Schur matrix B (F1, n={n}, m={m}) vs qd: {err:.2e}")
    assert err < 1e-30


@pytest.mark.parametrize("cond", [1e4, 1e12])
def test_cholesky_and_solve_errors_against_qd(ref_lib, cond):
    sddd = load_pkg()
    rng = np.random.default_rng(int(np.log10(cond)))
    n = 300
    A = spd_dd(rng, n, cond)
    g = np.zeros(n, DD)
    g["hi"] = rng.standard_normal(n)
    Lq = np.zeros(4 * n * n)
    assert ref_lib.qd_potrf(ctypes.c_long(n), ptr(A), ptr(Lq)) == 0
    xq = np.zeros(4 * n)
    ref_lib.qd_chol_solve(ctypes.c_long(n), ptr(Lq), ptr(g), ptr(xq))
    rows = []
    with sddd.Context(0) as c:
        for slices in (0, 16, 12):
            assert c.L.sddd_set_tc_split(c.h, slices) == 0
            dA, dx = to_dev(A), to_dev(g)
            assert c.L.sddd_Rpotrf(c.h, b"L", n, ctypes.c_void_p(dA.data_ptr()), n) == 0
            assert c.L.sddd_Rtrsv(c.h, b"L", b"N", b"N", n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(dx.data_ptr()), 1) == 0
            assert c.L.sddd_Rtrsv(c.h, b"L", b"T", b"N", n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(dx.data_ptr()), 1) == 0
            # the same factor through sddd_Rpotrs: the two Rtrsv with the
            # split off, the blocked solves (inverted diagonal blocks) on
            dxp = to_dev(g)
            assert c.L.sddd_Rpotrs(c.h, b"L", n, 1, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(dxp.data_ptr()), n) == 0
            L = from_dev(dA, n * n)
            x = from_dev(dx, n)
            xp = from_dev(dxp, n)
            if slices == 0:
                assert same(xp, x)
            eL = maxdiff(ref_lib, L, Lq, lower=1, order=n)
            ex = maxdiff(ref_lib, x, xq)
            exp_ = maxdiff(ref_lib, xp, xq)
            rows.append((slices, eL, ex, exp_))
        c.L.sddd_set_tc_split(c.h, 0)
    for slices, eL, ex, exp_ in rows:
        form = "plain dd" if slices == 0 else f"split, {slices} slices"
        print(f"cond {cond:.0e} order {n}, {form}: factor {eL:.2e}, solve {ex:.2e}, Rpotrs {exp_:.2e}")
    # factor: a backward-stable dd Cholesky is off by ~eps_dd * cond^(1/2)
    # relative (eps_dd = 2^-104 ~ 5e-32); the solve by ~eps_dd * cond
    eps = 2.0 ** -104
    plain, s16, s12 = rows
    assert plain[1] < 100 * eps * np.sqrt(cond) and plain[2] < 100 * eps * cond
    assert s16[1] < 100 * eps * np.sqrt(cond) and s16[2] < 100 * eps * cond
    # the blocked solve of the split form: as accurate as the substitution
    assert s16[3] < 100 * eps * cond
    # 12 slices carry 85 bits: its factor is off by ~2^-84 relative
    assert s12[1] < 100 * 2.0 ** -84 * np.sqrt(cond)


def _exact(v):
    """dd (hi, lo) record -> exact Fraction"""
    from fractions import Fraction
    return Fraction(float(v["hi"])) + Fraction(float(v["lo"]))


def _exact_pair(x):
    """(hi, lo) pair -> exact Fraction"""
    from fractions import Fraction
    return Fraction(x[0]) + Fraction(x[1])


def test_step_length_residual_and_gap_errors(oracle_lib, workdir):
    """At a real iterate (after 8 passes of a two-block problem): the
    step-length eigenvalues lambda_min(L D L^T), the two residual norms, the
    objectives C.X and b.y, X.Z and the relative gap from the GPU, against
    the same formulas evaluated exactly (Python Fractions of the same dd
    inputs; the eigenvalue in 60-digit mpmath), i.e. more accurately than a
    qd_real evaluation.  Bounds: 2^-100 of the summed magnitudes for the
    sums (a dd sum of N terms is off by at most about N 2^-104 of them);
    1e-25 of the spectral radius for the Lanczos eigenvalue."""
    import importlib
    from fractions import Fraction

    import mpmath
    sddd = load_pkg()
    P = importlib.import_module("sdpa_dd_b200.problems")
    import sdpa_problem
    text = P.control_like(sizes=(9, 6), m=25, seed=13)
    path = workdir / "qd_iterate.dat-s"
    path.write_text(text)
    prob = sdpa_problem.Problem(oracle_lib, text)
    par = sddd.param(P.write_param(str(workdir / "qd_iterate.param"), eps=1e-25))
    with sddd.Context(0) as c:
        c.read_problem(path)
        c.call("sddd_solver_start", ctypes.byref(par))
        for _ in range(8):
            assert c.L.sddd_iterate(c.h) == 0
        sizes = c.sizes
        X, Z, y = c.get("X"), c.get("Z"), c.get("y")
        Lx, Dx, Lz, Dz = c.get("invCholX"), c.get("Dx"), c.get("invCholZ"), c.get("Dz")
        eig = [c.dd_scalar("sddd_min_eig", w) for w in (0, 1)]
        rp, rd = sddd.SdddDD(), sddd.SdddDD()
        c.call("sddd_residuals", ctypes.byref(rp), ctypes.byref(rd))
        inner = [c.dd_scalar("sddd_inner", w) for w in (0, 1, 2)]
    offs = np.cumsum([0] + [n * n for n in sizes])

    def blk(a, l):
        return a[offs[l]:offs[l + 1]].reshape(sizes[l], sizes[l]).T  # [row][col]

    def full(mat, n):
        """a problem matrix as an n x n list of Fractions"""
        M = [[Fraction(0)] * n for _ in range(n)]
        if mat["dense"]:
            V = mat["val"].reshape(n, n).T
            for i in range(n):
                for j in range(n):
                    M[i][j] = _exact(V[i, j])
        else:
            for r, cc, v in zip(mat["rows"], mat["cols"], mat["val"]):
                M[r][cc] = M[cc][r] = _exact(v)
        return M

    def dot(M, N, n):
        s, a = Fraction(0), Fraction(0)
        for i in range(n):
            for j in range(n):
                s += M[i][j] * N[i][j]
                a += abs(M[i][j] * N[i][j])
        return s, a

    m = prob.m
    nb = len(sizes)
    Xe = [[[_exact(v) for v in row] for row in blk(X, l)] for l in range(nb)]
    Ze = [[[_exact(v) for v in row] for row in blk(Z, l)] for l in range(nb)]
    ye = [_exact(v) for v in y]
    be = [_exact(v) for v in prob.b]
    A = [[full(prob.A[k][l], sizes[l]) if l in prob.A[k] else None for l in range(nb)] for k in range(m)]
    C = [full(prob.C[l], sizes[l]) if l in prob.C else None for l in range(nb)]
    rows = []
    # objectives and X.Z
    cxs = [dot(C[l], Xe[l], sizes[l]) for l in range(nb) if C[l] is not None]
    cx = (sum(v[0] for v in cxs), sum(v[1] for v in cxs))
    by = (sum(b * v for b, v in zip(be, ye)), sum(abs(b * v) for b, v in zip(be, ye)))
    xzs = [dot(Xe[l], Ze[l], sizes[l]) for l in range(nb)]
    xz = (sum(v[0] for v in xzs), sum(v[1] for v in xzs))
    for name, got, (want, mag) in (("C.X", inner[0], cx), ("b.y", inner[1], by), ("X.Z", inner[2], xz)):
        err = abs(_exact_pair(got) - want)
        rows.append((name, float(err / mag)))
        assert err <= Fraction(2) ** -100 * mag, (name, float(err), float(mag))

    # relative gap (SolveInfo / Phase::updateCheck, sdpa_parts.cpp:890-908)
    def gap(p, d):
        return abs(p - d) / max(Fraction(1), (abs(p) + abs(d)) / 2)
    g_gpu, g_ex = gap(_exact_pair(inner[0]), _exact_pair(inner[1])), gap(cx[0], by[0])
    rows.append(("relative gap", float(abs(g_gpu - g_ex) / max(g_ex, Fraction(1, 10 ** 40)))))
    assert abs(g_gpu - g_ex) <= Fraction(2) ** -99 * (cx[1] + by[1])
    # residual norms (Residuals::compute, sdpa_dataset.cpp:625-645)
    prim, pmag = Fraction(0), Fraction(0)
    for k in range(m):
        s, a = be[k], abs(be[k])
        for l in range(nb):
            if A[k][l] is not None:
                d, am = dot(A[k][l], Xe[l], sizes[l])
                s -= d
                a += am
        prim, pmag = max(prim, abs(s)), max(pmag, a)
    dual, dmag = Fraction(0), Fraction(0)
    for l, n in enumerate(sizes):
        for i in range(n):
            for j in range(n):
                s = (C[l][i][j] if C[l] is not None else Fraction(0)) - Ze[l][i][j]
                a = abs(s) + abs(Ze[l][i][j])
                for k in range(m):
                    if A[k][l] is not None:
                        t = ye[k] * A[k][l][i][j]
                        s -= t
                        a += abs(t)
                dual, dmag = max(dual, abs(s)), max(dmag, a)
    for name, got, want, mag in (("primal residual", (rp.hi, rp.lo), prim, pmag), ("dual residual", (rd.hi, rd.lo), dual, dmag)):
        err = abs(_exact_pair(got) - want)
        rows.append((name, float(err / mag)))
        assert err <= Fraction(2) ** -100 * mag, (name, float(err), float(mag))
    # step-length eigenvalues: lambda_min(L D L^T) over the blocks
    mpmath.mp.dps = 60
    for which, (L_, D_) in enumerate(((Lx, Dx), (Lz, Dz))):
        lam, rad = None, mpmath.mpf(0)
        for l in range(nb):
            Lm = mpmath.matrix([[mpmath.mpf(float(v["hi"])) + mpmath.mpf(float(v["lo"])) for v in row] for row in blk(L_, l)])
            Dm = mpmath.matrix([[mpmath.mpf(float(v["hi"])) + mpmath.mpf(float(v["lo"])) for v in row] for row in blk(D_, l)])
            M = Lm * Dm * Lm.T
            M = (M + M.T) / 2
            ev = mpmath.eigsy(M, eigvals_only=True)
            lo = min(ev)
            lam = lo if lam is None or lo < lam else lam
            rad = max(rad, max(abs(e) for e in ev))
        got = mpmath.mpf(eig[which][0]) + mpmath.mpf(eig[which][1])
        err = abs(got - lam) / rad
        rows.append((f"min eig ({'X' if which == 0 else 'Z'})", float(err)))
        assert err <= mpmath.mpf("1e-25"), (which, float(err))
    for name, e in rows:
        print(f"{name}: error {e:.2e} (relative to the summed magnitudes / spectral radius)")
