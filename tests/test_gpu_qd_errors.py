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
