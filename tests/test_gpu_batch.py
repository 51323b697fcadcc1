"""Batches of independent problems (sddd_batch_*) on the GPU.

A batch solves each problem with the ordinary solver in its own worker
context, so every problem's iterates are those of a single sddd_solve: the
test requires identical phases, iteration counts and dd bits of the
objectives, of X, y, Z and of the gradient of the optimal value with
respect to c (sddd_adjoint), problem by problem.  The workload is the
batched construction at small sizes (dense random SDPs of uneven order and
constraint count) and one problem with an LP block, plus one problem whose
gradient cannot be formed (a constraint with a zero matrix: the Schur
matrix is singular, the solve stops at its first factorisation and the
adjoint refuses), which must fail alone.
"""
import ctypes
import importlib

import numpy as np
import pytest

from conftest import DD, load_pkg

pytestmark = pytest.mark.gpu


def _problems():
    load_pkg()
    return importlib.import_module("sdpa_dd_b200.problems")


def _same(a, b):
    a, b = np.ascontiguousarray(a).view(np.float64).copy(), np.ascontiguousarray(b).view(np.float64).copy()
    a[a == 0] = 0.0
    b[b == 0] = 0.0
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


LP_PROBLEM = '"one LP block"\n1 = mDIM\n1 = nBLOCK\n-2 = bLOCKsTRUCT\n{1}\n0 1 1 1 1.0\n1 1 1 1 1.0\n1 1 2 2 1.0\n'


# min x1 + x2 s.t. x1 I - I >= 0 with F_2 = 0: B has a zero row and column
ZERO_CONSTRAINT = '"a zero constraint"\n2 = mDIM\n1 = nBLOCK\n2 = bLOCKsTRUCT\n{1, 1}\n0 1 1 1 1.0\n0 1 2 2 1.0\n1 1 1 1 1.0\n1 1 2 2 1.0\n'


def test_batch_matches_single_solves(tmp_path):
    sddd = load_pkg()
    P = _problems()
    rng = np.random.default_rng(44)
    cases = []
    for q in range(12):
        n, m = int(rng.integers(10, 31)), int(rng.integers(20, 61))
        path = tmp_path / f"b{q}.dat-s"
        path.write_text(P.dense_random(n, m, seed=1000 + q))
        cases.append((path, n, m))
    lp = tmp_path / "lp.dat-s"
    lp.write_text(LP_PROBLEM)
    cases.append((lp, None, 1))  # block space: two order-1 blocks
    zero = tmp_path / "zero.dat-s"
    zero.write_text(ZERO_CONSTRAINT)
    par = sddd.param(P.write_param(str(tmp_path / "p.sdpa"), eps=1e-25, max_iter=100))
    with sddd.Batch(0, workers=5) as bt:
        for path, n, m in cases[:6]:
            bt.add_file(path, m, n * n)
        bad = bt.add_file(zero, 2, 4)
        for path, n, m in cases[6:]:
            bt.add_file(path, m, 2 if n is None else n * n)
        res = (sddd.SdddResult * len(bt.dims))()
        rc = bt.L.sddd_batch_solve(bt.h, ctypes.byref(par), 1, ctypes.cast(res, ctypes.c_void_p))
        assert rc == 0
        # the solve ended at its first Schur factorisation (stop reason 2);
        # the gradient was refused (a positive status: the factor's failing
        # column), for this problem alone
        assert bt.status(bad) > 0 and res[bad].stop_reason == 2
        idx = [q for q in range(len(bt.dims)) if q != bad]
        for q, (path, n, m) in zip(idx, cases):
            assert bt.status(q) == 0, q
            r = res[q]
            Xb, yb, Zb = bt.point(q)
            gb = bt.grad_c(q)
            with sddd.Context(0) as c:
                c.read_problem(path)
                rs = c.solve(par)
                L = c.L.sddd_space_len(c.h)
                X, y, Z = np.zeros(L, DD), np.zeros(m, DD), np.zeros(L, DD)
                c.call("sddd_get_point", X.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p), Z.ctypes.data_as(ctypes.c_void_p))
                gs, _ = c.adjoint(g_obj=(1.0, 0.0))
            assert (r.phase, r.iterations, r.stop_reason) == (rs.phase, rs.iterations, rs.stop_reason), q
            assert (r.objValPrimal.hi, r.objValPrimal.lo, r.objValDual.hi, r.objValDual.lo) == (
                rs.objValPrimal.hi, rs.objValPrimal.lo, rs.objValDual.hi, rs.objValDual.lo), q
            assert _same(Xb, X) and _same(yb, y) and _same(Zb, Z), q
            assert _same(gb, gs), q


def test_batch_gradient_is_the_envelope(tmp_path):
    """The batched gradient of c.x with respect to c is x = -y at the
    optimum (to the gap)."""
    sddd = load_pkg()
    P = _problems()
    par = sddd.param(P.write_param(str(tmp_path / "p.sdpa"), eps=1e-25, max_iter=100))
    with sddd.Batch(0) as bt:
        for q, (n, m) in enumerate(((12, 30), (20, 45), (15, 25))):
            path = tmp_path / f"e{q}.dat-s"
            path.write_text(P.dense_random(n, m, seed=2000 + q))
            bt.add_file(path, m, n * n)
        res = bt.solve(par, with_grad=True)
        for q in range(3):
            if sddd.PHASES[res[q].phase] != "pdOPT":
                continue
            X, y, Z = bt.point(q)
            g = bt.grad_c(q)
            err = np.abs((g["hi"] + y["hi"]) + (g["lo"] + y["lo"])).max() / max(1.0, np.abs(y["hi"]).max())
            assert err < 1e-18, (q, err)


def test_batched_core_matches_per_problem_core(tmp_path):
    """The batched Newton core (one captured CUDA graph per gathering of
    the workers' problems: batched F/G products, tiled pair products in the
    autotuned shape of each size class, one-CTA Cholesky per problem) gives
    every problem the bits the per-problem kernels give it: the same batch
    solved with the core on and off agrees in phase, iteration count,
    objectives and X, y, Z, problem by problem."""
    sddd = load_pkg()
    P = _problems()
    rng = np.random.default_rng(77)
    cases = []
    for q in range(18):
        n, m = int(rng.integers(10, 41)), int(rng.integers(20, 161))  # size classes m <= 64, <= 128, <= 256
        path = tmp_path / f"c{q}.dat-s"
        path.write_text(P.dense_random(n, m, seed=3000 + q))
        cases.append((path, n, m))
    par = sddd.param(P.write_param(str(tmp_path / "p.sdpa"), eps=1e-25, max_iter=100))
    out = {}
    for core in (1, 0):
        with sddd.Batch(0, workers=8) as bt:
            assert bt.L.sddd_batch_set_core(bt.h, core) == 0
            for path, n, m in cases:
                bt.add_file(path, m, n * n)
            res = bt.solve(par, with_grad=False)
            pts = [bt.point(q) for q in range(len(cases))]
            tuning = bt.L.sddd_batch_tuning(bt.h).decode()
            out[core] = (res, pts, tuning)
    (r1, p1, tuning), (r0, p0, _) = out[1], out[0]
    print("batched core tile shapes:", tuning)
    assert "m<=64" in tuning and "m<=128" in tuning
    for q in range(len(cases)):
        a, b = r1[q], r0[q]
        assert (a.phase, a.iterations, a.stop_reason) == (b.phase, b.iterations, b.stop_reason), q
        assert (a.objValPrimal.hi, a.objValPrimal.lo, a.objValDual.hi, a.objValDual.lo) == (
            b.objValPrimal.hi, b.objValPrimal.lo, b.objValDual.hi, b.objValDual.lo), q
        for u, v in zip(p1[q], p0[q]):
            assert _same(u, v), q
