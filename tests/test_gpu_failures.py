"""Failure paths, made on the host or by a flag that nothing sets; no GPU
fault, trap or endless wait is involved.

* Bounded waits: with sddd_test_withhold_block the triangular solves never
  publish one 64-entry block's completion flag, so every wait for it runs
  out of a short budget (sddd_set_wait_limit, 5 ms).  The call returns
  SDDD_ERR_CUDA naming the block, and the same context then solves
  normally, bit for bit as a fresh one (the reference-order wavefront solve
  of the plain form and the blocked solve of the split form).
* A NaN in the problem data: the Cholesky of the Schur matrix reports its
  first column as not positive definite (the reference's Rpotrf tests its
  pivots with isnan too) and the solve stops at once with stop reason 2;
  the context takes the next problem.
* A point that is not positive definite: sddd_set_point reports the failed
  Cholesky of X (status 1) instead of computing with it.
* A step too short to move: the solve stops with stop reason 4 ("cannot
  move") at the pass where the reference build stops with the same message.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import DD, ROOT, load_pkg
from test_oracle import same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def theta40(workdir):
    import importlib
    load_pkg()
    P = importlib.import_module("sdpa_dd_b200.problems")
    path = workdir / "fail_theta40.dat-s"
    path.write_text(P.theta(nv=40, p=0.5, seed=5))
    return path


def _factored(sddd, path, slices):
    c = sddd.Context(0)
    c.read_problem(path, sparse=True, kappa=1.2)
    assert c.L.sddd_set_tc_split(c.h, slices) == 0
    c.call("sddd_init_point", sddd.SdddDD(1.0e4, 0.0))
    c.call("sddd_newton_rhs", 0, sddd.SdddDD(1.0e3, 0.0), 1)
    c.call("sddd_schur_build")
    assert c.call("sddd_schur_factor") == 0
    return c


@pytest.mark.parametrize("slices", [0, 16])
def test_withheld_block_runs_out_of_its_wait_and_the_context_recovers(theta40, slices):
    sddd = load_pkg()
    ref = _factored(sddd, theta40, slices)
    try:
        assert ref.m > 5 * 64, ref.m
        ref.call("sddd_solve_dy")
        want = ref.get("Dy")
    finally:
        ref.close()
    c = _factored(sddd, theta40, slices)
    try:
        assert c.L.sddd_set_wait_limit(c.h, 0.005) == 0
        assert c.L.sddd_test_withhold_block(c.h, 2) == 0
        rc = c.L.sddd_solve_dy(c.h)
        msg = c.L.sddd_last_error(c.h).decode()
        assert rc == -2, (rc, msg)
        assert "block 2" in msg, msg
        # the context is usable: the same solve with every flag published
        assert c.L.sddd_test_withhold_block(c.h, -1) == 0
        assert c.L.sddd_set_wait_limit(c.h, 2.0) == 0
        assert c.L.sddd_solve_dy(c.h) == 0, c.L.sddd_last_error(c.h)
        assert same(c.get("Dy"), want)
    finally:
        c.close()


def test_wait_limit_range_is_checked(theta40):
    sddd = load_pkg()
    with sddd.Context(0) as c:
        for bad in (0.0, -1.0, 1e-6, 61.0, float("nan")):
            assert c.L.sddd_set_wait_limit(c.h, bad) == -1, bad
        assert c.L.sddd_test_withhold_block(c.h, -2) == -1


def test_nan_in_the_data_stops_with_a_cholesky_failure(workdir):
    sddd = load_pkg()
    import importlib
    P = importlib.import_module("sdpa_dd_b200.problems")
    rng = np.random.default_rng(3)
    n, m = 6, 8
    iu, ju = np.triu_indices(n)
    k = np.concatenate([np.full(len(iu), q) for q in range(m + 1)])
    val = np.zeros(len(k), DD)
    val["hi"] = rng.standard_normal(len(k))
    val["hi"][len(iu) + 3] = np.nan  # one entry of F_1
    b = np.zeros(m, DD)
    b["hi"] = rng.standard_normal(m)
    par = sddd.param(P.write_param(str(workdir / "nan.param"), eps=1e-20))
    with sddd.Context(0) as c:
        c.upload(m, [n], b, k, np.ones_like(k), np.tile(iu + 1, m + 1), np.tile(ju + 1, m + 1), val)
        r = c.solve(par)
        assert r.stop_reason == 2, r.stop_reason
        assert r.iterations == 0
        # the next problem in the same context solves
        path = workdir / "after_nan.dat-s"
        path.write_text(P.dense_random(n=8, m=5, seed=16))
        c.read_problem(path)
        r = c.solve(par)
        assert r.stop_reason == 1 and sddd.PHASES[r.phase] == "pdOPT", (r.stop_reason, r.phase)


def test_indefinite_point_is_refused(theta40):
    sddd = load_pkg()
    with sddd.Context(0) as c:
        c.read_problem(theta40)
        n = c.sizes[0]
        X = np.zeros(n * n, DD)
        X["hi"][:: n + 1] = 1.0
        X["hi"][5 * (n + 1)] = -1.0  # one negative eigenvalue
        Z = np.zeros(n * n, DD)
        Z["hi"][:: n + 1] = 1.0
        rc = c.L.sddd_set_point(c.h, X.ctypes.data_as(ctypes.c_void_p), np.zeros(c.m, DD).ctypes.data_as(ctypes.c_void_p),
                                Z.ctypes.data_as(ctypes.c_void_p))
        assert rc == 1, rc


def test_cannot_move_stops_where_the_reference_stops(workdir):
    """dense_n12_m20 at epsilon 1e-25: the reference build prints "cannot
    move" (Solutions::update, sdpa_dataset.cpp:136; sdpa_main.cpp:355) and
    stops in pFEAS, after 42 to 58 passes depending on its OpenMP thread
    count (tests/golden/solves.json); the GPU solve stops the same way, with
    stop reason 4, within that range."""
    import json
    sddd = load_pkg()
    import importlib
    P = importlib.import_module("sdpa_dd_b200.problems")
    g = json.loads((ROOT / "tests" / "golden" / "solves.json").read_text())["dense_n12_m20"]
    counts = [g["iterations"]] + [v["iterations"] for v in g["variants"]]
    data = workdir / "cannot_move.dat-s"
    data.write_text(P.dense_random(n=12, m=20, seed=10))
    param = P.write_param(str(workdir / "cannot_move.param"), eps=1e-25)
    ref_bin = ROOT / "oracle" / "_ref" / "sdpa_dd"
    if ref_bin.exists():
        out = subprocess.run([str(ref_bin), "-ds", str(data), "-o", str(workdir / "cannot_move.result"), "-p", param], capture_output=True,
                             text=True, env=dict(os.environ, OMP_NUM_THREADS="1"), timeout=300).stdout
        assert "cannot move" in out
        assert int(re.search(r"Iteration = (\d+)", out).group(1)) == g["iterations"]
    with sddd.Context(0) as c:
        c.read_problem(data)
        r = c.solve(sddd.param(param))
    assert r.stop_reason == 4, r.stop_reason
    assert sddd.PHASES[r.phase] == "pFEAS"
    assert min(counts) <= r.iterations <= max(counts), (r.iterations, counts)
