"""Solves from an initial point file (the reference's -id / -is) against
the reference build (tests/golden/init_point.json, made by
tests/golden/make_init_golden.py with oracle/_ref/sdpa_dd).

The workload is max-cut-shaped (40 vertices), where the reference's runs
agree in phase and iteration count whatever the thread count; the starting
point is strictly feasible and dyadic (x_i = ceil(lambda_max(L)/4) + 1,
X = diag(x) - L/4, Y = I), written dense and sparse.  Required: the same
phase and iteration count as the reference, and objectives within
max(1e-24, 10 x the spread of the reference's own runs), through the C ABI
(file and arrays) and through the drop-in command line."""
import ctypes
import importlib
import json
import re
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import DD, ROOT, load_pkg

pytestmark = pytest.mark.gpu
getcontext().prec = 60
GOLDEN_DIR = ROOT / "tests" / "golden"
G = json.loads((GOLDEN_DIR / "init_point.json").read_text())


def _problems():
    load_pkg()
    return importlib.import_module("sdpa_dd_b200.problems")


def _rel(a, b):
    a, b = Decimal(a), Decimal(b)
    return abs(a - b) / max(abs(b), Decimal(1))


def _check(flag, phase, iters, objP, objD):
    runs = G["runs"][flag]
    ref = runs[0]
    assert phase == ref["phase"] and iters == ref["iterations"], (phase, iters, ref["phase"], ref["iterations"])
    sp = max([_rel(r["objValPrimal32"], ref["objValPrimal32"]) for r in runs] + [Decimal(0)])
    sd = max([_rel(r["objValDual32"], ref["objValDual32"]) for r in runs] + [Decimal(0)])
    assert _rel(objP, ref["objValPrimal32"]) <= max(Decimal("1e-24"), 10 * sp)
    assert _rel(objD, ref["objValDual32"]) <= max(Decimal("1e-24"), 10 * sd)


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    P = _problems()
    td = tmp_path_factory.mktemp("init")
    data = td / "maxcut.dat-s"
    data.write_text(P.maxcut(n=G["n"], p=G["p"], seed=G["seed"]))
    param = P.write_param(str(td / "param.sdpa"), eps=G["eps"])
    return data, param, td


@pytest.mark.parametrize("flag,name", [("-id", "init_dense.txt"), ("-is", "init_sparse.txt")])
def test_init_file_through_c_abi(files, flag, name):
    sddd = load_pkg()
    data, param, _ = files
    par = sddd.param(param)
    with sddd.Context(0) as c:
        c.read_problem(data)
        assert c.L.sddd_read_initial_point(c.h, str(GOLDEN_DIR / name).encode(), int(flag == "-is"), par.lambdaStar) == 0
        r = c.solve(par)
        objP = Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)
        objD = Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo)
        _check(flag, sddd.PHASES[r.phase], r.iterations, objP, objD)
        # cleared, the same context starts from lambda I again (46 passes)
        assert c.L.sddd_clear_initial_point(c.h) == 0
        assert c.solve(par).iterations != r.iterations


def test_init_arrays_equal_init_file(files):
    """sddd_set_initial_point with the same x, X, Y solves identically."""
    sddd = load_pkg()
    data, param, _ = files
    par = sddd.param(param)
    L = _laplacian()
    n = G["n"]
    x = np.full(n, float(np.ceil(np.linalg.eigvalsh(L).max() / 4.0)) + 1.0)
    X = np.diag(x) - L / 4.0
    xs, Xs, Ys = (np.zeros(a, DD) for a in (n, n * n, n * n))
    xs["hi"], Xs["hi"], Ys["hi"] = x, X.T.ravel(), np.eye(n).ravel()
    res = []
    with sddd.Context(0) as c:
        c.read_problem(data)
        assert c.L.sddd_set_initial_point(c.h, *(v.ctypes.data_as(ctypes.c_void_p) for v in (xs, Xs, Ys))) == 0
        res.append(c.solve(par))
        assert c.L.sddd_read_initial_point(c.h, str(GOLDEN_DIR / "init_sparse.txt").encode(), 1, par.lambdaStar) == 0
        res.append(c.solve(par))
    a, b = res
    assert (a.iterations, a.phase, a.objValPrimal.hi, a.objValPrimal.lo, a.objValDual.hi, a.objValDual.lo) == (
        b.iterations, b.phase, b.objValPrimal.hi, b.objValPrimal.lo, b.objValDual.hi, b.objValDual.lo)


def _laplacian():
    rng = np.random.default_rng(G["seed"])
    n = G["n"]
    A = np.triu(rng.random((n, n)) < G["p"], 1)
    A = A | A.T
    return np.diag(A.sum(axis=1).astype(float)) - A.astype(float)


@pytest.mark.parametrize("flag,name", [("-id", "init_dense.txt"), ("-is", "init_sparse.txt")])
def test_init_file_through_the_command_line(files, flag, name):
    sddd = load_pkg()
    data, param, td = files
    out = td / f"cli{flag}.result"
    r = subprocess.run([str(sddd.BIN_PATH), "-ds", str(data), flag, str(GOLDEN_DIR / name), "-o", str(out), "-p", param],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = out.read_text()
    assert f"initial   is {GOLDEN_DIR / name}" in res
    phase = re.search(r"phase.value = (\w+)", res).group(1)
    iters = int(re.search(r"Iteration = (\d+)", res).group(1))
    objP = re.search(r"objValPrimal = (\S+)", r.stdout).group(1)
    objD = re.search(r"objValDual   = (\S+)", r.stdout).group(1)
    _check(flag, phase, iters, objP, objD)
