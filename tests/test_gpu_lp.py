"""SDPs with an LP block (negative block sizes) against the reference build
(tests/golden/lp_block.json, made by tests/golden/make_lp_golden.py with
oracle/_ref/sdpa_dd).

This build carries each LP entry as a positive semidefinite block of order 1
(the same problem: a 1 x 1 block is a non-negative scalar, its HKM direction
and step length are the LP ones, and the loop tests only max-abs norms and
sums over all entries), so its rounding differs from the reference's LP code
and the trajectories are not bit-identical.  Required: the reference's phase,
its iteration count within one, objectives within the requested accuracy
(1e-20, relative), and the result file's LP lists (xMat and yMat, after the
SDP block, 12 printed digits) equal to the reference's up to 1e-9 of the
largest entry.  A point written with sddd_write_point reads back with its LP
part (dense and sparse layout)."""
import ctypes
import importlib
import json
import re
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import ROOT, load_pkg

pytestmark = pytest.mark.gpu
getcontext().prec = 60
G = json.loads((ROOT / "tests" / "golden" / "lp_block.json").read_text())
REF = G["runs"][0]


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    load_pkg()
    P = importlib.import_module("sdpa_dd_b200.problems")
    td = tmp_path_factory.mktemp("lp")
    data = td / "lp.dat-s"
    data.write_text(P.with_lp(n=G["n"], q=G["q"], m=G["m"], seed=G["seed"]))
    param = P.write_param(str(td / "param.sdpa"), eps=G["eps"])
    return data, param, td


def _rel(a, b):
    a, b = Decimal(a), Decimal(b)
    return abs(a - b) / max(abs(b), Decimal(1))


def _check(phase, iters, objP, objD):
    assert phase == REF["phase"] and abs(iters - REF["iterations"]) <= 1, (phase, iters)
    eP, eD = _rel(objP, REF["objValPrimal32"]), _rel(objD, REF["objValDual32"])
    print(f"LP block: {phase} in {iters} iterations (reference {REF['iterations']}); objectives off by {float(eP):.1e}, {float(eD):.1e}")
    assert eP <= Decimal(G["eps"]) and eD <= Decimal(G["eps"])


def test_lp_block_through_c_abi(files):
    sddd = load_pkg()
    data, param, _ = files
    with sddd.Context(0) as c:
        c.read_problem(data)
        r = c.solve(sddd.param(param))
        _check(sddd.PHASES[r.phase], r.iterations, Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo),
               Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo))


def _lp_list(text, name):
    part = text.split(f"{name} = \n", 1)[1]
    lines = [ln.strip() for ln in part.splitlines()]
    # the SDP block ends with "   }", then the LP block's one list
    lists = [ln for ln in lines if re.fullmatch(r"\{[^{}]*\}", ln) and ln.count(",") == G["q"] - 1]
    return np.array([float(v) for v in lists[0].strip("{} ").split(",")])


def test_lp_block_through_the_command_line(files):
    sddd = load_pkg()
    data, param, td = files
    out = td / "cli.result"
    r = subprocess.run([str(sddd.BIN_PATH), "-ds", str(data), "-o", str(out), "-p", param], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = out.read_text()
    phase = re.search(r"phase.value = (\w+)", res).group(1)
    iters = int(re.search(r"Iteration = (\d+)", res).group(1))
    _check(phase, iters, re.search(r"objValPrimal = (\S+)", r.stdout).group(1), re.search(r"objValDual   = (\S+)", r.stdout).group(1))
    for name in ("xMat", "yMat"):
        got, want = _lp_list(res, name), np.array(REF[name])
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) <= 1e-9 * max(1.0, np.max(np.abs(want))), name


@pytest.mark.parametrize("sparse", [0, 1])
def test_lp_point_file_round_trip(files, sparse):
    sddd = load_pkg()
    data, param, td = files
    par = sddd.param(param)
    dump = td / f"lp_point_{sparse}.txt"
    with sddd.Context(0) as c:
        c.read_problem(data)
        c.solve(par)
        assert c.L.sddd_write_point(c.h, str(dump).encode(), sparse) == 0, c.L.sddd_last_error(c.h)
        ref = {w: c.get(w) for w in ("X", "Z", "y")}
    with sddd.Context(0) as c:
        c.read_problem(data)
        assert c.L.sddd_read_initial_point(c.h, str(dump).encode(), sparse, par.lambdaStar) == 0
        assert c.L.sddd_solver_start(c.h, ctypes.byref(par)) == 0
        for w in ("X", "Z", "y"):
            got = c.get(w)
            g = got["hi"].astype(np.longdouble) + got["lo"]
            want = ref[w]["hi"].astype(np.longdouble) + ref[w]["lo"]
            assert float(np.max(np.abs(g - want))) <= 2.0 ** -100 * max(float(np.max(np.abs(want))), 1e-300), w
