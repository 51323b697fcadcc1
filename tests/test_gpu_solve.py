"""End-to-end GPU solves through the C ABI and the drop-in command line,
against the reference's own results (tests/golden/solves.json, made by
tests/golden/make_golden.py from the reference build).

The reference is not reproducible run to run once mu nears the dd noise
floor: its OpenMP reductions add partial sums in arrival order, and the
Lanczos step length makes discrete choices (checkpoints, stopping tests) on
the results, so with 2-8 threads its final phase and iteration count vary
from run to run (the fixture keeps 8 such runs per workload).  The bar:

* trajectory: after every pass k of the main loop, up to the first pass at
  which the reference's own runs differ by more than 1e-20 in mu, the GPU's
  mu equals the one-thread reference's within max(1e-25, 10 x that spread)
  relative;
* where every reference run agrees (same phase, same iteration count): the
  same phase and iteration count exactly;
* elsewhere: a final phase that some reference run reached;
* objectives: within max(1e-24, 10 x the spread of the reference runs'
  objectives) relative of the one-thread reference's.
"""
import json
import subprocess

import pytest

from conftest import ROOT, load_pkg

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((ROOT / "tests" / "golden" / "solves.json").read_text())


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", ROOT / "tests" / "golden" / "make_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.CASES, mk.P


CASES, P = _cases()


def _dd_from_text(s):
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    return Decimal(s)


def _rel(a, b):
    from decimal import Decimal
    a, b = Decimal(a), Decimal(b)
    return abs(a - b) / max(abs(b), Decimal(1))


def _relative(a, b):
    return abs(a - b) / abs(b) if b != 0 else abs(a)


def _dec(x):
    from decimal import Decimal
    return Decimal(x[0]) + Decimal(x[1]) if isinstance(x, (list, tuple)) else Decimal(x)


def _spread(g, key):
    return max([_rel(v[key], g[key]) for v in g["variants"]], default=0)


def _deterministic(g):
    return all(v["phase"] == g["phase"] and v["iterations"] == g["iterations"] for v in g["variants"])


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_solve_matches_reference(name, workdir):
    import ctypes
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    sddd = load_pkg()
    make, eps = CASES[name]
    data = workdir / f"solve_{name}.dat-s"
    data.write_text(make())
    param_path = P.write_param(str(workdir / f"solve_{name}.param"), eps=eps)
    g = GOLDEN[name]
    par = sddd.param(param_path)
    with sddd.Context(0) as ctx:
        ctx.read_problem(data, sparse=True, kappa=1.2)
        # the main loop pass by pass: mu after each pass
        ctx.call("sddd_solver_start", ctypes.byref(par))
        mus = []
        res = sddd.SdddResult()
        while ctx.L.sddd_iterate(ctx.h) == 0:
            ctx.call("sddd_solver_result", ctypes.byref(res))
            mus.append((res.mu.hi, res.mu.lo))
        # the whole solve (pinpal with its final phase handling)
        r = ctx.solve(par)
    assert r.iterations == len(mus) or r.iterations == len(mus) + 1, (r.iterations, len(mus))

    mu1, spread = g["mu_trajectory"], g["mu_spread"]
    chaos = next((k for k, s_ in enumerate(spread) if s_ > 1e-20), len(spread))
    assert chaos >= 3, chaos
    for k in range(min(chaos, len(mus))):
        tol = max(Decimal("1e-25"), 10 * Decimal(spread[k]))
        assert _relative(_dec(mus[k]), _dec(mu1[k])) <= tol, (k, mus[k], mu1[k], spread[k])

    phase = sddd.PHASES[r.phase]
    if _deterministic(g):
        assert phase == g["phase"], (phase, g["phase"])
        assert r.iterations == g["iterations"], (r.iterations, g["iterations"])
    else:
        assert phase in {g["phase"]} | {v["phase"] for v in g["variants"]}, phase
    objP = Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)
    objD = Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo)
    assert _rel(objP, g["objValPrimal32"]) <= max(Decimal("1e-24"), 10 * _spread(g, "objValPrimal32")), (objP, g["objValPrimal32"])
    assert _rel(objD, g["objValDual32"]) <= max(Decimal("1e-24"), 10 * _spread(g, "objValDual32")), (objD, g["objValDual32"])


def test_cli_drop_in(workdir):
    sddd = load_pkg()
    name = "maxcut_n30"
    make, eps = CASES[name]
    data = workdir / "cli.dat-s"
    data.write_text(make())
    param_path = P.write_param(str(workdir / "cli.param"), eps=eps)
    out = workdir / "cli.result"
    r = subprocess.run([str(sddd.BIN_PATH), "-ds", str(data), "-o", str(out), "-p", param_path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    g = GOLDEN[name]
    assert f"phase.value = {g['phase']}" in text
    assert f"Iteration = {g['iterations']}" in text
    assert "objValPrimal = " + g["objValPrimal16"] in text
    assert "objValDual   = " + g["objValDual16"] in text
    assert "xVec = " in text and "yMat = " in text
    assert "objValPrimal = " + g["objValPrimal32"][:20] in r.stdout
