"""Problems with many blocks against the reference build
(tests/golden/many_blocks.json, made by tests/golden/make_blocks_golden.py
with oracle/_ref/sdpa_dd): an SDP block with an LP block of 200 entries, 80
small dense SDP blocks, and 70 small SDP blocks with an LP block of 100
entries.  Every LP entry is carried as an SDP block of order 1, so these
problems have 81 to 201 blocks, each with its own per-block results (the
inner products of the objectives and the step-length eigenvalues).

Required, as for the LP fixture (tests/test_gpu_lp.py; the LP entries and
the small blocks' eigenvalues round differently from the reference's own LP
and Rsyev code): the reference's phase, its iteration count within one, and
objectives within the requested accuracy (1e-20, relative) of the
one-thread reference's.  The 80-block problem is also replayed piece by
piece, bit for bit, in tests/test_gpu_pieces.py."""
import importlib.util
import json
from decimal import Decimal, getcontext

import pytest

from conftest import ROOT, load_pkg

pytestmark = pytest.mark.gpu
getcontext().prec = 60
G = json.loads((ROOT / "tests" / "golden" / "many_blocks.json").read_text())


def _cases():
    spec = importlib.util.spec_from_file_location("mkb", ROOT / "tests" / "golden" / "make_blocks_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.CASES, mk.P


CASES, P = _cases()


def _rel(a, b):
    a, b = Decimal(a), Decimal(b)
    return abs(a - b) / max(abs(b), Decimal(1))


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_many_blocks_match_reference(name, workdir):
    sddd = load_pkg()
    data = workdir / f"blocks_{name}.dat-s"
    data.write_text(CASES[name]())
    param = P.write_param(str(workdir / f"blocks_{name}.param"), eps=G["eps"])
    ref = G["cases"][name][0]
    assert all(r["phase"] == ref["phase"] and r["iterations"] == ref["iterations"] for r in G["cases"][name])
    with sddd.Context(0) as c:
        c.read_problem(data)
        assert c.nsdp > 64, c.nsdp
        r = c.solve(sddd.param(param))
    phase = sddd.PHASES[r.phase]
    objP = Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)
    objD = Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo)
    eP, eD = _rel(objP, ref["objValPrimal32"]), _rel(objD, ref["objValDual32"])
    print(f"{name}: {c.nsdp} blocks, {phase} in {r.iterations} iterations (reference {ref['iterations']}); "
          f"objectives off by {float(eP):.1e}, {float(eD):.1e}")
    assert phase == ref["phase"]
    assert abs(r.iterations - ref["iterations"]) <= 1
    assert eP <= Decimal(G["eps"]) and eD <= Decimal(G["eps"])
