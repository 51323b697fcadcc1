"""The sparse Schur path against the reference build.

The reference factors and solves a sparse B with Lal::getCholesky(
SparseMatrix&, int*) (sdpa_linear.cpp:353-395) and Lal::solveSystems(Vector&,
SparseMatrix&, Vector&) (:654-810) after renumbering the constraints by a
minimum-degree ordering (sdpa_chordal.cpp:348-438; the oracle's ordering in
oracle/spooles_shim.cpp stands in for SPOOLES, and the CPU tests in
tests/test_sparse_schur_cpu.py check it equals the product's).  Required:

* the device factor and solve equal the reference's functions bit for bit on
  the same structure and entries (random positive definite entries, and a
  negative pivot, which the reference turns into a zero row);
* on problems that take the sparse path, one Newton pass replayed piece by
  piece equals the reference's bit for bit: B, the factor in the reference's
  layout, Dy, Dz and Dx of predictor and corrector;
* whole solves (tests/golden/sparse_schur.json) reach the reference's phase,
  its iteration count within one and its objectives within the requested
  accuracy (1e-20 relative), and the dense form of the same problem agrees.
"""
import ctypes
import importlib.util
import json
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import DD, ROOT, RefSolver, load_pkg, ptr
from test_oracle import same

pytestmark = pytest.mark.gpu
getcontext().prec = 60
G = json.loads((ROOT / "tests" / "golden" / "sparse_schur.json").read_text())


def _mk():
    spec = importlib.util.spec_from_file_location("mks", ROOT / "tests" / "golden" / "make_sparse_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.CASES, mk.P


CASES, P = _mk()


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).cuda()


def from_dev(t, n):
    out = np.zeros(n, DD)
    out.view(np.float64)[:] = t.cpu().numpy()
    return out


@pytest.fixture(scope="module")
def sddd():
    return load_pkg()


@pytest.fixture(scope="module")
def files(workdir):
    out = {}
    for name, make in CASES.items():
        p = workdir / f"sparse_{name}.dat-s"
        p.write_text(make())
        out[name] = p
    return out


def _values(rng, di, ci, negative=None):
    m = len(di) - 1
    v = np.zeros(di[m], DD)
    v["hi"] = rng.standard_normal(di[m]) * 0.1
    v["lo"] = v["hi"] * 1e-17 * rng.standard_normal(di[m])
    d = di[:-1]
    v["hi"][d] = 4.0 + 10.0 * np.abs(rng.standard_normal(m))
    v["lo"][d] = 0.0
    if negative is not None:
        v["hi"][di[negative]] = -1.0
    return v


@pytest.mark.parametrize("name", ["chain40", "chain150"])
@pytest.mark.parametrize("negative", [None, "mid"])
def test_sparse_factor_and_solve_match_reference(sddd, ref_lib, files, name, negative):
    info, order, di, ci = sddd.plan_schur(files[name])
    assert info.sparse == 1 and info.nnz == len(ci)
    m = info.m
    rng = np.random.default_rng(17)
    vals = _values(rng, di, ci, m // 2 if negative else None)
    want = vals.copy()
    ref_lib.ref_sparse_getCholesky(ctypes.c_int(m), ptr(di), ptr(ci), ptr(want))
    with sddd.Context(0) as c:
        dv = to_dev(vals)
        rc = c.L.sddd_sparse_getCholesky(c.h, m, ptr(di), ptr(ci), ctypes.c_void_p(dv.data_ptr()))
        assert rc == 0, c.L.sddd_last_error(c.h)
        got = from_dev(dv, len(vals))
        r_ = same(got, want)
        assert r_, ("factor", r_)
        for trial in range(2):
            x = np.zeros(m, DD)
            x["hi"] = rng.standard_normal(m)
            xr = x.copy()
            ref_lib.ref_sparse_solveSystems(ctypes.c_int(m), ptr(di), ptr(ci), ptr(want), ptr(xr))
            dx = to_dev(x)
            rc = c.L.sddd_sparse_solveSystems(c.h, m, ptr(di), ptr(ci), ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dx.data_ptr()))
            assert rc == 0, c.L.sddd_last_error(c.h)
            r_ = same(from_dev(dx, m), xr)
            assert r_, ("solve", r_)


def test_sparse_structure_is_checked(sddd):
    with sddd.Context(0) as c:
        # row 0 reaches rows 1 and 2, so (2, 1) must be in row 1
        di = np.array([0, 3, 4, 5], np.int32)
        ci = np.array([0, 1, 2, 1, 2], np.int32)
        v = to_dev(np.ones(5, DD))
        assert c.L.sddd_sparse_getCholesky(c.h, 3, ptr(di), ptr(ci), ctypes.c_void_p(v.data_ptr())) == -1
        assert b"missing" in c.L.sddd_last_error(c.h)
        ci = np.array([0, 2, 1, 1, 2], np.int32)  # not ascending
        assert c.L.sddd_sparse_getCholesky(c.h, 3, ptr(di), ptr(ci), ctypes.c_void_p(v.data_ptr())) == -1


def _ddmul(ref_lib, a, b):
    aa, bb, out = np.array([a], DD), np.array([b], DD), np.zeros(1, DD)
    ref_lib.ref_dd_op(4, ctypes.c_long(1), ptr(aa), ptr(bb), ptr(out))
    return float(out["hi"][0]), float(out["lo"][0])


@pytest.mark.parametrize("name", ["chain40", "chain150"])
@pytest.mark.parametrize("k", [1, 4])
def test_sparse_newton_pieces_match_reference(sddd, ref_lib, files, name, k):
    """The GPU at the reference's point before its pass k+1, that pass
    replayed piece by piece on the sparse Schur path."""
    path = files[name]
    ref_lib.ref_sparse_layout.restype = ctypes.c_long
    ref_lib.ref_sparse_values.restype = ctypes.c_long
    ref = RefSolver(ref_lib, path)
    try:
        assert ref_lib.ref_schur_sparse(ref.h) == 1
        nnz = ref_lib.ref_sparse_layout(ref.h, None, None, None)
        r_order = np.zeros(ref.m, np.int32)
        r_di = np.zeros(ref.m + 1, np.int32)
        r_ci = np.zeros(nnz, np.int32)
        ref_lib.ref_sparse_layout(ref.h, ptr(r_order), ptr(r_di), ptr(r_ci))
        with sddd.Context(0) as c:
            c.read_problem(path, sparse=True, kappa=1.2)
            info, order, di, ci = c.schur_form()
            assert info.sparse == 1
            assert np.array_equal(order, r_order) and np.array_equal(di, r_di) and np.array_equal(ci, r_ci)
            for _ in range(k):
                assert ref.step() == 0
            X, y, Z = ref.get(0), ref.get(2), ref.get(1)
            assert c.set_point(X, y, Z) == 0
            c.dd_scalar("sddd_residuals", ctypes.byref(sddd.SdddDD()))
            assert ref.step() == 0
            phase = ref_lib.ref_phase_at_step(ref.h)
            dinf = int(phase in (0, 1))
            mu = ref.scalar(19)
            # predictor
            c.call("sddd_newton_rhs", 0, sddd.SdddDD(*_ddmul(ref_lib, ref.scalar(16), mu)), dinf)
            r_ = same(c.get("g"), ref.get(8))
            assert r_, ("g", r_)
            c.call("sddd_schur_build")
            r_ = same(c.get("B"), ref.get(6))
            assert r_, ("B", r_)
            assert c.call("sddd_schur_factor") == 0
            want = np.zeros(nnz, DD)
            ref_lib.ref_sparse_values(ref.h, ptr(want))
            r_ = same(c.sparse_factor_values(nnz), want)
            assert r_, ("sparse factor", r_)
            c.call("sddd_solve_dy")
            r_ = same(c.get("Dy"), ref.get(13))
            assert r_, ("Dy (predictor)", r_)
            c.call("sddd_make_dz_dx", dinf)
            r_ = same(c.get("Dz"), ref.get(14))
            assert r_, ("Dz (predictor)", r_)
            r_ = same(c.get("Dx"), ref.get(12))
            assert r_, ("Dx (predictor)", r_)
            # corrector (the same factor)
            c.call("sddd_newton_rhs", 1, sddd.SdddDD(*_ddmul(ref_lib, ref.scalar(6), mu)), dinf)
            c.call("sddd_solve_dy")
            r_ = same(c.get("Dy"), ref.get(10))
            assert r_, ("Dy (corrector)", r_)
    finally:
        ref.close()


def _rel(a, b):
    a, b = Decimal(a), Decimal(b)
    return abs(a - b) / max(abs(b), Decimal(1))


@pytest.mark.parametrize("name", sorted(G["cases"]))
def test_sparse_solves_match_reference(sddd, files, workdir, name):
    param = P.write_param(str(workdir / f"sparse_{name}.param"), eps=G["eps"])
    ref = G["cases"][name][0]
    assert all(r["sparse"] and r["phase"] == ref["phase"] for r in G["cases"][name])
    objs = {}
    for mode in (0, 1):
        with sddd.Context(0) as c:
            c.read_problem(files[name])
            c.set_schur_mode(mode)
            info = c.schur_form()[0]
            assert info.sparse == (1 if mode == 0 else 0)
            r = c.solve(sddd.param(param))
        phase = sddd.PHASES[r.phase]
        objP = Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)
        objD = Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo)
        eP, eD = _rel(objP, ref["objValPrimal32"]), _rel(objD, ref["objValDual32"])
        print(f"{name} ({'sparse' if mode == 0 else 'dense'}): {phase} in {r.iterations} iterations "
              f"(reference {ref['iterations']}); objectives off by {float(eP):.1e}, {float(eD):.1e}")
        assert phase == ref["phase"]
        assert abs(r.iterations - ref["iterations"]) <= 1
        assert eP <= Decimal(G["eps"]) and eD <= Decimal(G["eps"])
        objs[mode] = objP
    assert _rel(objs[0], objs[1]) <= Decimal(G["eps"])
