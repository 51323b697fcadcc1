"""Oracle Schur complement, formula choice and Lanczos eigenvalue against
the reference's own Newton / step-length code on small seeded problems."""
import ctypes

import numpy as np
import pytest

import sdpa_problem
from conftest import DD, RefSolver, as_dd, load_pkg, ptr
from test_oracle import same, spd, rand_dd

SMALL = {
    "dense": lambda P: P.dense_random(n=12, m=20, seed=10),
    "maxcut": lambda P: P.maxcut(n=30, p=0.2, seed=11),
    "theta": lambda P: P.theta(nv=16, p=0.5, seed=12),
    "control": lambda P: P.control_like(sizes=(9, 6), m=25, seed=13),
}


@pytest.fixture(scope="module")
def problems(workdir):
    P = load_pkg().problems if hasattr(load_pkg(), "problems") else __import__("sdpa_dd_b200.problems").problems
    out = {}
    for name, make in SMALL.items():
        path = workdir / f"{name}.dat-s"
        path.write_text(make(P))
        out[name] = path
    return out


@pytest.mark.parametrize("name", list(SMALL))
@pytest.mark.parametrize("steps", [0, 3])
def test_schur_matches_reference(oracle_lib, ref_lib, problems, name, steps):
    ref = RefSolver(ref_lib, problems[name])
    try:
        for _ in range(steps):
            assert ref.step() == 0
        X = ref.blocks_of(ref.get(0))
        Zi = ref.blocks_of(ref.get(5))
        B_ref = ref.schur()
        prob = sdpa_problem.Problem(oracle_lib, problems[name].read_text())
        assert prob.m == ref.m and prob.block_struct == ref.blocks
        # formula table
        f_ref = ref.formula()
        for l in range(prob.nblocks):
            for t, k in enumerate(prob.cons[l]):
                assert prob.formula[l][t] == f_ref[k, l]
        B = sdpa_problem.schur(prob, X, Zi)
        assert same(B, B_ref)
    finally:
        ref.close()


@pytest.mark.parametrize("n", [21, 40, 90])
def test_lanczos_matches_reference(oracle_lib, ref_lib, n):
    rng = np.random.default_rng(n)
    A = spd(rng, n)
    ref_lib.ref_Rpotrf(b"Lower", ctypes.c_long(n), ptr(A), ctypes.c_long(n))
    L = np.zeros(n * n, DD)
    oracle_lib.o_inv_lower(ctypes.c_long(n), ptr(A), ctypes.c_long(n), ptr(L), ctypes.c_long(n))
    G = rng.standard_normal((n, n))
    S = (G + G.T) / 2
    X = as_dd(S.T.ravel())
    r = np.zeros(1, DD)
    ref_lib.ref_lanczos_min_eig(ctypes.c_long(n), ptr(L), ptr(X), ptr(r))

    class ODD(ctypes.Structure):
        _fields_ = [("hi", ctypes.c_double), ("lo", ctypes.c_double)]
    oracle_lib.o_lanczos_min_eig.restype = ODD
    v = oracle_lib.o_lanczos_min_eig(ctypes.c_long(n), ptr(L), ptr(X))
    a = float(r["hi"][0]) + float(r["lo"][0])
    b = v.hi + v.lo
    # compare in dd: difference of the two dd numbers relative to |a|
    diff = (v.hi - float(r["hi"][0])) + (v.lo - float(r["lo"][0]))
    assert abs(diff) <= 1e-26 * abs(a), (a, b, diff)
