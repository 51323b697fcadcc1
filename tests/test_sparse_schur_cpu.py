"""The Schur form decision and the sparse form's layout, on the host.

The reference chooses between a dense and a sparse B in
Chordal::ordering_bMat (sdpa_chordal.cpp:348-438) and lays the sparse B out
in Newton::initialize_sparse_bMat (sdpa_newton.cpp:225-340).  Its ordering
comes from SPOOLES, a library the reference's sources do not include; the
oracle build runs the reference with its own minimum-degree ordering in
SPOOLES's place (oracle/spooles_shim.cpp), written independently of the
product's (sparse_schur.cpp).  Required: for every problem and mode the
product takes the reference's decision, and when it is sparse the same
ordering, diagonalIndex and column_index."""
import ctypes

import numpy as np
import pytest

from conftest import ROOT, load_pkg, ptr

import importlib.util

spec = importlib.util.spec_from_file_location("problems", ROOT / "sdpa-dd_b200" / "problems.py")
P = importlib.util.module_from_spec(spec)
spec.loader.exec_module(P)

CASES = {
    "chain40": lambda: P.chain_blocks(nblocks=40, n=10, per=4, overlap=2, seed=9),
    "chain60_lp": lambda: P.chain_blocks(nblocks=60, n=6, per=3, overlap=3, q=40, seed=11),
    "chain12_wide": lambda: P.chain_blocks(nblocks=12, n=5, per=8, overlap=4, seed=13),
    # m <= 100: dense whatever the blocks
    "chain20_small": lambda: P.chain_blocks(nblocks=20, n=4, per=3, overlap=1, seed=14),
    # 5 blocks: dense
    "chain5": lambda: P.chain_blocks(nblocks=5, n=6, per=30, overlap=5, seed=15),
    # a block that touches more than half of the constraints: dense
    "blocks_lp": lambda: P.blocks_with_lp(sizes=(6, 5, 4, 3, 3, 2, 2), q=20, m=120, seed=16),
}


def _ref_layout(ref_lib, path, mode):
    ref_lib.ref_open_mode.restype = ctypes.c_void_p
    ref_lib.ref_open_mode.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int]
    ref_lib.ref_sparse_layout.restype = ctypes.c_long
    h = ctypes.c_void_p(ref_lib.ref_open_mode(str(path).encode(), None, 1.2, mode))
    assert h.value
    try:
        if not ref_lib.ref_schur_sparse(h):
            return None
        dims = np.zeros(4096, np.int32)
        ref_lib.ref_dims(h, ptr(dims), 4096)
        m = int(dims[0])
        nnz = ref_lib.ref_sparse_layout(h, None, None, None)
        o, d, c = np.zeros(m, np.int32), np.zeros(m + 1, np.int32), np.zeros(nnz, np.int32)
        ref_lib.ref_sparse_layout(h, ptr(o), ptr(d), ptr(c))
        return o, d, c
    finally:
        ref_lib.ref_close(h)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_schur_form_matches_reference(ref_lib, workdir, name, mode):
    sddd = load_pkg()
    path = workdir / f"form_{name}.dat-s"
    if not path.exists():
        path.write_text(CASES[name]())
    want = _ref_layout(ref_lib, path, mode)
    info, order, di, ci = sddd.plan_schur(path, mode)
    assert bool(info.sparse) == (want is not None), (info.sparse, info.reason)
    if want is None:
        assert info.reason, "a dense decision names its reason"
        return
    assert info.extended == 2 * len(ci) - info.m
    assert np.array_equal(order, want[0])
    assert np.array_equal(di, want[1])
    assert np.array_equal(ci, want[2])


def test_decisions_are_the_expected_ones(workdir):
    sddd = load_pkg()
    expect = {"chain40": 1, "chain60_lp": 1, "chain12_wide": 1, "chain20_small": 0, "chain5": 0, "blocks_lp": 0}
    for name, sp in expect.items():
        path = workdir / f"form_{name}.dat-s"
        if not path.exists():
            path.write_text(CASES[name]())
        info = sddd.plan_schur(path, 0)[0]
        assert info.sparse == sp, (name, info.reason)
        assert sddd.plan_schur(path, 1)[0].sparse == 0
        assert sddd.plan_schur(path, 2)[0].sparse == 1


def test_layout_is_a_symbolic_factor(workdir):
    """Rows start at their diagonal, ascend, and every pair of later entries
    of a row meets again in the row of the earlier one (closure)."""
    sddd = load_pkg()
    path = workdir / "form_chain40.dat-s"
    if not path.exists():
        path.write_text(CASES["chain40"]())
    info, order, di, ci = sddd.plan_schur(path, 0)
    m = info.m
    assert sorted(order.tolist()) == list(range(m))
    rows = [set(ci[di[b]:di[b + 1]].tolist()) for b in range(m)]
    for b in range(m):
        r = ci[di[b]:di[b + 1]]
        assert r[0] == b and np.all(np.diff(r) > 0)
        for x in r[1:]:
            for z in r[1:]:
                if z > x:
                    assert z in rows[x]
