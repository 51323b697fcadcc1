"""The tensor-core split (INT8 slices on tcgen05) of the Cholesky trailing
update, through the C ABI.

* sddd_Rsyrk_tc against the exact value of C - P P^T (Python integers):
  |error(i,j)| <= k 2^-(7 S - 6) max|P(i,:)| max|P(j,:)| + 2^-104 |C(i,j)|
  for S slices (the split keeps 7S+1 bits of each row's scale), and the
  strict upper triangle untouched;
* sddd_Rpotrf with the split against the plain dd factor: within 1e-28
  relative to max|L| on well-conditioned SPD matrices, the same failing
  column on an indefinite one;
* whole solves with the split against the reference's golden results, under
  the bar of the plain solve (tests/test_gpu_solve.py) on the workloads with
  m > 64, where the split runs.
"""
import ctypes
import json

import numpy as np
import pytest

from conftest import DD, ROOT, load_pkg, ptr

pytestmark = pytest.mark.gpu

SCALE = 220  # values are integers times 2^-SCALE (all test data lies well above 2^-110)


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).cuda()


def from_dev(t, n):
    return t.cpu().numpy().view(DD)[:n].copy()


def exact_int(a):
    """dd array -> object array of exact integers (value * 2^SCALE)."""
    out = np.empty(a.shape, dtype=object)
    flat_hi, flat_lo, o = a["hi"].ravel(), a["lo"].ravel(), out.ravel()
    for q in range(flat_hi.size):
        tot = 0
        for v in (float(flat_hi[q]), float(flat_lo[q])):
            num, den = v.as_integer_ratio()
            sh = SCALE - (den.bit_length() - 1)
            assert sh >= 0, v
            tot += num << sh
        o[q] = tot
    return out


def rand_dd(rng, shape, lo_scale=1e-17, mag=None):
    out = np.zeros(shape, DD)
    hi = rng.standard_normal(shape) if mag is None else mag
    out["hi"] = hi
    out["lo"] = hi * rng.uniform(-1, 1, shape) * lo_scale
    return out


@pytest.fixture(scope="module")
def ctx():
    sddd = load_pkg()
    c = sddd.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n,k,ldc,slices", [(1, 64, 1, 16), (31, 64, 31, 16), (150, 64, 150, 16), (150, 37, 160, 16), (300, 64, 300, 12),
                                            (257, 64, 257, 8)])
def test_syrk_tc_matches_exact(ctx, n, k, ldc, slices):
    rng = np.random.default_rng(1000 + n + k + slices)
    # rows of different scales, with a zero row and tiny entries
    P = np.zeros((n, k), DD)
    P["hi"] = rng.standard_normal((n, k)) * np.exp2(rng.integers(-6, 7, (n, 1)))
    P["lo"] = P["hi"] * rng.uniform(-1, 1, (n, k)) * 1e-17
    if n > 3:
        P[2, :] = (0.0, 0.0)
        P[3, : k // 2]["hi"] *= 2.0 ** -20
        P[3, : k // 2]["lo"] *= 2.0 ** -20
    Pc = np.ascontiguousarray(P.T).ravel()  # column-major n x k, ld n
    C = rand_dd(rng, (ldc, n))  # column j = C[j, :]  (column-major, ld = ldc)
    C0 = C.copy()
    dP, dC = to_dev(Pc), to_dev(C.ravel())
    rc = ctx.L.sddd_Rsyrk_tc(ctx.h, n, k, ctypes.c_void_p(dP.data_ptr()), n, ctypes.c_void_p(dC.data_ptr()), ldc, slices)
    assert rc == 0, ctx.L.sddd_last_error(ctx.h)
    got = from_dev(dC, ldc * n).reshape(n, ldc)  # [j, i]
    Pi = exact_int(P)
    prod = Pi.dot(Pi.T)  # scale 2^(2 SCALE)
    rowmax = np.abs(P["hi"]).max(axis=1)
    absprod = np.abs(P["hi"]).dot(np.abs(P["hi"]).T)
    Ci = exact_int(C0.reshape(n, ldc)[:, :n].T)  # [i, j]
    Gi = exact_int(got[:, :n].T)
    for i in range(n):
        for j in range(n):
            if i < j:
                assert got[j, i]["hi"] == C0.reshape(n, ldc)[j, i]["hi"] and got[j, i]["lo"] == C0.reshape(n, ldc)[j, i]["lo"], (i, j)
                continue
            want = (Ci[i, j] << SCALE) - prod[i, j]  # scale 2^(2 SCALE)
            err = abs((Gi[i, j] << SCALE) - want)
            # digits beyond diagonal S + 1 dropped; the int64 carry of the
            # small diagonals rounded once (2^-105 of 2^(e_i + e_j) <=
            # 16 M_i M_j); the dd sum of the groups and its subtraction from C
            bound = (k * 2.0 ** -(7 * slices - 6) + 2.0 ** -101) * rowmax[i] * rowmax[j] + 2.0 ** -103 * (abs(
                float(C0.reshape(n, ldc)[j, i]["hi"]) - float(prod[i, j]) / 2.0 ** (2 * SCALE)) + absprod[i, j])
            assert err / 2.0 ** (2 * SCALE) <= bound + 1e-300, (i, j, err / 2.0 ** (2 * SCALE), bound)
    # rows beyond n in the leading dimension untouched
    if ldc > n:
        assert np.array_equal(got[:, n:].view(np.float64), C0.reshape(n, ldc)[:, n:].view(np.float64))


@pytest.mark.parametrize("n,k,slices", [(1, 1, 16), (33, 700, 16), (150, 100, 16), (5, 32767, 16), (70, 333, 12)])
def test_dot_pairs_tc_matches_exact(ctx, n, k, slices):
    """sddd_Rdot_pairs_tc (the Schur complement's F1 pair products) against
    exact integer arithmetic: rows of W scaled over several binades, a zero
    row, tiny entries; the bound is the split's truncation (7S+1 bits of each
    row's scale, k terms) plus the dd rebuild."""
    rng = np.random.default_rng(2000 + n + k + slices)
    W = np.zeros((n, k), DD)
    W["hi"] = rng.standard_normal((n, k)) * np.exp2(rng.integers(-6, 7, (n, 1)))
    W["lo"] = W["hi"] * rng.uniform(-1, 1, (n, k)) * 1e-17
    V = np.zeros((n, k), DD)
    V["hi"] = rng.standard_normal((n, k))
    V["lo"] = V["hi"] * rng.uniform(-1, 1, (n, k)) * 1e-17
    if n > 3:
        W[2, :] = (0.0, 0.0)
        W[3, : k // 2]["hi"] *= 2.0 ** -20
        W[3, : k // 2]["lo"] *= 2.0 ** -20
    C = np.zeros((n, n), DD)  # [j, i]: column-major
    C["hi"] = 7.0  # entries above the diagonal stay untouched
    dW, dV, dC = to_dev(W.ravel()), to_dev(V.ravel()), to_dev(C.ravel())
    rc = ctx.L.sddd_Rdot_pairs_tc(ctx.h, n, k, ctypes.c_void_p(dW.data_ptr()), k, ctypes.c_void_p(dV.data_ptr()), k, ctypes.c_void_p(dC.data_ptr()),
                                  n, slices)
    assert rc == 0, ctx.L.sddd_last_error(ctx.h)
    got = from_dev(dC, n * n).reshape(n, n)  # [j, i]
    Wi, Vi = exact_int(W), exact_int(V)
    prod = Wi.dot(Vi.T)  # [i, j] at scale 2^(2 SCALE)
    wmax, vmax = np.abs(W["hi"]).max(axis=1), np.abs(V["hi"]).max(axis=1)
    Gi = exact_int(got.T)  # [i, j]
    worst = 0.0
    for i in range(n):
        for j in range(n):
            if j > i:
                assert got[j, i]["hi"] == 7.0 and got[j, i]["lo"] == 0.0, (i, j)
                continue
            err = abs((Gi[i, j] << SCALE) - prod[i, j]) / 2.0 ** (2 * SCALE)
            bound = k * 2.0 ** -(7 * slices - 6) * wmax[i] * vmax[j] + 2.0 ** -104 * abs(float(prod[i, j]) / 2.0 ** (2 * SCALE))
            assert err <= bound + 1e-300, (i, j, err, bound)
            if bound > 0:
                worst = max(worst, err / bound)
    print(f"n={n} k={k} S={slices}: worst error {worst:.2e} of its bound")


def test_schur_tc_error_against_qd(ref_lib):
    """The Schur matrix of an all-dense block (the F1 pair products on the
    tensor cores) against the qd_real oracle, beside the plain dd form."""
    sddd = load_pkg()
    rng = np.random.default_rng(8)
    n, m = 40, 90
    As = rng.standard_normal((m, n, n)) / np.sqrt(n)
    As = (As + As.transpose(0, 2, 1)) / 2
    iu, ju = np.triu_indices(n)
    kk = np.concatenate([np.full(len(iu), q + 1) for q in range(m)])
    val = np.zeros(len(kk), DD)
    val["hi"] = np.concatenate([As[q][iu, ju] for q in range(m)])
    b = np.zeros(m, DD)
    b["hi"] = rng.standard_normal(m)
    G = rng.standard_normal((n, n))
    X = np.zeros(n * n, DD)
    X["hi"] = (np.eye(n) + G @ G.T / n).T.ravel()
    H = rng.standard_normal((n, n))
    Z = np.zeros(n * n, DD)
    Z["hi"] = (np.eye(n) + H @ H.T / n).T.ravel()
    out = {}
    with sddd.Context(0) as c:
        c.upload(m, [n], b, kk, np.ones_like(kk), np.tile(iu + 1, m), np.tile(ju + 1, m), val)
        assert c.set_point(X, np.zeros(m, DD), Z) == 0
        for slices in (0, 16):
            assert c.L.sddd_set_tc_split(c.h, slices) == 0
            c.call("sddd_schur_build")
            out[slices] = c.get("B")
        Zi = c.get("invZ")
    Adense = np.zeros(m * n * n, DD)
    Adense["hi"] = np.concatenate([As[q].T.ravel() for q in range(m)])
    Bq = np.zeros(4 * m * m)
    ref_lib.qd_schur_dense(ctypes.c_long(n), ctypes.c_long(m), ptr(Adense), ptr(X), ptr(Zi), ptr(Bq))
    err = {}
    for slices, B in out.items():
        o = np.zeros(2)
        ref_lib.qd_maxdiff(ctypes.c_long(m * m), ptr(np.ascontiguousarray(B)), ptr(Bq), ctypes.c_int(0), ctypes.c_long(0), ptr(o))
        err[slices] = o[0] / o[1]
        print(f"Schur matrix (n={n}, m={m}) vs qd, {'plain dd' if slices == 0 else 'split, 16 slices'}: {err[slices]:.2e}")
    assert err[0] < 1e-30
    assert err[16] < 1e-28


def _spd(rng, n):
    G = rng.standard_normal((n, n)) / np.sqrt(n)
    A = G @ G.T + np.eye(n)
    out = np.zeros(n * n, DD)
    out["hi"] = A.T.ravel()
    return out


@pytest.mark.parametrize("n", [200, 1000, 2085])
def test_potrf_tc_matches_plain(ctx, n):
    rng = np.random.default_rng(77 + n)
    A = _spd(rng, n)
    dA1, dA2 = to_dev(A), to_dev(A)
    assert ctx.L.sddd_set_tc_split(ctx.h, 0) == 0
    assert ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA1.data_ptr()), n) == 0
    assert ctx.L.sddd_set_tc_split(ctx.h, 16) == 0
    try:
        info = ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA2.data_ptr()), n)
    finally:
        ctx.L.sddd_set_tc_split(ctx.h, 0)
    assert info == 0
    L1 = from_dev(dA1, n * n).reshape(n, n)  # [j, i]
    L2 = from_dev(dA2, n * n).reshape(n, n)
    low = np.tril(np.ones((n, n), bool)).T  # [j, i] with i >= j
    d = (L2["hi"] - L1["hi"]) + (L2["lo"] - L1["lo"])
    scale = np.abs(L1["hi"][low]).max()
    rel = np.abs(d[low]).max() / scale
    assert rel <= 1e-28, rel


def test_potrf_tc_reports_failing_column(ctx):
    rng = np.random.default_rng(5)
    n = 300
    A = _spd(rng, n)
    A["hi"][200 * n + 200] = -5.0
    dA1, dA2 = to_dev(A), to_dev(A)
    i1 = ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA1.data_ptr()), n)
    ctx.L.sddd_set_tc_split(ctx.h, 16)
    try:
        i2 = ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA2.data_ptr()), n)
    finally:
        ctx.L.sddd_set_tc_split(ctx.h, 0)
    assert i1 == i2 == 201


def test_tc_split_rejects_bad_slice_counts(ctx):
    for s in (-1, 1, 7, 17):
        assert ctx.L.sddd_set_tc_split(ctx.h, s) == -1
    assert ctx.L.sddd_get_tc_split(ctx.h) == 0


GOLDEN = json.loads((ROOT / "tests" / "golden" / "solves.json").read_text())


@pytest.mark.parametrize("name", ["theta_nv24", "dense_n50_m100"])
def test_solve_tc_matches_reference(name, workdir):
    import importlib.util
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    spec = importlib.util.spec_from_file_location("mk", ROOT / "tests" / "golden" / "make_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    sddd = load_pkg()
    make, eps = mk.CASES[name]
    data = workdir / f"tc_{name}.dat-s"
    data.write_text(make())
    par = sddd.param(mk.P.write_param(str(workdir / f"tc_{name}.param"), eps=eps))
    g = GOLDEN[name]
    with sddd.Context(0) as c:
        c.read_problem(data, sparse=True, kappa=1.2)
        assert c.L.sddd_set_tc_split(c.h, 16) == 0
        c.call("sddd_solver_start", ctypes.byref(par))
        mus = []
        res = sddd.SdddResult()
        while c.L.sddd_iterate(c.h) == 0:
            c.call("sddd_solver_result", ctypes.byref(res))
            mus.append(Decimal(res.mu.hi) + Decimal(res.mu.lo))
        r = c.solve(par)
    spread = g["mu_spread"]
    chaos = next((q for q, s_ in enumerate(spread) if s_ > 1e-20), len(spread))
    for q in range(min(chaos, len(mus))):
        want = Decimal(g["mu_trajectory"][q][0]) + Decimal(g["mu_trajectory"][q][1])
        tol = max(Decimal("1e-25"), 10 * Decimal(spread[q]))
        assert abs(mus[q] - want) / abs(want) <= tol, (q, mus[q], want)
    phase = sddd.PHASES[r.phase]
    assert phase in {g["phase"]} | {v["phase"] for v in g["variants"]}, phase

    def rel(a, b):
        a, b = Decimal(a), Decimal(b)
        return abs(a - b) / max(abs(b), Decimal(1))

    spreadP = max([rel(v["objValPrimal32"], g["objValPrimal32"]) for v in g["variants"]], default=0)
    spreadD = max([rel(v["objValDual32"], g["objValDual32"]) for v in g["variants"]], default=0)
    objP = Decimal(r.objValPrimal.hi) + Decimal(r.objValPrimal.lo)
    objD = Decimal(r.objValDual.hi) + Decimal(r.objValDual.lo)
    assert rel(objP, g["objValPrimal32"]) <= max(Decimal("1e-24"), 10 * spreadP)
    assert rel(objD, g["objValDual32"]) <= max(Decimal("1e-24"), 10 * spreadD)
