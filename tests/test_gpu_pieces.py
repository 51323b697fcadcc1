"""GPU parity of the hot-path pieces, through the C ABI (libsddd.so).

Every piece is given the same inputs as the reference and must return the
reference's dd results bit for bit (+0 and -0 compared equal):
  - the 18 dd operation shapes against QD;
  - dd GEMM / Cholesky / triangular solves against the oracle;
  - at real iterates of small seeded problems (dense F1, max-cut F3,
    theta F2+F3, two-block F1, 80 small blocks): L_X^-1, L_Z^-1, Z^-1, the residuals, the
    Schur matrix B, the predictor and corrector right-hand sides and the
    directions Dx, Dy, Dz of the reference's own pinpal state.
The step-length eigenvalue (Lanczos / small-block path) must agree within
1e-25 (relative to max(1, |lambda|)): its tridiagonal eigensolver differs
from the reference's QR by design, and both are accurate to dd rounding of
the spectrum's scale, not of lambda_min itself.
"""
import ctypes

import numpy as np
import pytest

from conftest import DD, RefSolver, as_dd, load_pkg, ptr


def sddd_dd(hi, lo):
    return load_pkg().SdddDD(hi, lo)
from test_oracle import adversarial, rand_dd, same, spd

pytestmark = pytest.mark.gpu

SMALL = {
    "dense": lambda P: P.dense_random(n=12, m=20, seed=10),
    "maxcut": lambda P: P.maxcut(n=30, p=0.2, seed=11),
    "theta": lambda P: P.theta(nv=24, p=0.5, seed=12),
    "control": lambda P: P.control_like(sizes=(9, 6), m=25, seed=13),
    "dense_big": lambda P: P.dense_random(n=50, m=40, seed=14),
    # 80 dense blocks of orders 2..8 (more per-block results than the
    # solver's earlier fixed scratch held)
    "blocks80": lambda P: P.blocks_with_lp(sizes=np.random.default_rng(21).integers(2, 9, 80), q=0, m=60, seed=21),
}


@pytest.fixture(scope="module")
def sddd():
    return load_pkg()


@pytest.fixture(scope="module")
def problems(workdir):
    P = load_pkg()
    import importlib
    prob = importlib.import_module("sdpa_dd_b200.problems")
    out = {}
    for name, make in SMALL.items():
        path = workdir / f"gpu_{name}.dat-s"
        path.write_text(make(prob))
        out[name] = path
    return out


def to_dev(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).cuda()
    return t


def from_dev(t, n):
    out = t.cpu().numpy().view(DD)
    return out[:n].copy()


@pytest.mark.parametrize("op", list(range(18)))
def test_device_dd_ops_match_qd(sddd, ref_lib, op):
    import torch
    L = sddd.lib()
    rng = np.random.default_rng(300 + op)
    n = 20000
    a, b = adversarial(rng, n), adversarial(rng, n)
    if op == 7:
        a["hi"], a["lo"] = np.abs(a["hi"]), np.where(a["hi"] < 0, -a["lo"], a["lo"])
    b["hi"][:500] = -a["hi"][:500]
    da, db = to_dev(a), to_dev(b)
    dout = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    assert L.sddd_dd_op(None, op, n, ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(dout.data_ptr())) == 0
    got = from_dev(dout, n)
    want = np.zeros(n, DD)
    ref_lib.ref_dd_op(op, ctypes.c_long(n), ptr(a), ptr(b), ptr(want))
    assert same(got, want)


@pytest.fixture(scope="module")
def ctx(sddd):
    c = sddd.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (65, 33, 17), (130, 70, 129)])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("ab", ["one_zero", "random", "zero_alpha", "one_beta"])
def test_device_gemm_matches_rgemm(ctx, ref_lib, m, n, k, ta, tb, ab):
    """sddd_Rgemm (MPLAPACK's argument list) against the reference's own
    Rgemm (oracle/_ref), alpha and beta included, bit for bit."""
    import torch
    rng = np.random.default_rng(m + 7 * n + 13 * k)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    A, B, C = rand_dd(rng, ra * ca), rand_dd(rng, rb * cb), rand_dd(rng, m * n)
    alpha, beta = {"one_zero": ((1.0, 0.0), (0.0, 0.0)), "zero_alpha": ((0.0, 0.0), (0.75, 0.0)), "one_beta": ((-2.5, 1e-17), (1.0, 0.0)),
                   "random": ((rng.standard_normal(), 3e-18), (rng.standard_normal(), -2e-18))}[ab]
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rc = ctx.L.sddd_Rgemm(ctx.h, ta.encode(), tb.encode(), m, n, k, sddd_dd(*alpha), ctypes.c_void_p(dA.data_ptr()), ra,
                          ctypes.c_void_p(dB.data_ptr()), rb, sddd_dd(*beta), ctypes.c_void_p(dC.data_ptr()), m)
    assert rc == 0, ctx.L.sddd_last_error(ctx.h)
    want = C.copy()
    al, be = np.array([alpha], DD), np.array([beta], DD)
    ref_lib.ref_Rgemm(ta.encode(), tb.encode(), ctypes.c_long(m), ctypes.c_long(n), ctypes.c_long(k), ptr(al), ptr(A), ctypes.c_long(ra), ptr(B),
                      ctypes.c_long(rb), ptr(be), ptr(want), ctypes.c_long(m))
    assert same(from_dev(dC, m * n), want)


def test_dd_blas_argument_checks(ctx):
    """Bad arguments are reported with the position the reference's
    Mxerbla_dd names; forms SDPA never calls are refused, not guessed."""
    one = sddd_dd(1.0, 0.0)
    assert ctx.L.sddd_Rgemm(ctx.h, b"X", b"N", 2, 2, 2, one, None, 2, None, 2, one, None, 2) == -1
    assert b"parameter 1" in ctx.L.sddd_last_error(ctx.h)
    assert ctx.L.sddd_Rgemm(ctx.h, b"N", b"N", 4, 2, 2, one, None, 3, None, 2, one, None, 4) == -1
    assert b"parameter 8" in ctx.L.sddd_last_error(ctx.h)
    assert ctx.L.sddd_Rtrsv(ctx.h, b"L", b"N", b"N", 3, None, 3, None, 0) == -1
    assert b"parameter 8" in ctx.L.sddd_last_error(ctx.h)
    assert ctx.L.sddd_Rtrsv(ctx.h, b"U", b"N", b"N", 3, None, 3, None, 1) == -7
    assert ctx.L.sddd_Rpotrf(ctx.h, b"Q", 3, None, 3) == -1
    assert ctx.L.sddd_Rpotrf(ctx.h, b"U", 3, None, 3) == -7
    assert ctx.L.sddd_Rpotrs(ctx.h, b"L", 3, 1, None, 2, None, 3) == -1
    assert b"parameter 5" in ctx.L.sddd_last_error(ctx.h)
    # a device base off the 16-byte dd alignment is refused on the host,
    # before anything reads it
    buf = to_dev(np.zeros(32, DD))
    odd = ctypes.c_void_p(buf.data_ptr() + 8)
    assert ctx.L.sddd_Rpotrf(ctx.h, b"L", 3, odd, 3) == -1
    assert b"parameter 3" in ctx.L.sddd_last_error(ctx.h) and b"16-byte" in ctx.L.sddd_last_error(ctx.h)
    ok = ctypes.c_void_p(buf.data_ptr())
    assert ctx.L.sddd_Rgemm(ctx.h, b"N", b"N", 2, 2, 2, one, ok, 2, odd, 2, one, ok, 2) == -1
    assert b"parameter 9" in ctx.L.sddd_last_error(ctx.h)
    assert ctx.L.sddd_Rtrsv(ctx.h, b"L", b"N", b"N", 3, ok, 3, odd, 1) == -1
    assert b"parameter 7" in ctx.L.sddd_last_error(ctx.h)


@pytest.mark.parametrize("n", [1, 5, 33, 63, 64, 65, 130, 257, 700])
def test_device_potrf_trsv_match(ctx, oracle_lib, n):
    rng = np.random.default_rng(500 + n)
    A = spd(rng, n)
    A["lo"] = rng.standard_normal(n * n) * 1e-18
    want = A.copy()
    info = oracle_lib.o_potrf(ctypes.c_long(n), ptr(want), ctypes.c_long(n))
    assert info == 0
    dA = to_dev(A)
    got_info = ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA.data_ptr()), n)
    assert got_info == 0
    got = from_dev(dA, n * n).reshape(n, n)
    w = want.reshape(n, n)
    for j in range(n):  # lower triangle of column j = row j of the (col-major) view
        assert same(got[j, j:], w[j, j:]), j
    # solves with the factor
    b = rand_dd(rng, n)
    for tr in ("N", "T"):
        x = b.copy()
        oracle_lib.o_trsv(ctypes.c_char(tr.encode()), ctypes.c_long(n), ptr(want), ctypes.c_long(n), ptr(x))
        dx = to_dev(b)
        ctx.L.sddd_Rtrsv(ctx.h, b"L", tr.encode(), b"N", n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(dx.data_ptr()), 1)
        assert same(from_dev(dx, n), x), tr


@pytest.mark.parametrize("n,lda", [(300, 320), (9800, 9800)])
def test_device_trsv_wavefront_matches_rtrsv(ctx, oracle_lib, n, lda):
    """The one-launch solve with more 64-entry blocks than co-resident CTAs
    (9800 = 153 full blocks + 8), a leading dimension above n and zero
    right-hand-side entries (the forward loop's skip)."""
    rng = np.random.default_rng(n)
    L = np.zeros(lda * n, DD)
    for j in range(n):
        col = L[j * lda:(j + 1) * lda]
        col["hi"][j] = 1.0 + rng.random()
        col["hi"][j + 1:n] = rng.standard_normal(n - j - 1) / np.sqrt(n)
        col["lo"][j:n] = col["hi"][j:n] * rng.uniform(-1, 1, n - j) * 1e-17
    dL = to_dev(L)
    for tr in ("N", "T"):
        b = rand_dd(rng, n)
        b[rng.random(n) < 0.05] = (0.0, 0.0)
        x = b.copy()
        oracle_lib.o_trsv(ctypes.c_char(tr.encode()), ctypes.c_long(n), ptr(L), ctypes.c_long(lda), ptr(x))
        dx = to_dev(b)
        assert ctx.L.sddd_Rtrsv(ctx.h, b"L", tr.encode(), b"N", n, ctypes.c_void_p(dL.data_ptr()), lda, ctypes.c_void_p(dx.data_ptr()), 1) == 0
        assert same(from_dev(dx, n), x), tr


@pytest.mark.parametrize("col", [0, 31, 32, 63, 97, 127, 149])
def test_device_potrf_reports_failing_column(ctx, oracle_lib, col):
    """A negative pivot at the first and last column of a diagonal block,
    either side of the block's 32-column halves, and the matrix's last
    column: the 1-based column comes back, as Rpotrf's info does."""
    rng = np.random.default_rng(9)
    n = 150
    A = spd(rng, n)
    A["hi"][col * n + col] = -3.0
    want = A.copy()
    i1 = oracle_lib.o_potrf(ctypes.c_long(n), ptr(want), ctypes.c_long(n))
    dA = to_dev(A)
    i2 = ctx.L.sddd_Rpotrf(ctx.h, b"L", n, ctypes.c_void_p(dA.data_ptr()), n)
    assert i1 == i2 == col + 1


def _dd_scalar_eq(a, b):
    return (a[0] == b["hi"] or (a[0] == 0 and b["hi"] == 0)) and (a[1] == b["lo"] or (a[1] == 0 and b["lo"] == 0))


@pytest.mark.parametrize("name", list(SMALL))
@pytest.mark.parametrize("k", [0, 2, 6])
def test_newton_pieces_match_reference(sddd, ctx, ref_lib, problems, name, k):
    """Set the GPU to the reference's point before its pass k+1 and replay
    that pass piece by piece."""
    path = problems[name]
    ref = RefSolver(ref_lib, path)
    try:
        ctx.read_problem(path, sparse=True, kappa=1.2)
        assert ctx.m == ref.m and ctx.sizes == ref.blocks
        f_ref = ref.formula()
        assert np.array_equal(ctx.formula(), f_ref)
        for _ in range(k):
            assert ref.step() == 0
        X, y, Z = ref.get(0), ref.get(2), ref.get(1)
        if k == 0:
            # Solutions::initialize sets the inverses directly (lambda I)
            ctx.call("sddd_init_point", sddd.SdddDD(1.0e4, 0.0))
        else:
            assert ctx.set_point(X, y, Z) == 0
        for w_ref, w_gpu in ((3, "invCholX"), (4, "invCholZ"), (5, "invZ")):
            r_ = same(ctx.get(w_gpu), ref.get(w_ref))
            assert r_, (w_gpu, r_)
        ctx.dd_scalar("sddd_residuals", ctypes.byref(sddd.SdddDD()))  # residuals of the point
        r_ = same(ctx.get("dualMat"), ref.get(15))
        assert r_, ("dualMat", r_)
        r_ = same(ctx.get("primalVec"), ref.get(16))
        assert r_, ("primalVec", r_)
        # one reference pass
        rc = ref.step()
        assert rc == 0
        phase = ref_lib.ref_phase_at_step(ref.h)
        dinf = int(phase in (0, 1))  # noINFO or pFEAS
        beta_p, mu = ref.scalar(16), ref.scalar(19)
        # predictor: RHS, Schur, Cholesky, Dy, Dz, Dx
        import importlib
        bm = _ddmul(ref_lib, beta_p, mu)
        ctx.call("sddd_newton_rhs", 0, sddd.SdddDD(*bm), dinf)
        r_ = same(ctx.get("g"), ref.get(8))
        assert r_, ("g (predictor)", r_)
        ctx.call("sddd_schur_build")
        B = ctx.get("B")
        r_ = same(B, _ref_B_at(ref_lib, path, X, y, Z, k))
        assert r_, ("Schur matrix", r_)
        assert ctx.call("sddd_schur_factor") == 0
        ctx.call("sddd_solve_dy")
        r_ = same(ctx.get("Dy"), ref.get(13))
        assert r_, ("Dy (predictor)", r_)
        ctx.call("sddd_make_dz_dx", dinf)
        r_ = same(ctx.get("Dz"), ref.get(14))
        assert r_, ("Dz (predictor)", r_)
        r_ = same(ctx.get("Dx"), ref.get(12))
        assert r_, ("Dx (predictor)", r_)
        # corrector
        beta_c = ref.scalar(6)
        bm = _ddmul(ref_lib, beta_c, mu)
        ctx.call("sddd_newton_rhs", 1, sddd.SdddDD(*bm), dinf)
        ctx.call("sddd_solve_dy")
        r_ = same(ctx.get("Dy"), ref.get(10))
        assert r_, ("Dy (corrector)", r_)
        ctx.call("sddd_make_dz_dx", dinf)
        r_ = same(ctx.get("Dz"), ref.get(11))
        assert r_, ("Dz (corrector)", r_)
        r_ = same(ctx.get("Dx"), ref.get(9))
        assert r_, ("Dx (corrector)", r_)
        # step-length eigenvalues
        for which, sel in ((0, 17), (1, 18)):
            got = ctx.dd_scalar("sddd_min_eig", which)
            want = ref.scalar(sel)
            diff = (got[0] - want["hi"]) + (got[1] - want["lo"])
            assert abs(diff) <= 1e-25 * max(1.0, abs(want["hi"])), (which, got, want)
    finally:
        ref.close()


def _ddmul(ref_lib, a, b):
    aa = np.array([a], DD)
    bb = np.array([b], DD)
    out = np.zeros(1, DD)
    ref_lib.ref_dd_op(4, ctypes.c_long(1), ptr(aa), ptr(bb), ptr(out))
    return float(out["hi"][0]), float(out["lo"][0])


def _ref_B_at(ref_lib, path, X, y, Z, k):
    """The reference's B at point (X, y, Z): a second reference solver set to
    that point (Make_bMat reads X and Z^-1 only)."""
    r = RefSolver(ref_lib, path)
    try:
        if k > 0:
            assert ref_lib.ref_set_point(r.h, ptr(X), ptr(y), ptr(Z)) == 0
        return r.schur()
    finally:
        r.close()
