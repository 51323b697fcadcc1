"""The CPU restatement (oracle/) pinned against the reference build
(oracle/_ref): QD arithmetic, the decimal reader, the MPLAPACK kernels in
the order the reference runs them, the Schur complement and the Lanczos
step-length eigenvalue.  Integer/bit work is compared bit for bit; the
Lanczos value within 1e-26 relative (its tridiagonal eigensolver differs
by design: bisection + inverse iteration instead of implicit QR)."""
import ctypes

import numpy as np
import pytest

from conftest import DD, as_dd, ptr

c_long = ctypes.c_long


def rand_dd(rng, n, scale=1.0):
    hi = rng.standard_normal(n) * scale
    lo = hi * rng.uniform(-1, 1, n) * 2.0 ** -53
    out = np.zeros(n, dtype=DD)
    out["hi"] = hi + lo  # renormalise
    out["lo"] = (hi - out["hi"]) + lo
    return out


def adversarial(rng, n):
    base = rand_dd(rng, n)
    base["hi"][: n // 4] = np.ldexp(1.0, rng.integers(-60, 60, n // 4))
    base["lo"][: n // 4] = 0.0
    base["hi"][n // 4: n // 2] *= 1e30
    base["lo"][n // 4: n // 2] *= 1e30
    return base


def bits(a):
    return a.view(np.uint64)


class Same:
    """Truthy when two dd arrays are bitwise equal (+0 == -0); otherwise
    falsy and its repr names the first differing entry."""

    def __init__(self, a, b):
        a = np.asarray(a).view(np.float64).copy()
        b = np.asarray(b).view(np.float64).copy()
        a[a == 0] = 0.0
        b[b == 0] = 0.0
        self.ok = a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
        self.msg = "equal"
        if not self.ok:
            if a.shape != b.shape:
                self.msg = f"shapes {a.shape} vs {b.shape}"
            else:
                bad = np.nonzero(a.view(np.uint64) != b.view(np.uint64))[0]
                i = int(bad[0]) // 2
                self.msg = (f"{len(bad)} doubles differ; first dd #{i}: got ({a[2*i]!r}, {a[2*i+1]!r}) want ({b[2*i]!r}, {b[2*i+1]!r})"
                            f"; max |diff| {np.max(np.abs(a - b)):.3e}")

    def __bool__(self):
        return self.ok

    def __repr__(self):
        return self.msg


def same(a, b):
    """bitwise equal, treating +0 and -0 as equal"""
    return Same(a, b)


@pytest.mark.parametrize("op", list(range(18)))
def test_dd_ops_match_qd(oracle_lib, ref_lib, op):
    rng = np.random.default_rng(100 + op)
    n = 4000
    a, b = adversarial(rng, n), adversarial(rng, n)
    if op in (7,):
        a["hi"], a["lo"] = np.abs(a["hi"]), np.where(a["hi"] < 0, -a["lo"], a["lo"])
    # cancellation cases for add/sub
    b["hi"][:200] = -a["hi"][:200]
    b["lo"][:200] = rng.standard_normal(200) * 1e-20
    o1 = np.zeros(n, DD)
    o2 = np.zeros(n, DD)
    oracle_lib.o_dd_op(op, c_long(n), ptr(a), ptr(b), ptr(o1))
    ref_lib.ref_dd_op(op, c_long(n), ptr(a), ptr(b), ptr(o2))
    assert same(o1, o2)


def test_decimal_reader_matches_qd(oracle_lib, ref_lib):
    rng = np.random.default_rng(7)
    strs = ["0", "1", "-1", "0.5", "1.0E4", "1.0E-30", "+1.0e+00", "0.250000", "-0.250000", "123456789012345678901234567890",
            "3.14159265358979323846264338327950288", "1e-300", "9.999999999999999e299", "2.", "-.0"]
    for _ in range(3000):
        v = rng.standard_normal() * 10.0 ** rng.integers(-40, 40)
        strs.append(repr(float(v)))
        strs.append("%.25e" % v)
        strs.append("%.3f" % (v % 1000))
    for s in strs:
        o1 = np.zeros(1, DD)
        o2 = np.zeros(1, DD)
        r1 = oracle_lib.o_dd_read(s.encode(), ptr(o1))
        r2 = ref_lib.ref_dd_read(s.encode(), ptr(o2))
        assert r1 == r2, s
        assert same(o1, o2), (s, o1, o2)


def _mat(rng, n, m=None):
    return rand_dd(rng, n * (m or n)).reshape((m or n), n).T.copy()  # column-major storage via transpose copy


def spd(rng, n):
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    out = np.zeros(n * n, DD)
    out["hi"] = A.T.ravel()
    return out


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (33, 17, 65), (64, 64, 64)])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_gemm_matches_rgemm(oracle_lib, ref_lib, m, n, k, ta, tb):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    A = rand_dd(rng, ra * ca)
    B = rand_dd(rng, rb * cb)
    C1 = np.zeros(m * n, DD)
    C2 = rand_dd(rng, m * n)  # beta = 0 overwrites
    one = as_dd([1.0])
    zero = as_dd([0.0])
    oracle_lib.o_gemm(ctypes.c_char(ta.encode()), ctypes.c_char(tb.encode()), c_long(m), c_long(n), c_long(k), ptr(A), c_long(ra), ptr(B), c_long(rb), ptr(C1), c_long(m))
    ref_lib.ref_Rgemm(ta.encode(), tb.encode(), c_long(m), c_long(n), c_long(k), ptr(one), ptr(A), c_long(ra), ptr(B), c_long(rb), ptr(zero), ptr(C2), c_long(m))
    assert same(C1, C2)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 63, 64, 65, 100, 129, 200])
def test_potrf_matches_rpotrf(oracle_lib, ref_lib, n):
    rng = np.random.default_rng(n)
    A = spd(rng, n)
    A["lo"] = rng.standard_normal(n * n) * 1e-18 * (A["hi"] != 0)
    A1, A2 = A.copy(), A.copy()
    i1 = oracle_lib.o_potrf(c_long(n), ptr(A1), c_long(n))
    i2 = ref_lib.ref_Rpotrf(b"Lower", c_long(n), ptr(A2), c_long(n))
    assert i1 == i2 == 0
    L1 = A1.reshape(n, n).T  # row-major view of column-major
    L2 = A2.reshape(n, n).T
    assert same(np.tril(L1["hi"]), np.tril(L2["hi"])) and same(np.tril(L1["lo"]), np.tril(L2["lo"]))


def test_potrf_failure_column(oracle_lib, ref_lib):
    rng = np.random.default_rng(5)
    n = 90
    A = spd(rng, n)
    A["hi"][70 * n + 70] = -5.0  # indefinite at column 71 (1-based)
    A1, A2 = A.copy(), A.copy()
    i1 = oracle_lib.o_potrf(c_long(n), ptr(A1), c_long(n))
    i2 = ref_lib.ref_Rpotrf(b"Lower", c_long(n), ptr(A2), c_long(n))
    assert i1 == i2 == 71


@pytest.mark.parametrize("n", [1, 5, 64, 150])
def test_triangular_kernels_match(oracle_lib, ref_lib, n):
    rng = np.random.default_rng(1000 + n)
    A = spd(rng, n)
    ref_lib.ref_Rpotrf(b"Lower", c_long(n), ptr(A), c_long(n))
    L = A.copy()
    Lm = L.reshape(n, n)
    for j in range(n):  # zero the strict upper part (column-major: row index fastest)
        Lm[j, :j] = np.zeros(j, DD)
    b = rand_dd(rng, n)
    for tr in ("N", "T"):
        x1, x2 = b.copy(), b.copy()
        oracle_lib.o_trsv(ctypes.c_char(tr.encode()), c_long(n), ptr(L), c_long(n), ptr(x1))
        ref_lib.ref_Rtrsv(b"Lower", tr.encode(), b"NonUnit", c_long(n), ptr(L), c_long(n), ptr(x2), c_long(1))
        assert same(x1, x2), tr
        x1, x2 = b.copy(), b.copy()
        oracle_lib.o_trmv(ctypes.c_char(tr.encode()), c_long(n), ptr(L), c_long(n), ptr(x1))
        ref_lib.ref_Rtrmv(b"Lower", tr.encode(), b"NotUnit", c_long(n), ptr(L), c_long(n), ptr(x2), c_long(1))
        assert same(x1, x2), tr
    # inverse of L (Rtrsm on identity) and L^-T L^-1 (Rtrmm)
    X1 = np.zeros(n * n, DD)
    oracle_lib.o_inv_lower(c_long(n), ptr(L), c_long(n), ptr(X1), c_long(n))
    X2 = np.zeros(n * n, DD)
    X2["hi"][:: n + 1] = 1.0
    one = as_dd([1.0])
    ref_lib.ref_Rtrsm(b"Left", b"Lower", b"NoTraspose", b"NonUnitDiagonal", c_long(n), c_long(n), ptr(one), ptr(L), c_long(n), ptr(X2), c_long(n))
    assert same(X1, X2)
    Y1, Y2 = X1.copy(), X1.copy()
    oracle_lib.o_trmm_lt(c_long(n), ptr(X1), c_long(n), ptr(Y1), c_long(n))
    ref_lib.ref_Rtrmm(b"Left", b"Lower", b"Transpose", b"NonUnitDiag", c_long(n), c_long(n), ptr(one), ptr(X1), c_long(n), ptr(Y2), c_long(n))
    assert same(Y1, Y2)
    # gemv and dot
    M = rand_dd(rng, n * n)
    y1 = np.zeros(n, DD)
    y2 = rand_dd(rng, n)
    zero = as_dd([0.0])
    oracle_lib.o_gemv(c_long(n), c_long(n), ptr(M), c_long(n), ptr(b), ptr(y1))
    ref_lib.ref_Rgemv(b"NoTranspose", c_long(n), c_long(n), ptr(one), ptr(M), c_long(n), ptr(b), c_long(1), ptr(zero), ptr(y2), c_long(1))
    assert same(y1, y2)


def test_dot_matches_rdot(oracle_lib, ref_lib):
    rng = np.random.default_rng(11)
    n = 5000
    x, y = rand_dd(rng, n), rand_dd(rng, n)
    oracle_lib.o_dot.restype = None
    r1 = np.zeros(1, DD)
    r2 = np.zeros(1, DD)
    # o_dot returns a struct by value: call through a tiny shim with restype
    class ODD(ctypes.Structure):
        _fields_ = [("hi", ctypes.c_double), ("lo", ctypes.c_double)]
    oracle_lib.o_dot.restype = ODD
    v = oracle_lib.o_dot(c_long(n), ptr(x), c_long(1), ptr(y), c_long(1))
    r1["hi"], r1["lo"] = v.hi, v.lo
    ref_lib.ref_Rdot(c_long(n), ptr(x), c_long(1), ptr(y), c_long(1), ptr(r2))
    assert same(r1, r2)
