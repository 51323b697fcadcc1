"""The C-ABI library without a GPU: it loads, exports every entry point
include/sddd.h declares, and its host-side dd arithmetic, decimal reader and
32-digit printer equal QD's (the reference build) bit for bit."""
import ctypes
import re

import numpy as np
import pytest

from conftest import DD, ROOT, load_pkg, ptr
from test_oracle import adversarial, same


def declared_symbols():
    text = (ROOT / "include" / "sddd.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(sddd_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    sddd = load_pkg()
    L = sddd.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert b"sm_100a" in L.sddd_version()


@pytest.mark.parametrize("op", list(range(18)))
def test_host_dd_ops_match_qd(ref_lib, op):
    L = load_pkg().lib()
    rng = np.random.default_rng(200 + op)
    n = 3000
    a, b = adversarial(rng, n), adversarial(rng, n)
    if op == 7:
        a["hi"], a["lo"] = np.abs(a["hi"]), np.where(a["hi"] < 0, -a["lo"], a["lo"])
    b["hi"][:100] = -a["hi"][:100]
    o1, o2 = np.zeros(n, DD), np.zeros(n, DD)
    assert L.sddd_host_dd_op(op, n, ptr(a), ptr(b), ptr(o1)) == 0
    ref_lib.ref_dd_op(op, ctypes.c_long(n), ptr(a), ptr(b), ptr(o2))
    assert same(o1, o2)


def test_host_decimal_reader_matches_qd(ref_lib):
    L = load_pkg().lib()
    rng = np.random.default_rng(3)
    strs = ["0", "-0.250000", "+1.0e+00", "1.0E-30", "123456789012345678901234567890", "2.", "-.5"]
    for _ in range(2000):
        v = rng.standard_normal() * 10.0 ** rng.integers(-30, 30)
        strs += [repr(float(v)), "%.20e" % v]
    for s in strs:
        o1, o2 = np.zeros(1, DD), np.zeros(1, DD)
        r1 = L.sddd_host_dd_read(s.encode(), ptr(o1))
        r2 = ref_lib.ref_dd_read(s.encode(), ptr(o2))
        assert r1 == r2 and same(o1, o2), s


def test_host_32_digit_output_matches_qd(ref_lib):
    sddd = load_pkg()
    L = sddd.lib()
    rng = np.random.default_rng(4)
    vals = [(-41.9, 0.0), (0.0, 0.0), (1.0, 0.0), (-4.19e1, 5.4e-15), (9.999999999999999e-1, 9e-17), (1e300, 0.0), (1e-300, 0.0)]
    for _ in range(2000):
        hi = rng.standard_normal() * 10.0 ** rng.integers(-40, 40)
        vals.append((hi, hi * rng.uniform(-1, 1) * 2.0 ** -53))
    buf1 = ctypes.create_string_buffer(128)
    buf2 = ctypes.create_string_buffer(128)
    for hi, lo in vals:
        s = hi + lo
        lo2 = (hi - s) + lo
        d = sddd.SdddDD(s, lo2)
        n1 = L.sddd_host_dd_to_string(d, 32, buf1, 128)
        a = np.array([(s, lo2)], DD)
        n2 = ref_lib.ref_dd_to_string(ptr(a), 32, buf2, 128)
        assert n1 > 0 and n2 > 0
        assert buf1.value == buf2.value, (hi, lo, buf1.value, buf2.value)


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    sddd = load_pkg()
    L = sddd.lib()
    h = ctypes.c_void_p()
    rc = L.sddd_create(0, ctypes.byref(h))
    assert rc < 0 and not h.value
    assert L.sddd_last_error(None)
