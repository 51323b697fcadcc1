"""Exact decimal printing of dd values (sddd_dd_to_decimal), the number
format of the full-precision point files that sddd_write_point writes.

The reference writes only the high double of its results; the point files
carry 34 significant digits of hi + lo.  Here every printed string must be
hi + lo correctly rounded (half to even) to the requested digits, checked
with Python's exact decimal arithmetic; no GPU is needed."""
import ctypes
import math
import random
from decimal import ROUND_HALF_EVEN, Context, Decimal

import pytest

from conftest import load_pkg


def _lib():
    sddd = load_pkg()
    return sddd, sddd.lib()


def _exact(hi, lo):
    # a double's Decimal is exact; 2200 digits hold any sum of two doubles
    return Context(prec=2200).add(Decimal(hi), Decimal(lo))


def _want(hi, lo, digits):
    v = _exact(hi, lo)
    if v == 0:
        return Decimal(0)
    return Context(prec=digits, rounding=ROUND_HALF_EVEN, Emax=999999, Emin=-999999).plus(v)


def _print(L, sddd, hi, lo, digits):
    buf = ctypes.create_string_buffer(128)
    n = L.sddd_dd_to_decimal(sddd.SdddDD(hi, lo), digits, buf, 128)
    assert n > 0
    return buf.value.decode()


def _cases():
    rng = random.Random(5)
    out = [(1.0, 0.0), (-1.0, 0.0), (0.1, 5.551115123125783e-18), (1.0, 2.0 ** -60), (1.0, -(2.0 ** -60)), (5e-324, 0.0), (1.7976931348623157e308, 0.0),
           (2.0 ** -1022, 2.0 ** -1074), (123456789.0, -1e-9), (9.999999999999999e22, 4e6)]
    for _ in range(400):
        hi = math.ldexp(rng.uniform(0.5, 1.0), rng.randint(-1000, 1000)) * rng.choice([-1, 1])
        e = math.frexp(hi)[1]
        lo = math.ldexp(rng.uniform(-0.5, 0.5), e - 53) if rng.random() < 0.9 else 0.0
        out.append((hi, lo))
    return out


@pytest.mark.parametrize("digits", [1, 17, 34, 40])
def test_decimal_strings_are_correctly_rounded(digits):
    sddd, L = _lib()
    for hi, lo in _cases():
        s = _print(L, sddd, hi, lo, digits)
        got = Decimal(s)
        want = _want(hi, lo, digits)
        assert got == want, (hi, lo, digits, s, str(want))
        # at most `digits` significant digits in the mantissa
        mant = s.lstrip("-").split("e")[0].replace(".", "")
        assert len(mant) <= digits


def test_special_values():
    sddd, L = _lib()
    assert _print(L, sddd, 0.0, 0.0, 34) == "0"
    assert _print(L, sddd, math.inf, 0.0, 34) == "inf"
    assert _print(L, sddd, -math.inf, 0.0, 34) == "-inf"
    assert _print(L, sddd, math.nan, 0.0, 34) == "nan"
    buf = ctypes.create_string_buffer(8)
    assert L.sddd_dd_to_decimal(sddd.SdddDD(1.0, 0.0), 0, buf, 8) < 0  # digits out of range
    # a short buffer truncates but reports the full length
    n = L.sddd_dd_to_decimal(sddd.SdddDD(math.pi, 1.2246467991473532e-16), 34, buf, 8)
    assert n == len("3.141592653589793238462643383279503e+00") and buf.value.decode() == "3.14159"


def test_34_digits_read_back_within_a_few_dd_ulps():
    """The reader (QD's parser, as the reference's) turns a 34-digit string
    back into the dd to within a few units of 2^-104 of the value.  Outside
    1e-200 .. 1e200 the reader's own power of ten (10^e, e near -300) has a
    subnormal low part and the read loses dd precision whatever the digits,
    so the check stays inside that range."""
    sddd, L = _lib()
    out = (ctypes.c_double * 2)()
    for hi, lo in _cases():
        if abs(hi) < 1e-200 or abs(hi) > 1e200:
            continue
        s = _print(L, sddd, hi, lo, 34)
        assert L.sddd_host_dd_read(s.encode(), out) == 0
        err = abs(_exact(out[0], out[1]) - _exact(hi, lo))
        assert err <= Decimal(8) * Decimal(2) ** -104 * abs(_exact(hi, lo)), (hi, lo, s)
