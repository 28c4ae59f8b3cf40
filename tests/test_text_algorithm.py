"""The device "%e" algorithm of k_text.cu, restated in Python, against libc's
printf (CPU only).  The restatement follows the kernel step for step: the
decimal exponent from the binary one, the value times 10^(6-E) as a
double-double from the table in mph_pow10.h (with the kernel's 2^256 scaling),
the rounding decided from the high part unless it is a half-integer within
2^-70 of the scaled value, and then an exact comparison.  FMA is evaluated
exactly (rational arithmetic, one rounding), as the device's is.  So the
algorithm and its table are checked on every kind of value without a GPU; the
kernel itself is checked against printf in tests/test_gpu_text.py."""
import ctypes as C
import math
import os
import re
from fractions import Fraction

import numpy as np

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mphexplicit_b200", "csrc")


def _table():
    t = {}
    with open(os.path.join(CSRC, "mph_pow10.h")) as f:
        for line in f:
            m = re.match(r"\s*\{(\S+), (\S+)\},\s*// (-?\d+)", line)
            if m:
                t[int(m.group(3))] = (float.fromhex(m.group(1)), float.fromhex(m.group(2)))
    return t


TABLE = _table()


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _scaled(x, s):
    hi, lo = TABLE[s]
    xs = x * 2.0 ** 256 if s > 250 else (x * 2.0 ** -256 if s < -250 else x)
    p = xs * hi
    pe = _fma(xs, hi, -p)
    c = _fma(xs, lo, pe)
    qh = p + c
    return qh, c - (qh - p)


def device_format_e(x: float) -> str:
    bits = np.float64(x).view(np.uint64).item()
    sign = "-" if bits >> 63 else ""
    be, fr = (bits >> 52) & 0x7FF, bits & ((1 << 52) - 1)
    if be == 0x7FF:
        return sign + ("nan" if fr else "inf")
    if be == 0 and fr == 0:
        return sign + "0.000000e+00"
    m = (fr | (1 << 52)) if be else fr
    e = be - 1075 if be else -1074
    ax = abs(x)
    E = ((e + m.bit_length() - 1) * 78913) >> 18
    qh, ql = _scaled(ax, 6 - E)
    if qh < 1e6:
        E -= 1
        qh, ql = _scaled(ax, 6 - E)
    elif qh >= 1e7:
        E += 1
        qh, ql = _scaled(ax, 6 - E)
    r = math.floor(qh)
    f = qh - r
    if f != 0.5:
        up = f > 0.5
    elif abs(ql) > 2.0 ** -70:
        up = ql > 0
    else:  # exact: sign of m 2^e 10^s - (r + 1/2), ties to even
        d = Fraction(m) * Fraction(2) ** e * Fraction(10) ** (6 - E) - (Fraction(r) + Fraction(1, 2))
        up = d > 0 or (d == 0 and r % 2 == 1)
    r += 1 if up else 0
    if r >= 10 ** 7:
        r, E = 10 ** 6, E + 1
    digits = str(r)
    return "%s%s.%se%s%02d" % (sign, digits[0], digits[1:], "-" if E < 0 else "+", abs(E))


def _printf(v: float) -> str:
    buf = C.create_string_buffer(64)
    n = C.CDLL(None).snprintf(buf, 64, b"%e", C.c_double(v))
    return buf.raw[:n].decode()


def _values():
    rng = np.random.default_rng(3)
    ties = np.concatenate([np.arange(129, 1280, 2)[::8] / 128.0, np.arange(641, 6400, 2)[::40] / 64.0,
                           np.array([12345675.0, 12345665.0, 0.0029296875, 1.0078125])])
    p10 = 10.0 ** np.arange(-300, 300, 7, dtype=np.float64)
    bits = rng.integers(0, 2 ** 63, size=3000, dtype=np.int64).view(np.float64)
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 2.2250738585072014e-308,
                        1.7976931348623157e308, 9.9999995, 999999.5, 3.4028234663852886e38])
    v = np.concatenate([ties, -ties, np.nextafter(ties, np.inf), p10, np.nextafter(p10, 0), p10 * 9.9999995,
                        bits[np.isfinite(bits)], rng.normal(0, 1, 500), special])
    return v


def test_restated_algorithm_equals_printf_for_doubles_and_floats():
    vals = _values()
    with np.errstate(over="ignore"):
        as_float = vals.astype(np.float32).astype(np.float64)
    for arr in (vals, as_float):
        bad = [(float(v), device_format_e(float(v)), _printf(float(v))) for v in arr
               if device_format_e(float(v)) != _printf(float(v))]
        assert not bad, bad[:5]
