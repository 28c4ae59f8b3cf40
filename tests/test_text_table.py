"""The power-of-ten table of the device "%e" formatter (CPU only): the
committed header is what its generator prints, and every entry is the
double-double of 10^s * 2^-scale(s) to within 2^-106 relative."""
import os
import re
import subprocess
import sys
from fractions import Fraction

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mphexplicit_b200", "csrc")


def test_header_is_generated():
    out = subprocess.run([sys.executable, os.path.join(CSRC, "gen_pow10.py")], capture_output=True, text=True,
                         check=True).stdout
    with open(os.path.join(CSRC, "mph_pow10.h")) as f:
        assert f.read() == out


def test_entries_are_double_double_of_powers_of_ten():
    n = 0
    with open(os.path.join(CSRC, "mph_pow10.h")) as f:
        for line in f:
            m = re.match(r"\s*\{(\S+), (\S+)\},\s*// (-?\d+)", line)
            if not m:
                continue
            hi, lo, s = float.fromhex(m.group(1)), float.fromhex(m.group(2)), int(m.group(3))
            sc = 256 if s > 250 else (-256 if s < -250 else 0)
            v = Fraction(10) ** s * Fraction(2) ** (-sc)
            assert abs(hi) >= 2.0 ** -1022 and (lo == 0.0 or abs(lo) >= 2.0 ** -1022), s  # both normal
            assert abs(Fraction(hi) + Fraction(lo) - v) <= v * Fraction(1, 2 ** 106), s
            n += 1
    assert n == 340 + 310 + 1
