"""Generates mph_pow10.h: 10^s for s in [POW10_MIN, POW10_MAX] as double-double
pairs {hi, lo}, hi = RN(v), lo = RN(v - hi), with v = 10^s * 2^-scale(s) and
scale(s) = 256 for s > 250, -256 for s < -250, 0 otherwise (so that neither
part leaves the normal range).  The device "%e" formatter (k_text.cu) scales
its argument by 2^scale(s) before the multiplication.  Exact rational
arithmetic; run `python gen_pow10.py > mph_pow10.h` to regenerate."""
from fractions import Fraction

POW10_MIN, POW10_MAX = -310, 340


def scale(s):
    return 256 if s > 250 else (-256 if s < -250 else 0)


def entry(s):
    v = Fraction(10) ** s * Fraction(2) ** (-scale(s))
    hi = float(v)  # float(Fraction) rounds to nearest, ties to even
    lo = float(v - Fraction(hi))
    return hi, lo


def main():
    print("// generated by gen_pow10.py: 10^s * 2^-scale(s) as {hi, lo} double pairs,")
    print("// scale(s) = 256 for s > 250, -256 for s < -250, else 0")
    print("#pragma once")
    print("#define MPH_POW10_MIN (%d)" % POW10_MIN)
    print("#define MPH_POW10_MAX (%d)" % POW10_MAX)
    print("static __device__ const double2 kMphPow10[%d] = {" % (POW10_MAX - POW10_MIN + 1))
    for s in range(POW10_MIN, POW10_MAX + 1):
        hi, lo = entry(s)
        print("    {%s, %s},  // %d" % (hi.hex(), lo.hex(), s))
    print("};")


if __name__ == "__main__":
    main()
