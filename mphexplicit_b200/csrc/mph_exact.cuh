// mph_exact.cuh — correctly rounded FP64 arithmetic helpers for the
// bit-exact FP64 form.
#pragma once

namespace mph {

// Round-to-nearest quotient x/y from yi = RN(1/y), by Markstein's method
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990; see also Muller et
// al., Handbook of Floating-Point Arithmetic, the FMA-based division
// chapter): start from q0 = RN(x*yi), then twice form the exact remainder
// r = x - q*y with one FMA and correct q += r*yi.  The first correction
// brings q within half an ulp plus a tiny term, the second (Markstein's
// step) yields RN(x/y).  Valid for finite, normal operands without overflow
// or underflow of the intermediates, which is the range the pair kernels use
// (lengths between ~1e-9 and ~1e3 m, forces far from the double limits); a
// zero numerator returns x*yi, i.e. a zero with the IEEE sign.  The FP64
// kernels call this where the reference divides, and
// mph_check_exact_division() compares it bit for bit with the hardware
// IEEE division on random and adversarial operands.
__device__ __forceinline__ double div_rn(double x, double y, double yi) {
    double q = x * yi;
    double r = __fma_rn(-q, y, x);
    q = __fma_rn(r, yi, q);
    r = __fma_rn(-q, y, x);
    q = __fma_rn(r, yi, q);
    return x == 0.0 ? x * yi : q;
}

// div_rn without the zero-numerator branch, for the pair sweeps.  For x = +-0
// the two corrections give +0 where x/y is -0 (x*yi gives the IEEE sign);
// every quotient taken this way in the sweeps reaches the particle's state
// only through products and sums that start at +0.0 (a DensityA / DensityP /
// DivergenceP / GravityCenter / force accumulator), and such a sum never
// holds -0.0 (+0 + -0 = +0, and an exact cancellation rounds to +0), so
// adding a zero of either sign leaves it unchanged: the results are
// bit-identical to those of div_rn (and of the reference's `/`).
__device__ __forceinline__ double div_rs(double x, double y, double yi) {
    double q = x * yi;
    double r = __fma_rn(-q, y, x);
    q = __fma_rn(r, yi, q);
    r = __fma_rn(-q, y, x);
    return __fma_rn(r, yi, q);
}

}  // namespace mph
