// Power-of-two scalings shared by the mixed-precision paths: equilibrate's
// radix scale (src/lapack/dense_utilities.jl:191-213) and the exponent scale
// of _mixed_extended_correction (src/lapack/extended_lapack.jl:114-131).
#pragma once
#include <cuda_runtime.h>

namespace oxi {

// 2^round(log2 v) clamped to Float64's exponent range (equilibrate's radix
// scale, ldexp(1, clamp(round(Int, log2(v)), ...))): the integer nearest the
// double log2 v rounds to, ties to even.  With v = f 2^e (f in [1/2, 1)),
// log2 v = (e - 1/2) + delta, delta = log2(f sqrt 2).  Away from the midpoint
// the sign of delta decides; within half a unit in the last place of e - 1/2
// the rounded log2 IS e - 1/2 and the tie goes to the even neighbour.  This is
// the result of a correctly rounded log2 followed by round-half-even, whatever
// the device log2's last bit would be.
__device__ __forceinline__ double radix_scale(double v) {
    int e;
    const double f = frexp(v, &e);
    const double s_hi = 1.4142135623730951, s_lo = -9.667293313452913e-17;  // sqrt 2 = s_hi + s_lo
    const double d = fma(f, s_hi, -1.0) + f * s_lo;                             // f sqrt 2 - 1
    const double delta = d * 1.4426950408889634;                               // / ln 2 (d is tiny at a tie)
    const double m = (double)e - 0.5;
    const double up = nextafter(m, INFINITY) - m, dn = m - nextafter(m, -INFINITY);
    int r;
    if (delta < 0.5 * up && -delta < 0.5 * dn) r = (int)rint(m);
    else r = delta > 0 ? e : e - 1;
    r = max(-1022, min(1023, r));
    return ldexp(1.0, r);
}

// power of two 2^exponent(m) (Julia's exponent: floor(log2 m)), 0 for m == 0
__device__ __forceinline__ double binary_scale(double m) {
    if (m == 0.0) return 0.0;
    int e;
    frexp(m, &e);
    return ldexp(1.0, e - 1);
}

}  // namespace oxi
