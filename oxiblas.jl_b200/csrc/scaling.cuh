// Power-of-two scalings shared by the mixed-precision paths: equilibrate's
// radix scale (src/lapack/dense_utilities.jl:191-213) and the exponent scale
// of _mixed_extended_correction (src/lapack/extended_lapack.jl:114-131).
#pragma once
#include <cuda_runtime.h>

namespace oxi {

// 2^round(log2 v) clamped to Float64's exponent range (equilibrate's radix
// scale).  log2 v = e + log2 f with v = f 2^e, f in [0.5, 1): it rounds to e
// exactly when f >= 2^-1/2 (an irrational bound, so no ties arise).
__device__ __forceinline__ double radix_scale(double v) {
    int e;
    const double f = frexp(v, &e);
    int r = (f >= 0.70710678118654757) ? e : e - 1;
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
