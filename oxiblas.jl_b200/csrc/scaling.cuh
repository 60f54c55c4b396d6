// Power-of-two scalings shared by the mixed-precision paths: equilibrate's
// radix scale (src/lapack/dense_utilities.jl:191-213) and the exponent scale
// of _mixed_extended_correction (src/lapack/extended_lapack.jl:114-131).
#pragma once
#include <cuda_runtime.h>

namespace oxi {

// 2^round(log2 v) clamped to Float64's exponent range (equilibrate's radix
// scale): log2 rounded to the nearest integer, ties to even (Julia's round),
// the same formula as the reference's ldexp(1, clamp(round(Int, log2(v)), ...)).
__device__ __forceinline__ double radix_scale(double v) {
    double e = rint(log2(v));
    e = fmin(1023.0, fmax(-1022.0, e));
    return ldexp(1.0, (int)e);
}

// power of two 2^exponent(m) (Julia's exponent: floor(log2 m)), 0 for m == 0
__device__ __forceinline__ double binary_scale(double m) {
    if (m == 0.0) return 0.0;
    int e;
    frexp(m, &e);
    return ldexp(1.0, e - 1);
}

}  // namespace oxi
