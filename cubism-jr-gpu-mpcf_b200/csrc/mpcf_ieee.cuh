// mpcf_ieee.cuh -- correctly rounded (IEEE round-to-nearest-even) reciprocals
// for the reference-rounding stage kernel, without branches.
//
// Method: Newton-Raphson iteration for 1/x from the special-function unit's
// approximate double-precision reciprocal, y <- y + y (1 - x y) with fused
// multiply-adds (each step doubles the correct bits), as in Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34 (1990), and Cornea-Hasegan, Golliver and
// Markstein, "Correctness proofs outline for Newton-Raphson based
// floating-point divide and square root algorithms", ARITH 14 (1999).
// Zero, infinite and NaN inputs take the approximate reciprocal itself,
// which is exact for them (+-inf, +-0, NaN).
//
// rcp_rn_f64_weight(x): 1/x rounded to double, for the WENO weights'
//   denominators x = 10 (beta + eps)^2 of the FP32 reference form (beta
//   float, so x is exact in double and normal, or zero, or infinite).  Two
//   Newton steps give about 1 ulp, a third step the correctly rounded value.
// rcp_rn_f32(x): 1/x rounded to float, for any float x.  x is exact in
//   double; two Newton steps give 1/x to about 2^-52 relative, and 1/x lies
//   at least 2^-49 (relative) from every midpoint of two floats (x has 24
//   significant bits and a midpoint 25, so 1 - m x is a nonzero multiple of
//   2^-48 near 1), so one rounding to float is the correctly rounded value,
//   subnormal results and overflow to infinity included.
//
// Both are checked against the compiler's IEEE division over every float
// input (tests/test_gpu_ieee.py through mpcf_selftest_ieee).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

namespace mpcf {

__device__ __forceinline__ double rcp_seed_f64(const double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

__device__ __forceinline__ double rcp_rn_f64_weight(const double x)
{
    const double y0 = rcp_seed_f64(x);
    double e = __fma_rn(-x, y0, 1.0);
    double y = __fma_rn(y0, e, y0);
    e = __fma_rn(-x, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-x, y, 1.0);
    y = __fma_rn(y, e, y);
    return (x != 0.0 && fabs(x) < CUDART_INF) ? y : y0;
}

__device__ __forceinline__ float rcp_rn_f32(const float x)
{
    const double X = (double)x;
    const double y0 = rcp_seed_f64(X);
    double e = __fma_rn(-X, y0, 1.0);
    double y = __fma_rn(y0, e, y0);
    e = __fma_rn(-X, y, 1.0);
    y = __fma_rn(y, e, y);
    return __double2float_rn((X != 0.0 && fabs(X) < CUDART_INF) ? y : y0);
}

} // namespace mpcf
