// Correctly rounded division by a divisor shared by many dividends.
//
// The candidate z-normalisation (t - mu) / sigma divides every point of a
// window by the same sigma.  With y = RN(1/b) computed once (a correctly
// rounded reciprocal), each quotient takes one multiply and four FMAs:
//   q0 = RN(a*y)                         within 2 ulp of a/b
//   r0 = RN(a - b*q0),  q1 = RN(q0 + r0*y)   within 1 ulp
//   r1 = a - b*q1 (exact, q1 being faithful), q2 = RN(q1 + r1*y) = RN(a/b)
// The last step is Markstein's theorem (P. Markstein, IBM J. Res. Develop.
// 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point Arithmetic,
// 2nd ed., 2018, section 4.7): with y within half an ulp of 1/b and q within
// one ulp of a/b, RN(q + (a - b q) y) equals RN(a/b).  The theorem needs every
// intermediate to stay a normal number; rcp_div_in_range() accepts divisors
// and quotient estimates in [2^-450, 2^450], where residuals are at least
// about 2^-952, and the callers divide directly outside it (zero dividends,
// extreme ranges, NaN).
//
// The header compiles as host C (for the CPU check of the method against
// IEEE division) and as CUDA device code.
#pragma once

#if defined(__CUDACC__)
#include <string.h>
#define FSM_RD_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#if defined(__cplusplus)
#define FSM_RD_HD inline
#else
#define FSM_RD_HD static inline
#endif
#endif

// round-to-nearest product and fused multiply-add, never contracted
FSM_RD_HD double rcp_div_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
FSM_RD_HD double rcp_div_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

// |x| in [2^-450, 2^450] (false for zero, subnormals, infinities and NaN),
// two floating-point comparisons
FSM_RD_HD int rcp_div_in_range(double x) {
    const double ax = fabs(x);
    return ax >= 0x1p-450 && ax <= 0x1p+450;
}

// The same test on the integer pipe, for kernels whose floating-point pipe
// is the busier one: |x| in [2^-450, 2^450) from the biased exponent field e,
// 1023 - 450 <= e < 1023 + 450 (implies rcp_div_in_range(x))
FSM_RD_HD int rcp_div_in_range_bits(double x) {
#if defined(__CUDA_ARCH__)
    const unsigned hi = (unsigned)__double2hiint(x);
#else
    unsigned long long u;
    memcpy(&u, &x, 8);
    const unsigned hi = (unsigned)(u >> 32);
#endif
    const unsigned e = (hi >> 20) & 0x7ffu;
    return e - 573u < 900u;
}

// RN(a / b) from y = RN(1 / b); the caller has checked rcp_div_in_range(b)
// and rcp_div_in_range(q0), q0 = rcp_div_estimate(a, y)
FSM_RD_HD double rcp_div_estimate(double a, double y) { return rcp_div_mul(a, y); }

FSM_RD_HD double rcp_div_finish(double a, double b, double y, double q0) {
    const double r0 = rcp_div_fma(-q0, b, a);
    const double q1 = rcp_div_fma(r0, y, q0);
    const double r1 = rcp_div_fma(-q1, b, a);
    return rcp_div_fma(r1, y, q1);
}
