// gft_math.cuh -- elementary functions for the throughput kernels.
//
// Written with a two/three-term Cody-Waite reduction by pi (W. J. Cody,
// W. Waite, "Software Manual for the Elementary Functions", 1980):
// r = x - k*pi with k = rint(x/pi), |r| <= pi/2, then sin(x) = (-1)^k sin(r),
// cos(x) = (-1)^k cos(r).  On the reduced range:
//   float : minimax polynomials fitted for this library by the Remez exchange
//           (gft_math_fit.py regenerates them): sin r = r + r^3 P(r^2), degree 9,
//           relative error <= 6.1e-9; cos r = 1 + r^2 Q(r^2), degree 10, absolute
//           error <= 2.5e-10 -- both below float's rounding, and two multiply-adds
//           shorter each than the Taylor series of equal accuracy (degree 13 / 14);
//   double: Taylor series, sin to r^23, cos to r^24 (omitted term <= 1e-19).
// The reduction uses the 1.5*2^p rounding constant (no conversion to integer):
// it holds for |x| < 1.3e7 (float) / 1.4e15 (double); phases that large do not
// occur in the evolution (the step kernels flag |theta| > 1e4).
// asin: odd series x + x^3/6 + 3x^5/40 + ... for |x| <= 1/4 (float) or 1/8
// (double) -- the link update's argument is dt * E ~ 1e-3 -- and CUDA's asin
// otherwise.
#pragma once

#include <cuda_runtime.h>

namespace gft {

// Taylor coefficients (-1)^n / (2n+1)!  and  (-1)^n / (2n)!
#define GFT_S3 (-1.0 / 6.0)
#define GFT_S5 (1.0 / 120.0)
#define GFT_S7 (-1.0 / 5040.0)
#define GFT_S9 (1.0 / 362880.0)
#define GFT_S11 (-1.0 / 39916800.0)
#define GFT_S13 (1.0 / 6227020800.0)
#define GFT_S15 (-1.0 / 1307674368000.0)
#define GFT_S17 (1.0 / 355687428096000.0)
#define GFT_S19 (-1.0 / 121645100408832000.0)
#define GFT_S21 (1.0 / 51090942171709440000.0)
#define GFT_S23 (-1.0 / 25852016738884976640000.0)
#define GFT_C2 (-1.0 / 2.0)
#define GFT_C4 (1.0 / 24.0)
#define GFT_C6 (-1.0 / 720.0)
#define GFT_C8 (1.0 / 40320.0)
#define GFT_C10 (-1.0 / 3628800.0)
#define GFT_C12 (1.0 / 479001600.0)
#define GFT_C14 (-1.0 / 87178291200.0)
#define GFT_C16 (1.0 / 20922789888000.0)
#define GFT_C18 (-1.0 / 6402373705728000.0)
#define GFT_C20 (1.0 / 2432902008176640000.0)
#define GFT_C22 (-1.0 / 1124000727777607680000.0)
#define GFT_C24 (1.0 / 620448401733239439360000.0)

// Float minimax coefficients on |r| <= pi/2 (gft_math_fit.py): sin r = r + r^3 P(r^2), cos r = 1 + r^2 Q(r^2).
#define GFT_FS3 (-0.16666659712791443f)
#define GFT_FS5 (0.00833306647837162f)
#define GFT_FS7 (-0.00019809602235909551f)
#define GFT_FS9 (2.605780537123792e-06f)
#define GFT_FC2 (-0.5f)
#define GFT_FC4 (0.04166664183139801f)
#define GFT_FC6 (-0.00138884037733078f)
#define GFT_FC8 (2.4761886379565112e-05f)
#define GFT_FC10 (-2.607710598567792e-07f)

__device__ __forceinline__ void sincos_poly(float r, float& s, float& c)
{
    const float r2 = r * r;
    float ps = GFT_FS9;
    ps = fmaf(ps, r2, GFT_FS7);
    ps = fmaf(ps, r2, GFT_FS5);
    ps = fmaf(ps, r2, GFT_FS3);
    s = fmaf(ps * r2, r, r);
    float pc = GFT_FC10;
    pc = fmaf(pc, r2, GFT_FC8);
    pc = fmaf(pc, r2, GFT_FC6);
    pc = fmaf(pc, r2, GFT_FC4);
    pc = fmaf(pc, r2, GFT_FC2);
    c = fmaf(pc, r2, 1.0f);
}

__device__ __forceinline__ float sin_poly(float r)
{
    const float r2 = r * r;
    float ps = GFT_FS9;
    ps = fmaf(ps, r2, GFT_FS7);
    ps = fmaf(ps, r2, GFT_FS5);
    ps = fmaf(ps, r2, GFT_FS3);
    return fmaf(ps * r2, r, r);
}

// x = k*pi + r: t = x/pi + 1.5*2^23 rounds x/pi to the integer k held in the
// low mantissa bits of t (valid while |x/pi| < 2^22, i.e. |x| < 1.3e7; the
// step kernels flag phases beyond 1e4 with GFT_W_RANGE); then
// r = x - k*PI_A - k*PI_B with PI_A = float(pi), PI_B = float(pi - PI_A).
// Returns r and the sign bit (-1)^k as an integer mask.
__device__ __forceinline__ float reduce_pi(float x, unsigned& sign)
{
    const float t = fmaf(x, 0.3183098861837907f, 12582912.0f);
    const float kf = t - 12582912.0f;
    sign = __float_as_uint(t) << 31;
    const float r = fmaf(-kf, 3.1415927410125732f, x);
    return fmaf(-kf, -8.742277657347586e-08f, r);
}

__device__ __forceinline__ float gsin(float x)
{
    unsigned sg;
    const float r = reduce_pi(x, sg);
    return __uint_as_float(__float_as_uint(sin_poly(r)) ^ sg);
}

__device__ __forceinline__ void gsincos(float x, float& s, float& c)
{
    unsigned sg;
    const float r = reduce_pi(x, sg);
    sincos_poly(r, s, c);
    s = __uint_as_float(__float_as_uint(s) ^ sg);
    c = __uint_as_float(__float_as_uint(c) ^ sg);
}

// Out-of-line wide-argument paths: taken only when |x| > 1/4 (asin) or c >= 1/64
// (sqrt), which the link update's small increments never reach; keeping them out
// of the inlined step body shortens the hot loop's code (measured 1-1.5 % faster).
static __device__ __noinline__ float gasin_wide(float x) { return asinf(x); }
static __device__ __noinline__ double gasin_wide(double x) { return asin(x); }
static __device__ __noinline__ float sqrt1m_wide(float c) { return -c / (1.0f + sqrtf(1.0f - c)); }
static __device__ __noinline__ double sqrt1m_wide(double c) { return -c / (1.0 + sqrt(1.0 - c)); }

__device__ __forceinline__ float gasin(float x)
{
    if (fabsf(x) > 0.25f) return gasin_wide(x);
    // asin x = sum_n C(2n,n) / (4^n (2n+1)) x^(2n+1); through n = 6 the first
    // omitted term is < 1e-9 relative at |x| = 1/4
    const float x2 = x * x;
    float p = 924.0f / 53248.0f;           // n = 6
    p = fmaf(p, x2, 252.0f / 11264.0f);    // n = 5
    p = fmaf(p, x2, 70.0f / 2304.0f);      // n = 4
    p = fmaf(p, x2, 20.0f / 448.0f);       // n = 3
    p = fmaf(p, x2, 6.0f / 80.0f);         // n = 2
    p = fmaf(p, x2, 2.0f / 12.0f);         // n = 1
    return fmaf(p * x2, x, x);
}

// ---- double ----------------------------------------------------------------
__device__ __forceinline__ void sincos_poly(double r, double& s, double& c)
{
    const double r2 = r * r;
    double ps = GFT_S23;
    ps = fma(ps, r2, GFT_S21);
    ps = fma(ps, r2, GFT_S19);
    ps = fma(ps, r2, GFT_S17);
    ps = fma(ps, r2, GFT_S15);
    ps = fma(ps, r2, GFT_S13);
    ps = fma(ps, r2, GFT_S11);
    ps = fma(ps, r2, GFT_S9);
    ps = fma(ps, r2, GFT_S7);
    ps = fma(ps, r2, GFT_S5);
    ps = fma(ps, r2, GFT_S3);
    s = fma(ps * r2, r, r);
    double pc = GFT_C24;
    pc = fma(pc, r2, GFT_C22);
    pc = fma(pc, r2, GFT_C20);
    pc = fma(pc, r2, GFT_C18);
    pc = fma(pc, r2, GFT_C16);
    pc = fma(pc, r2, GFT_C14);
    pc = fma(pc, r2, GFT_C12);
    pc = fma(pc, r2, GFT_C10);
    pc = fma(pc, r2, GFT_C8);
    pc = fma(pc, r2, GFT_C6);
    pc = fma(pc, r2, GFT_C4);
    pc = fma(pc, r2, GFT_C2);
    c = fma(pc, r2, 1.0);
}

__device__ __forceinline__ double sin_poly(double r)
{
    const double r2 = r * r;
    double ps = GFT_S23;
    ps = fma(ps, r2, GFT_S21);
    ps = fma(ps, r2, GFT_S19);
    ps = fma(ps, r2, GFT_S17);
    ps = fma(ps, r2, GFT_S15);
    ps = fma(ps, r2, GFT_S13);
    ps = fma(ps, r2, GFT_S11);
    ps = fma(ps, r2, GFT_S9);
    ps = fma(ps, r2, GFT_S7);
    ps = fma(ps, r2, GFT_S5);
    ps = fma(ps, r2, GFT_S3);
    return fma(ps * r2, r, r);
}

// As for float, with t = x/pi + 1.5*2^52 (valid while |x| < 1.4e15) and
// pi = PI_A + PI_B + PI_C, each the double nearest to the remainder; with FMA
// each step rounds once, so r carries a relative error of ~1 ulp.
__device__ __forceinline__ double reduce_pi(double x, unsigned long long& sign)
{
    const double t = fma(x, 0.3183098861837907, 6755399441055744.0);
    const double kd = t - 6755399441055744.0;
    sign = (unsigned long long)__double_as_longlong(t) << 63;
    double r = fma(-kd, 3.141592653589793, x);
    r = fma(-kd, 1.2246467991473532e-16, r);
    return fma(-kd, -2.9947698097183397e-33, r);
}

__device__ __forceinline__ double gsin(double x)
{
    unsigned long long sg;
    const double r = reduce_pi(x, sg);
    return __longlong_as_double(__double_as_longlong(sin_poly(r)) ^ (long long)sg);
}

__device__ __forceinline__ void gsincos(double x, double& s, double& c)
{
    unsigned long long sg;
    const double r = reduce_pi(x, sg);
    sincos_poly(r, s, c);
    s = __longlong_as_double(__double_as_longlong(s) ^ (long long)sg);
    c = __longlong_as_double(__double_as_longlong(c) ^ (long long)sg);
}

__device__ __forceinline__ double gasin(double x)
{
    if (fabs(x) > 0.125) return gasin_wide(x);
    // through n = 9 the first omitted term is < 1e-20 relative at |x| = 1/8
    const double x2 = x * x;
    double p = 48620.0 / 4980736.0;            // n = 9
    p = fma(p, x2, 12870.0 / 1114112.0);        // n = 8
    p = fma(p, x2, 3432.0 / 245760.0);          // n = 7
    p = fma(p, x2, 924.0 / 53248.0);            // n = 6
    p = fma(p, x2, 252.0 / 11264.0);            // n = 5
    p = fma(p, x2, 70.0 / 2304.0);              // n = 4
    p = fma(p, x2, 20.0 / 448.0);               // n = 3
    p = fma(p, x2, 6.0 / 80.0);                 // n = 2
    p = fma(p, x2, 2.0 / 12.0);                 // n = 1
    return fma(p * x2, x, x);
}

// sqrt(1 - c) - 1 for the link update's |c|^2 = c (tiny in practice):
// -c/2 - c^2/8 - c^3/16 - 5c^4/128 when c < 1/64 (float: the first omitted
// term is 7c^4/128 < 4e-9 relative) or c < 1/8192 (double: < 2e-17), else the
// exact -c / (1 + sqrt(1 - c)).
__device__ __forceinline__ float sqrt1m_minus1(float c)
{
    if (c < 0.015625f) return c * fmaf(c, fmaf(c, fmaf(c, -5.0f / 128.0f, -1.0f / 16.0f), -1.0f / 8.0f), -0.5f);
    return sqrt1m_wide(c);
}

__device__ __forceinline__ double sqrt1m_minus1(double c)
{
    if (c < 0.0001220703125) return c * fma(c, fma(c, fma(c, -5.0 / 128.0, -1.0 / 16.0), -1.0 / 8.0), -0.5);
    return sqrt1m_wide(c);
}

// 1/sqrt(s) and 1/d for arguments of order one: the hardware approximations
// (rsqrt.approx, rcp.approx; relative error below 2^-22) refined by one
// Newton-Raphson step each, r <- r (3 - s r^2) / 2 and q <- q (2 - d q), which
// squares that error; the results are within about one ulp of the rounded
// quotients.
__device__ __forceinline__ float rsqrt_nr(float s)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(s));
    return r * fmaf(-0.5f * s * r, r, 1.5f);
}
__device__ __forceinline__ float rcp_nr(float d)
{
    float q;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(q) : "f"(d));
    return q * fmaf(-d, q, 2.0f);
}

// 1 - a0/|a| of a quaternion with scalar part w and |vector part|^2 = v2,
// without cancellation: v2 / (|a| (|a| + w)) = v2 r^2 / (1 + w r) when w >= 0
// (r = 1/|a|), else 1 - w r.  Float form of the energy terms' plaquette and
// electric traces; a few ulp of the same expression evaluated with IEEE
// square root and division (checked by gft_selftest_math).
__device__ __forceinline__ float one_minus_cos_nr(float w, float v2)
{
    const float r = rsqrt_nr(fmaf(w, w, v2));
    const float c = w * r;
    return (w >= 0.0f) ? v2 * r * r * rcp_nr(1.0f + c) : 1.0f - c;
}

}  // namespace gft
