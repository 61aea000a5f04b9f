// gft_math.cuh -- elementary functions for the throughput kernels.
//
// Written from the Taylor series of sin, cos and asin with a two/three-term
// Cody-Waite reduction by pi (W. J. Cody, W. Waite, "Software Manual for the
// Elementary Functions", 1980): r = x - k*pi with k = rint(x/pi), |r| <= pi/2,
// then sin(x) = (-1)^k sin(r), cos(x) = (-1)^k cos(r).  The series are
// truncated where the first omitted term is below the format's rounding:
//   float : sin to r^13, cos to r^14  (omitted term <= 7e-10 at |r| = pi/2)
//   double: sin to r^23, cos to r^24  (omitted term <= 1e-19)
// Arguments beyond |x| > 2^13 (float) / 2^20 (double) fall back to the CUDA
// library functions, whose reduction is exact for any argument.
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

__device__ __forceinline__ void sincos_poly(float r, float& s, float& c)
{
    const float r2 = r * r;
    float ps = (float)GFT_S13;
    ps = fmaf(ps, r2, (float)GFT_S11);
    ps = fmaf(ps, r2, (float)GFT_S9);
    ps = fmaf(ps, r2, (float)GFT_S7);
    ps = fmaf(ps, r2, (float)GFT_S5);
    ps = fmaf(ps, r2, (float)GFT_S3);
    s = fmaf(ps * r2, r, r);
    float pc = (float)GFT_C14;
    pc = fmaf(pc, r2, (float)GFT_C12);
    pc = fmaf(pc, r2, (float)GFT_C10);
    pc = fmaf(pc, r2, (float)GFT_C8);
    pc = fmaf(pc, r2, (float)GFT_C6);
    pc = fmaf(pc, r2, (float)GFT_C4);
    pc = fmaf(pc, r2, (float)GFT_C2);
    c = fmaf(pc, r2, 1.0f);
}

__device__ __forceinline__ float sin_poly(float r)
{
    const float r2 = r * r;
    float ps = (float)GFT_S13;
    ps = fmaf(ps, r2, (float)GFT_S11);
    ps = fmaf(ps, r2, (float)GFT_S9);
    ps = fmaf(ps, r2, (float)GFT_S7);
    ps = fmaf(ps, r2, (float)GFT_S5);
    ps = fmaf(ps, r2, (float)GFT_S3);
    return fmaf(ps * r2, r, r);
}

// pi = PI_A + PI_B: PI_A = float(pi), PI_B = float(pi - PI_A)
__device__ __forceinline__ float reduce_pi(float x, int& k)
{
    const float kf = rintf(x * 0.3183098861837907f);
    k = (int)kf;
    const float r = fmaf(-kf, 3.1415927410125732f, x);
    return fmaf(-kf, -8.742277657347586e-08f, r);
}

__device__ __forceinline__ float gsin(float x)
{
    if (fabsf(x) > 8192.0f) return sinf(x);
    int k;
    const float r = reduce_pi(x, k);
    const float s = sin_poly(r);
    return (k & 1) ? -s : s;
}

__device__ __forceinline__ void gsincos(float x, float& s, float& c)
{
    if (fabsf(x) > 8192.0f) {
        sincosf(x, &s, &c);
        return;
    }
    int k;
    const float r = reduce_pi(x, k);
    sincos_poly(r, s, c);
    if (k & 1) {
        s = -s;
        c = -c;
    }
}

__device__ __forceinline__ float gasin(float x)
{
    if (fabsf(x) > 0.25f) return asinf(x);
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

// pi = PI_A + PI_B + PI_C (each the double nearest to the remainder); with
// FMA each step rounds once, so r carries a relative error of ~1 ulp.
__device__ __forceinline__ double reduce_pi(double x, int& k)
{
    const double kd = rint(x * 0.3183098861837907);
    k = (int)kd;
    double r = fma(-kd, 3.141592653589793, x);
    r = fma(-kd, 1.2246467991473532e-16, r);
    return fma(-kd, -2.9947698097183397e-33, r);
}

__device__ __forceinline__ double gsin(double x)
{
    if (fabs(x) > 1048576.0) return sin(x);
    int k;
    const double r = reduce_pi(x, k);
    const double s = sin_poly(r);
    return (k & 1) ? -s : s;
}

__device__ __forceinline__ void gsincos(double x, double& s, double& c)
{
    if (fabs(x) > 1048576.0) {
        sincos(x, &s, &c);
        return;
    }
    int k;
    const double r = reduce_pi(x, k);
    sincos_poly(r, s, c);
    if (k & 1) {
        s = -s;
        c = -c;
    }
}

__device__ __forceinline__ double gasin(double x)
{
    if (fabs(x) > 0.125) return asin(x);
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

}  // namespace gft
