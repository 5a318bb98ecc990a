// phase.cuh -- sin and cos of one argument for the Green kernels.
//
// Cody-Waite reduction modulo pi/2 with a three-part split of pi/2 (each part
// short enough that n * part is exact for the arguments these kernels see,
// |x| < 2^20 in FP64, |x| < 2^12 in FP32), then the Taylor series of sin and
// cos on [-pi/4, pi/4] (coefficients 1/n!), truncated where the next term is
// far below half an ulp: x^17/17! and x^18/18! in FP64, x^9/9! and x^10/10! in
// FP32.  The split parts were computed from the decimal expansion of pi with
// exact rational arithmetic.  The quadrant n mod 4 rotates (sin, cos).
//
// Host and device share this code so the CPU test suite can check it against
// the C library (tests/test_phase.py).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define BB_HD __host__ __device__ __forceinline__
#else
#define BB_HD inline
#endif

namespace bb {

BB_HD void sincos_cw(double x, double *s, double *c) {
    const double n = rint(x * 0.6366197723675814);  // x * 2/pi
    double r = fma(-n, 1.5707963267341256, x);      // pi/2, leading 33 bits
    r = fma(-n, 6.077100506303966e-11, r);          // next 33 bits
    r = fma(-n, 2.0222662487959506e-21, r);         // remainder
    const double r2 = r * r;
    double ps = 1.0 / 355687428096000.0;            // 1/17!
    ps = fma(ps, r2, -1.0 / 1307674368000.0);       // 1/15!
    ps = fma(ps, r2, 1.0 / 6227020800.0);           // 1/13!
    ps = fma(ps, r2, -1.0 / 39916800.0);            // 1/11!
    ps = fma(ps, r2, 1.0 / 362880.0);               // 1/9!
    ps = fma(ps, r2, -1.0 / 5040.0);                // 1/7!
    ps = fma(ps, r2, 1.0 / 120.0);                  // 1/5!
    ps = fma(ps, r2, -1.0 / 6.0);                   // 1/3!
    const double sr = fma(ps * r2, r, r);
    double pc = 1.0 / 6402373705728000.0;           // 1/18!
    pc = fma(pc, r2, -1.0 / 20922789888000.0);      // 1/16!
    pc = fma(pc, r2, 1.0 / 87178291200.0);          // 1/14!
    pc = fma(pc, r2, -1.0 / 479001600.0);           // 1/12!
    pc = fma(pc, r2, 1.0 / 3628800.0);              // 1/10!
    pc = fma(pc, r2, -1.0 / 40320.0);               // 1/8!
    pc = fma(pc, r2, 1.0 / 720.0);                  // 1/6!
    pc = fma(pc, r2, -1.0 / 24.0);                  // 1/4!
    pc = fma(pc, r2, 0.5);                          // 1/2!
    const double cr = fma(-pc, r2, 1.0);
    const int q = (int)(long long)n & 3;
    const double ss = (q & 1) ? cr : sr, cc = (q & 1) ? sr : cr;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

BB_HD void sincos_cw(float x, float *s, float *c) {
    const float n = rintf(x * 0.636619746685f);      // x * 2/pi
    float r = fmaf(-n, 1.5703125f, x);               // pi/2, leading 12 bits
    r = fmaf(-n, 4.837512969970703e-4f, r);          // next 12 bits
    r = fmaf(-n, 7.549790126404332e-8f, r);          // remainder
    const float r2 = r * r;
    float ps = 1.0f / 362880.0f;                     // 1/9!
    ps = fmaf(ps, r2, -1.0f / 5040.0f);              // 1/7!
    ps = fmaf(ps, r2, 1.0f / 120.0f);                // 1/5!
    ps = fmaf(ps, r2, -1.0f / 6.0f);                 // 1/3!
    const float sr = fmaf(ps * r2, r, r);
    float pc = 1.0f / 3628800.0f;                    // 1/10!
    pc = fmaf(pc, r2, -1.0f / 40320.0f);             // 1/8!
    pc = fmaf(pc, r2, 1.0f / 720.0f);                // 1/6!
    pc = fmaf(pc, r2, -1.0f / 24.0f);                // 1/4!
    pc = fmaf(pc, r2, 0.5f);                         // 1/2!
    const float cr = fmaf(-pc, r2, 1.0f);
    const int q = (int)n & 3;
    const float ss = (q & 1) ? cr : sr, cc = (q & 1) ? sr : cr;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

}  // namespace bb
