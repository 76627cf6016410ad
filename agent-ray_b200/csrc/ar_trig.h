// ar_trig.h: sin and cos of a sampling angle, bit-identical on the host (the
// CPU oracle) and on the device (the kernels).
//
// The integrators turn a uniform number u in [0, 1) into an angle
// phi = 2*pi*u and take its sine and cosine (cosine-weighted hemisphere,
// GGX half-vector, uniform sphere).  The CUDA and host math libraries each
// round sinf/cosf within their own error bounds, so a one-ulp difference in a
// direction could send a path through glass onto a different surface.  This
// routine uses only IEEE-754 single-precision multiplies and adds, each
// rounded on its own (the device path spells them with the _rn intrinsics, so
// it does not depend on the translation unit's -fmad setting; host code must be
// built with -ffp-contract=off), so both sides get the same bits.
//
// Method:
//   * Cody-Waite range reduction (W. J. Cody and W. Waite, "Software Manual for
//     the Elementary Functions", 1980): k = rint(x * 2/pi) and
//     r = x - k*P1 - k*P2 - k*P3 with pi/2 = P1 + P2 + P3, where P1 (8
//     significant bits) and P2 (12 bits) are short enough that k*P1 and k*P2
//     are exact for |k| < 2^11, and P3 is the float nearest the remainder;
//   * sin(r) and cos(r) on |r| <= pi/4 from their Taylor series through r^11
//     and r^12 (truncation error below 1e-11, far under the float rounding),
//     evaluated by Horner's rule in r^2 with the coefficients 1/n! rounded to
//     float;
//   * the quadrant k mod 4 selects and signs the pair.
// Accuracy (tests/test_cpu_oracle.py, against float64 sin/cos over [0, 2*pi]):
// absolute error below 1.5e-7 (measured: 9.4e-8).
// Domain: finite |x| < 2^11 * pi/2 (the callers pass [0, 2*pi]).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define AR_TRIG_FN __host__ __device__ __forceinline__
#else
#define AR_TRIG_FN inline
#endif

namespace ar_trig {

AR_TRIG_FN float mul(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
AR_TRIG_FN float add(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
AR_TRIG_FN float sub(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}

// s = sin(x), c = cos(x).
AR_TRIG_FN void sincos(float x, float* s, float* c) {
    const float two_over_pi = 0.636619747f;
    const float p1 = 1.5703125f;              // 201 / 128
    const float p2 = 4.83751297e-04f;         // 2029 / 2^22
    const float p3 = 7.54979013e-08f;         // pi/2 - p1 - p2, rounded
    const float k = rintf(mul(x, two_over_pi));
    float r = sub(x, mul(k, p1));
    r = sub(r, mul(k, p2));
    r = sub(r, mul(k, p3));
    const float r2 = mul(r, r);
    // sin(r) = r + r^3 (-1/3! + r^2 (1/5! + r^2 (-1/7! + r^2 (1/9! - r^2/11!))))
    float ps = add(2.75573188e-06f, mul(r2, -2.50521079e-08f));
    ps = add(-1.98412701e-04f, mul(r2, ps));
    ps = add(8.33333377e-03f, mul(r2, ps));
    ps = add(-1.66666672e-01f, mul(r2, ps));
    const float sr = add(r, mul(mul(r, r2), ps));
    // cos(r) = 1 - r^2/2 + r^4 (1/4! + r^2 (-1/6! + r^2 (1/8! + r^2 (-1/10! + r^2/12!))))
    float pc = add(-2.75573200e-07f, mul(r2, 2.08767559e-09f));
    pc = add(2.48015876e-05f, mul(r2, pc));
    pc = add(-1.38888892e-03f, mul(r2, pc));
    pc = add(4.16666679e-02f, mul(r2, pc));
    const float cr = add(sub(1.0f, mul(0.5f, r2)), mul(mul(r2, r2), pc));
    const int q = int(k) & 3;
    const float sv = (q & 1) ? cr : sr;
    const float cv = (q & 1) ? sr : cr;
    *s = (q & 2) ? -sv : sv;
    *c = ((q + 1) & 2) ? -cv : cv;
}

}  // namespace ar_trig
