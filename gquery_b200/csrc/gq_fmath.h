// Fixed floating-point semantics for the query arithmetic.
//
// gQuery's traversal is DrJit code; its array library decides how dot products,
// norms, interpolation and the inverse trigonometric functions round.  DrJit is
// not available to pin those choices, so this header fixes them once, for the
// CUDA kernels and for the CPU restatement alike, using only correctly rounded
// IEEE-754 operations (+, -, *, /, sqrt, fma).  The same inputs therefore give
// the same bits on the host and on the GPU.  Rules:
//   * arithmetic written with Python operators in the reference is plain
//     IEEE arithmetic, never contracted into an FMA (build with --fmad=false
//     under nvcc and -ffp-contract=off under g++);
//   * array-library calls use fused forms:
//       dot(a,b)        = fma(a_n, b_n, ... fma(a_1, b_1, a_0*b_0))
//       norm(v)         = sqrt(dot(v,v))
//       normalize(v)    = v * (1 / sqrt(dot(v,v)))
//       lerp(a,b,t)     = fma(b, t, fma(-a, t, a))
//       cross(a,b)_i    = fma(a_j, b_k, -(a_k * b_j))
//       clamp(x,lo,hi)  = fmax(fmin(x, hi), lo)    (NaN-suppressing min/max)
//       epsilon         = 2^-24
//   * acos / asin / atan2 are evaluated with the single-precision polynomial
//     method of the Cephes library (S. L. Moshier, "Methods and Programs for
//     Mathematical Functions", 1989): range reduction by the half-angle identity
//     for |x| > 1/2 (asin/acos) and by tan(pi/4) / tan(pi/2) shifts (atan), then an
//     odd polynomial in the reduced argument.  Horner steps use fma.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GQ_HD __host__ __device__ __forceinline__
#else
#define GQ_HD static inline
#endif

#define GQ_EPS_F 5.9604644775390625e-08f  /* 2^-24 */
#define GQ_PI_F 3.14159265358979323846f
#define GQ_PIO2_F 1.57079632679489661923f
#define GQ_PIO4_F 0.785398163397448309616f
#define GQ_INF_F (__builtin_inff())

GQ_HD float gq_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}
GQ_HD float gq_min(float a, float b) { return fminf(a, b); }
GQ_HD float gq_max(float a, float b) { return fmaxf(a, b); }
GQ_HD float gq_sqrt(float a) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(a);
#else
    return sqrtf(a);
#endif
}
GQ_HD float gq_div(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
// max(min(x, hi), lo): a NaN x gives hi (fminf returns the other operand).  On the
// device a [0, 1] clamp may be folded into a saturate, which maps NaN to 0, so the NaN
// case is spelled out there (t of a zero-length segment is 0/0).
GQ_HD float gq_clamp(float x, float lo, float hi) {
#if defined(__CUDA_ARCH__)
    return x != x ? hi : gq_max(gq_min(x, hi), lo);
#else
    return gq_max(gq_min(x, hi), lo);
#endif
}

GQ_HD float gq_dot2(float ax, float ay, float bx, float by) { return gq_fma(ay, by, ax * bx); }
GQ_HD float gq_dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return gq_fma(az, bz, gq_fma(ay, by, ax * bx));
}
GQ_HD float gq_norm2(float x, float y) { return gq_sqrt(gq_dot2(x, y, x, y)); }
GQ_HD float gq_norm3(float x, float y, float z) { return gq_sqrt(gq_dot3(x, y, z, x, y, z)); }
GQ_HD float gq_lerp(float a, float b, float t) { return gq_fma(b, t, gq_fma(-a, t, a)); }
GQ_HD float gq_rsqrt(float x) { return gq_div(1.0f, gq_sqrt(x)); }

// ---- inverse trigonometric functions (Cephes single-precision method) ----

// asin on [0, 1/2]:  x + x^3 P(x^2)
GQ_HD float gq_asin_kernel(float x, float z) {
    float p = 4.2163199048e-2f;
    p = gq_fma(p, z, 2.4181311049e-2f);
    p = gq_fma(p, z, 4.5470025998e-2f);
    p = gq_fma(p, z, 7.4953002686e-2f);
    p = gq_fma(p, z, 1.6666752422e-1f);
    return gq_fma(p * z, x, x);
}

GQ_HD float gq_asin(float x) {
    float a = fabsf(x);
    float r;
    if (!(a <= 1.0f)) {
        r = (a > 1.0f) ? __builtin_nanf("") : a;  // NaN in -> NaN out
        return r;
    }
    if (a > 0.5f) {
        float z = 0.5f * (1.0f - a);
        float s = gq_sqrt(z);
        r = GQ_PIO2_F - 2.0f * gq_asin_kernel(s, z);
    } else {
        r = gq_asin_kernel(a, a * a);
    }
    return x < 0.0f ? -r : r;
}

GQ_HD float gq_acos(float x) {
    if (!(fabsf(x) <= 1.0f)) return __builtin_nanf("");
    if (x < -0.5f) {
        float z = 0.5f * (1.0f + x);
        return GQ_PI_F - 2.0f * gq_asin_kernel(gq_sqrt(z), z);
    }
    if (x > 0.5f) {
        float z = 0.5f * (1.0f - x);
        return 2.0f * gq_asin_kernel(gq_sqrt(z), z);
    }
    return GQ_PIO2_F - gq_asin_kernel(x, x * x);
}

// atan for x >= 0
GQ_HD float gq_atan_pos(float x) {
    float y0, t;
    if (x > 2.414213562373095f) {  // tan(3 pi / 8)
        y0 = GQ_PIO2_F;
        t = gq_div(-1.0f, x);
    } else if (x > 0.4142135623730950f) {  // tan(pi / 8)
        y0 = GQ_PIO4_F;
        t = gq_div(x - 1.0f, x + 1.0f);
    } else {
        y0 = 0.0f;
        t = x;
    }
    float z = t * t;
    float p = 8.05374449538e-2f;
    p = gq_fma(p, z, -1.38776856032e-1f);
    p = gq_fma(p, z, 1.99777106478e-1f);
    p = gq_fma(p, z, -3.33329491539e-1f);
    return y0 + gq_fma(p * z, t, t);
}

GQ_HD float gq_atan(float x) {
    if (x != x) return x;
    float r = gq_atan_pos(fabsf(x));
    return x < 0.0f ? -r : r;
}

GQ_HD float gq_atan2(float y, float x) {
    if (x != x || y != y) return __builtin_nanf("");
    if (x == 0.0f) {
        if (y > 0.0f) return GQ_PIO2_F;
        if (y < 0.0f) return -GQ_PIO2_F;
        return signbit(x) ? (signbit(y) ? -GQ_PI_F : GQ_PI_F) : y;
    }
    if (y == 0.0f) {
        if (x > 0.0f) return y;
        return signbit(y) ? -GQ_PI_F : GQ_PI_F;
    }
    if (isinf(x) || isinf(y)) {
        if (isinf(x) && isinf(y)) {
            float base = x > 0.0f ? GQ_PIO4_F : 3.0f * GQ_PIO4_F;
            return y > 0.0f ? base : -base;
        }
        if (isinf(y)) return y > 0.0f ? GQ_PIO2_F : -GQ_PIO2_F;
        // finite y, infinite x
        if (x > 0.0f) return y > 0.0f ? 0.0f : -0.0f;
        return y > 0.0f ? GQ_PI_F : -GQ_PI_F;
    }
    float w = 0.0f;
    if (x < 0.0f) w = (y < 0.0f) ? -GQ_PI_F : GQ_PI_F;
    return w + gq_atan(gq_div(y, x));
}
