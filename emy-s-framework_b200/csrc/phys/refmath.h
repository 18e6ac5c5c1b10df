// Float functions whose exact results the reference simulator's CPU build depends on,
// restated so that the device computes the same bits as the host it is compared with.
//
// The reference (RocketSim + Bullet 3.24, x86-64, glibc) takes three kinds of inexact
// single-precision values from outside its own sources:
//   1. btVector3::normalize seeds its Newton step with the CPU's `rsqrtss` estimate
//      (bullet3-3.24/LinearMath/btVector3.h:324).  The estimate is a hardware table: on the
//      CPUs measured it depends only on the exponent's parity and the top 10-12 mantissa
//      bits.  rsqrtEstimate() reads a 2 x 4096 table sampled from the host CPU at start-up
//      (sampleRsqrtTable(), which also checks that the CPU's estimate has that form);
//   2. sinf / cosf (btTransformUtil::integrateTransform, Car.cpp:725-726, MathTypes.cpp)
//      come from glibc, whose x86-64 build runs the ARM optimized-routines algorithm
//      (Szabolcs Nagy, 2018: double-precision polynomials, reduction by a prescaled 2/pi
//      multiply for |x| < 120) with FMA contraction on CPUs that have FMA;
//   3. atan2f / asinf (btInternalEdgeUtility, btBoxBoxDetector, btMatrix3x3::getEulerYPR)
//      come from glibc's single-precision fdlibm atan2f / atanf (Sun Microsystems, 1993:
//      reduction to four breakpoints and an 11-term odd polynomial) and its asinf
//      (x + x^3 p(x^2) with a 5-term polynomial below 0.5, half-angle form above).
// None of these is correctly rounded; CUDA's own functions differ from glibc's on 0.1-0.8 %
// of inputs.  The routines below evaluate the published methods with the same operation
// order, so they return glibc's bits: checked against the host library over every float
// (sin/cos for |x| < 120, asin, atan) and on dense samples (atan2) in tests/test_refmath.py.
// Outside |x| < 120, which no simulated angle reaches, rsSinf / rsCosf use the platform
// function.
#pragma once
#include "hd.h"

#include <xmmintrin.h>

namespace rsb {

RSB_HD uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}
RSB_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

// ------------------------------------------------------------------ rsqrtss estimate

// Table of the host CPU's estimate: entry (p << 12) | i holds rsqrtss((1 + i / 4096) * 2^p)
// as bits.  Filled once per device before the first launch.
constexpr int kRsqrtTableSize = 2 * 4096;
#if defined(__CUDACC__)
__device__ uint32_t g_rsqrtTable[kRsqrtTableSize];
#endif

// rsqrtss on one float from a sampled table: +-0 and subnormals give +-inf, +inf gives 0,
// other negatives the default NaN, NaNs pass through quieted.  A normal x = m 2^(2k + p)
// gives estimate(m 2^p) scaled by 2^-k, which is exact.
RSB_HD float rsqrtFromTable(const uint32_t* table, float x) {
    const uint32_t u = f2u(x);
    const uint32_t ax = u & 0x7fffffffu;
    if (ax < 0x00800000u) return u2f((u & 0x80000000u) | 0x7f800000u);
    if (ax > 0x7f800000u) return u2f(u | 0x00400000u);
    if (u & 0x80000000u) return u2f(0xffc00000u);
    if (ax == 0x7f800000u) return 0.f;
    const int e = (int)(u >> 23) - 127;
    const int p = e & 1;
    const int k = (e - p) / 2;
    const uint32_t t = table[(p << 12) | ((u >> 11) & 0xfffu)];
    return u2f((uint32_t)((int)t - k * (1 << 23)));
}

// The estimate btVector3::normalize starts from: the sampled table on the device, the
// instruction itself on the host.
RSB_HD float rsqrtEstimate(float x) {
#if defined(__CUDA_ARCH__)
    return rsqrtFromTable(g_rsqrtTable, x);
#else
    return _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x)));
#endif
}

// Samples the host CPU's rsqrtss into `table` and checks, over every mantissa of [1, 4) and
// a spread of exponents, that the estimate has the form rsqrtEstimate() assumes.  Returns
// false (table then holds correctly rounded 1/sqrt of each entry's input) when it does not.
inline bool sampleRsqrtTable(uint32_t* table) {
    auto est = [](float x) { return _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x))); };
    for (int p = 0; p < 2; p++)
        for (int i = 0; i < 4096; i++) table[(p << 12) | i] = f2u(est(u2f((uint32_t)(127 + p) << 23 | (uint32_t)i << 11)));
    bool ok = true;
    for (int p = 0; p < 2 && ok; p++)
        for (uint32_t m = 0; m < (1u << 23); m++)
            if (f2u(est(u2f((uint32_t)(127 + p) << 23 | m))) != table[(p << 12) | (m >> 11)]) { ok = false; break; }
    for (int e = 1; e < 254 && ok; e += 3)
        for (uint32_t m = 0; m < (1u << 23); m += 4093) {
            const uint32_t u = (uint32_t)e << 23 | m;
            const int q = e - 127, p = q & 1, k = (q - p) / 2;
            if (f2u(est(u2f(u))) != (uint32_t)((int)table[(p << 12) | (m >> 11)] - k * (1 << 23))) { ok = false; break; }
        }
    if (!ok)
        for (int p = 0; p < 2; p++)
            for (int i = 0; i < 4096; i++)
                table[(p << 12) | i] = f2u(1.f / sqrtf(u2f((uint32_t)(127 + p) << 23 | (uint32_t)i << 11)));
    return ok;
}

// ------------------------------------------------------------------ sin / cos

// Coefficients of the quadrant polynomials: cos ~ c0 + c1 x^2 + ... + c4 x^8, sin ~ x + s1 x^3 +
// s2 x^5 + s3 x^7 on |x| <= pi/4; the second set returns -cos (quadrants 2 and 3).
struct SinCosPoly {
    double c0, c1, c2, c3, c4, s1, s2, s3;
};
RSB_HD SinCosPoly sinCosPoly(int neg) {
    const double sg = neg ? -1.0 : 1.0;
    return SinCosPoly{sg * 0x1p0, sg * -0x1.ffffffd0c621cp-2, sg * 0x1.55553e1068f19p-5, sg * -0x1.6c087e89a359dp-10,
                      sg * 0x1.99343027bf8c3p-16, -0x1.555545995a603p-3, 0x1.1107605230bc4p-7, -0x1.994eb3774cf24p-13};
}

// Exponent and top 3 mantissa bits of |x|: the range tests compare these, not |x| itself.
RSB_HD uint32_t absTop12(float x) { return (f2u(x) >> 20) & 0x7ffu; }

// Odd quadrant n: the cosine polynomial; even: the sine polynomial.  Products feeding an add
// are fused, as the FMA build of the reference's C library evaluates them.
RSB_HD float sinCosQuadrant(double x, double x2, const SinCosPoly& p, int n) {
    if ((n & 1) == 0) {
        const double x3 = x * x2;
        const double s1 = fma(x2, p.s3, p.s2);
        const double x7 = x3 * x2;
        const double s = fma(x3, p.s1, x);
        return (float)fma(x7, s1, s);
    }
    const double x4 = x2 * x2;
    const double c2 = fma(x2, p.c4, p.c3);
    const double c1 = fma(x2, p.c1, p.c0);
    const double x6 = x4 * x2;
    const double c = fma(x4, p.c2, c1);
    return (float)fma(x6, c2, c);
}

// x minus the nearest multiple of pi/2 (|x| < 120): 2/pi prescaled by 2^24 so the quadrant
// lands in bits 24..31 of a truncated integer, rounded by adding half a quadrant.
RSB_HD double sinCosReduce(double x, int& n) {
    const double r = x * 0x1.45F306DC9C883p+23;
    n = ((int32_t)r + 0x800000) >> 24;
    return fma(-(double)n, 0x1.921FB54442D18p0, x);
}

RSB_HD float rsSinf(float y) {
    const double x = y;
    if (absTop12(y) < absTop12(0x1.921FB6p-1f)) {
        if (absTop12(y) < absTop12(0x1p-12f)) return y;
        return sinCosQuadrant(x, x * x, sinCosPoly(0), 0);
    }
    if (absTop12(y) < absTop12(120.0f)) {
        int n;
        const double r = sinCosReduce(x, n);
        const double s = ((n & 3) == 1 || (n & 3) == 2) ? -1.0 : 1.0;
        return sinCosQuadrant(r * s, r * r, sinCosPoly(n & 2), n);
    }
    return sinf(y);
}

RSB_HD float rsCosf(float y) {
    const double x = y;
    if (absTop12(y) < absTop12(0x1.921FB6p-1f)) {
        if (absTop12(y) < absTop12(0x1p-12f)) return 1.0f;
        return sinCosQuadrant(x, x * x, sinCosPoly(0), 1);
    }
    if (absTop12(y) < absTop12(120.0f)) {
        int n;
        const double r = sinCosReduce(x, n);
        const double s = ((n & 3) == 1 || (n & 3) == 2) ? -1.0 : 1.0;
        return sinCosQuadrant(r * s, r * r, sinCosPoly(n & 2), n ^ 1);
    }
    return cosf(y);
}

// ------------------------------------------------------------------ atan / atan2 / asin

// atan in single precision: reduce |x| to one of four breakpoints (0.5, 1, 1.5, inf) with
// atan(b) split into high and low parts, then an odd polynomial in the remainder.
RSB_HD float rsAtanf(float x) {
    const float hi[4] = {4.6364760399e-01f, 7.8539812565e-01f, 9.8279368877e-01f, 1.5707962513e+00f};
    const float lo[4] = {5.0121582440e-09f, 3.7748947079e-08f, 3.4473217170e-08f, 7.5497894159e-08f};
    const float T0 = 3.3333334327e-01f, T1 = -2.0000000298e-01f, T2 = 1.4285714924e-01f, T3 = -1.1111110449e-01f,
                T4 = 9.0908870101e-02f, T5 = -7.6918758452e-02f, T6 = 6.6610731184e-02f, T7 = -5.8335702866e-02f,
                T8 = 4.9768779427e-02f, T9 = -3.6531571299e-02f, T10 = 1.6285819933e-02f;
    const int32_t hx = (int32_t)f2u(x), ix = hx & 0x7fffffff;
    int id;
    if (ix >= 0x4c000000) {  // |x| >= 2^25
        if (ix > 0x7f800000) return x + x;
        return hx > 0 ? hi[3] + lo[3] : -hi[3] - lo[3];
    }
    if (ix < 0x3ee00000) {  // |x| < 0.4375
        if (ix < 0x31000000) return x;
        id = -1;
    } else {
        x = fabsf(x);
        if (ix < 0x3f980000) {
            if (ix < 0x3f300000) { id = 0; x = (2.0f * x - 1.0f) / (2.0f + x); }
            else { id = 1; x = (x - 1.0f) / (x + 1.0f); }
        } else {
            if (ix < 0x401c0000) { id = 2; x = (x - 1.5f) / (1.0f + 1.5f * x); }
            else { id = 3; x = -1.0f / x; }
        }
    }
    const float z = x * x, w = z * z;
    const float s1 = z * (T0 + w * (T2 + w * (T4 + w * (T6 + w * (T8 + w * T10)))));
    const float s2 = w * (T1 + w * (T3 + w * (T5 + w * (T7 + w * T9))));
    if (id < 0) return x - x * (s1 + s2);
    const float r = hi[id] - ((x * (s1 + s2) - lo[id]) - x);
    return hx < 0 ? -r : r;
}

RSB_HD float rsAtan2f(float y, float x) {
    const float tiny = 1.0e-30f, piO4 = 7.8539818525e-01f, piO2 = 1.5707963705e+00f, pi = 3.1415927410e+00f,
                piLo = -8.7422776573e-08f;
    const int32_t hx = (int32_t)f2u(x), ix = hx & 0x7fffffff, hy = (int32_t)f2u(y), iy = hy & 0x7fffffff;
    if (ix > 0x7f800000 || iy > 0x7f800000) return x + y;
    if (hx == 0x3f800000) return rsAtanf(y);
    const int m = ((hy >> 31) & 1) | ((hx >> 30) & 2);  // 2 * sign(x) + sign(y)
    if (iy == 0) return m < 2 ? y : (m == 2 ? pi + tiny : -pi - tiny);
    if (ix == 0) return hy < 0 ? -piO2 - tiny : piO2 + tiny;
    if (ix == 0x7f800000) {
        if (iy == 0x7f800000) {
            const float q[4] = {piO4 + tiny, -piO4 - tiny, 3.0f * piO4 + tiny, -3.0f * piO4 - tiny};
            return q[m];
        }
        const float q[4] = {0.0f, -0.0f, pi + tiny, -pi - tiny};
        return q[m];
    }
    if (iy == 0x7f800000) return hy < 0 ? -piO2 - tiny : piO2 + tiny;
    const int k = (iy - ix) >> 23;
    float z;
    if (k > 60) z = piO2 + 0.5f * piLo;
    else if (hx < 0 && k < -60) z = 0.0f;
    else z = rsAtanf(fabsf(y / x));
    switch (m) {
        case 0: return z;
        case 1: return u2f(f2u(z) ^ 0x80000000u);
        case 2: return pi - (z - piLo);
        default: return (z - piLo) - pi;
    }
}

RSB_HD float rsAsinf(float x) {
    const float pio2Hi = 1.57079637050628662109375f, pio2Lo = -4.37113900018624283e-8f,
                pio4Hi = 0.785398185253143310546875f;
    const float p0 = 1.666675248e-1f, p1 = 7.495297643e-2f, p2 = 4.547037598e-2f, p3 = 2.417951451e-2f,
                p4 = 4.216630880e-2f;
    const int32_t hx = (int32_t)f2u(x), ix = hx & 0x7fffffff;
    if (ix == 0x3f800000) return x * pio2Hi + x * pio2Lo;
    if (ix > 0x3f800000) return (x - x) / (x - x);
    if (ix < 0x3f000000) {  // |x| < 0.5
        if (ix < 0x32000000) return x;
        const float t = x * x;
        const float w = t * (p0 + t * (p1 + t * (p2 + t * (p3 + t * p4))));
        return x + x * w;
    }
    const float t = (1.0f - fabsf(x)) * 0.5f;
    const float p = t * (p0 + t * (p1 + t * (p2 + t * (p3 + t * p4))));
    const float s = sqrtf(t);
    float r;
    if (ix >= 0x3F79999A) {  // |x| > 0.975
        r = pio2Hi - (2.0f * (s + s * p) - pio2Lo);
    } else {
        const float w = u2f(f2u(s) & 0xfffff000u);
        const float c = (t - w * w) / (s + w);
        const float pp = 2.0f * s * p - (pio2Lo - 2.0f * c);
        const float q = pio4Hi - 2.0f * w;
        r = pio4Hi - (pp - q);
    }
    return hx > 0 ? r : -r;
}

}  // namespace rsb
