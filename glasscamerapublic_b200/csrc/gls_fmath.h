// gls_fmath.h — scalar arithmetic with a fixed rounding sequence, usable on
// the host and the device, for the registration path (SURF, homography,
// warps), whose outputs are compared bit for bit across the CPU and the GPU.
//
//  * fadd/fsub/fmul/fdiv (float) and dadd/dsub/dmul/ddiv (double) are single
//    IEEE operations in round-to-nearest: on the device the _rn intrinsics,
//    which the compiler never contracts into FMAs; on the host the plain
//    operators (host code is built without FP contraction).
//  * gls_atan2f, gls_sinf, gls_cosf are this library's own elementary
//    functions (the reference calls the platform's atan2f/sinf/cosf, whose
//    last-ulp behaviour differs between libraries). Method:
//      atan: argument reduction to t = min/max in [0, 1], then to
//            |u| <= tan(pi/12) by atan(t) = pi/6 + atan((sqrt3 t - 1)/(sqrt3 + t)),
//            and the Taylor series of atan through u^13 (truncation
//            < 2e-10 on |u| <= 0.268); quadrant and sign restored per
//            C99 Annex F (signed zeros, infinities, NaN);
//      sin/cos: reduction by pi/2 in double, then the Taylor series through
//            r^9 (sin) and r^10 (cos) on |r| <= pi/4.
//    Accuracy: atan2f within 3 float ulps, sinf/cosf within 2 ulps (tests
//    compare them with a double-precision evaluation).
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define GLS_HD __host__ __device__ __forceinline__
#else
#define GLS_HD inline
#endif

namespace glsm {

#if defined(__CUDA_ARCH__)
GLS_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
GLS_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
GLS_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
GLS_HD float fdiv(float a, float b) { return __fdiv_rn(a, b); }
GLS_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
GLS_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
GLS_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
GLS_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
GLS_HD double dsqrt(double a) { return __dsqrt_rn(a); }
GLS_HD float fsqrt(float a) { return __fsqrt_rn(a); }
#else
GLS_HD float fadd(float a, float b) { return a + b; }
GLS_HD float fsub(float a, float b) { return a - b; }
GLS_HD float fmul(float a, float b) { return a * b; }
GLS_HD float fdiv(float a, float b) { return a / b; }
GLS_HD double dadd(double a, double b) { return a + b; }
GLS_HD double dsub(double a, double b) { return a - b; }
GLS_HD double dmul(double a, double b) { return a * b; }
GLS_HD double ddiv(double a, double b) { return a / b; }
GLS_HD double dsqrt(double a) { return std::sqrt(a); }
GLS_HD float fsqrt(float a) { return std::sqrt(a); }
#endif

constexpr float kPi = 3.14159265358979323846f;
constexpr float kPi_2 = 1.57079632679489661923f;
constexpr float kPi_6 = 0.52359877559829887308f;
constexpr float kSqrt3 = 1.73205080756887729353f;
constexpr float kTanPi_12 = 0.26794919243112270647f;

// atan(u) for |u| <= tan(pi/12): u * (1 - u^2/3 + u^4/5 - ... + u^12/13)
GLS_HD float atan_core(float u) {
    const float z = fmul(u, u);
    float p = 1.0f / 13.0f;
    p = fsub(fmul(p, z), 1.0f / 11.0f);
    p = fadd(fmul(p, z), 1.0f / 9.0f);
    p = fsub(fmul(p, z), 1.0f / 7.0f);
    p = fadd(fmul(p, z), 1.0f / 5.0f);
    p = fsub(fmul(p, z), 1.0f / 3.0f);
    p = fmul(p, z);
    return fadd(u, fmul(u, p));
}

GLS_HD float gls_atan2f(float y, float x) {
    if (x != x || y != y) return x + y;  // NaN
    const bool yneg = std::signbit(y), xneg = std::signbit(x);
    const float ax = std::fabs(x), ay = std::fabs(y);
    float r;
    if (ay == 0.0f) {
        r = xneg ? kPi : 0.0f;
    } else if (std::isinf(ax) && std::isinf(ay)) {
        r = xneg ? 3.0f * kPi / 4.0f : kPi / 4.0f;
    } else if (ax == 0.0f || std::isinf(ay)) {
        r = kPi_2;
    } else if (std::isinf(ax)) {
        r = xneg ? kPi : 0.0f;
    } else {
        const bool swap = ay > ax;
        float t = swap ? fdiv(ax, ay) : fdiv(ay, ax);
        float a;
        if (t > kTanPi_12) {
            const float u = fdiv(fsub(fmul(t, kSqrt3), 1.0f), fadd(t, kSqrt3));
            a = fadd(kPi_6, atan_core(u));
        } else {
            a = atan_core(t);
        }
        if (swap) a = fsub(kPi_2, a);
        if (xneg) a = fsub(kPi, a);
        r = a;
    }
    return yneg ? -r : r;
}

// sin(r), cos(r) for |r| <= pi/4
GLS_HD float sin_core(float r) {
    const float z = fmul(r, r);
    float p = 1.0f / 362880.0f;
    p = fsub(fmul(p, z), 1.0f / 5040.0f);
    p = fadd(fmul(p, z), 1.0f / 120.0f);
    p = fsub(fmul(p, z), 1.0f / 6.0f);
    p = fmul(p, z);
    return fadd(r, fmul(r, p));
}
GLS_HD float cos_core(float r) {
    const float z = fmul(r, r);
    float p = -1.0f / 3628800.0f;
    p = fadd(fmul(p, z), 1.0f / 40320.0f);
    p = fsub(fmul(p, z), 1.0f / 720.0f);
    p = fadd(fmul(p, z), 1.0f / 24.0f);
    p = fsub(fmul(p, z), 0.5f);
    return fadd(1.0f, fmul(z, p));
}

// quadrant reduction: x = k pi/2 + r, with r formed in double (the
// product k pi/2 and the difference are exact to ~1e-16 for |x| < 2^20)
GLS_HD int reduce_pi_2(float x, float* r) {
    constexpr double kInvPi_2 = 0.63661977236758134308;
    constexpr double kPi_2d = 1.57079632679489661923;
    const double k = std::rint(dmul(double(x), kInvPi_2));
    *r = float(dsub(double(x), dmul(k, kPi_2d)));
    return int(k) & 3;
}

GLS_HD float gls_sinf(float x) {
    if (!std::isfinite(x)) return x - x;
    if (std::fabs(x) <= kPi / 4.0f) return sin_core(x);
    float r;
    switch (reduce_pi_2(x, &r)) {
        case 0: return sin_core(r);
        case 1: return cos_core(r);
        case 2: return -sin_core(r);
        default: return -cos_core(r);
    }
}

GLS_HD float gls_cosf(float x) {
    if (!std::isfinite(x)) return x - x;
    if (std::fabs(x) <= kPi / 4.0f) return cos_core(x);
    float r;
    switch (reduce_pi_2(x, &r)) {
        case 0: return cos_core(r);
        case 1: return -sin_core(r);
        case 2: return -cos_core(r);
        default: return sin_core(r);
    }
}

}  // namespace glsm
