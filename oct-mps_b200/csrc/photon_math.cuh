// Device arithmetic of the photon method.
//
// Everything here is deterministic IEEE arithmetic so that a host
// implementation of the same steps reproduces it bit for bit: the file is
// compiled with -fmad=false (only the fmaf/fma calls written out fuse),
// float division and square root are the correctly rounded ones, double
// division rounds toward minus infinity like the reference's FAST_DIV
// (src/octmps_kernel.h:38), and log / sin / cos are the project's own
// series (no CUDA math-library transcendentals):
//  * log: x = m*2^e, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s),
//    s = (m-1)/(m+1), by the Taylor series of atanh (terms to s^9 in float,
//    s^21 in double); log 2 split in a short high part and a low part so
//    that e*log2_hi is exact (Cody and Waite's method).
//  * sin/cos of the azimuth: float: exact reduction of the turn fraction
//    t in [0,1) to r = t - rint(4t)/4, then Taylor polynomials of sin and
//    cos of 2*pi*r (to r^9 / r^10); double: psi = 2*PI_const*t as in the
//    reference (src/octmps_kernel.cuh:846), Cody-Waite reduction by pi/2
//    held in two doubles, Taylor polynomials to r^17 / r^18.
#ifndef OCTMPS_PHOTON_MATH_CUH
#define OCTMPS_PHOTON_MATH_CUH

#include <cmath>
#include <cstdint>
#include <cstring>

namespace octmps {

// Bit casts and fused multiply-adds usable on both sides: the host derives a
// few per-job constants (region_consts.h) with the kernel's own logarithm.
__host__ __device__ __forceinline__ uint32_t bits_of(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}
__host__ __device__ __forceinline__ float float_of(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}
__host__ __device__ __forceinline__ uint64_t bits_of(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}
__host__ __device__ __forceinline__ double double_of(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}
__host__ __device__ __forceinline__ float fma_rn(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
__host__ __device__ __forceinline__ double fma_rn(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

__host__ __device__ __forceinline__ float log_method(float x) {
    if (x == 0.0f) return -float_of(0x7f800000u);
    if (!(x > 0.0f) || std::isinf(x)) return x < 0.0f ? float_of(0x7fc00000u) : x;
    uint32_t b = bits_of(x);
    int e = 0;
    if (b < 0x00800000u) {
        b = bits_of(x * 0x1p23f);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    uint32_t mb = (b & 0x007fffffu) | 0x3f800000u;
    if (mb > 0x3fb504f3u) {
        mb -= 0x00800000u;
        e += 1;
    }
    const float m = float_of(mb);
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    const float t = s + s;
    float p = fma_rn(z, 0x1.c71c72p-4f, 0x1.24924ap-3f);
    p = fma_rn(z, p, 0x1.99999ap-3f);
    p = fma_rn(z, p, 0x1.555556p-2f);
    const float lm = fma_rn(t * z, p, t);
    const float ef = (float)e;
    return fma_rn(ef, 0x1.62e400p-1f, fma_rn(ef, 0x1.7f7d1cp-20f, lm));
}

// log_method for a positive, finite, normal x (the step-size draws, 1 - a
// random number in [0, 1): at least 2^-24): the same operations without the
// special cases, which such an x never reaches.
__device__ __forceinline__ float log_method_normal(float x) {
    const uint32_t b = bits_of(x);
    const bool hi = (b & 0x007fffffu) > 0x003504f3u;  // mantissa above sqrt(2)
    const uint32_t mb = ((b & 0x007fffffu) | 0x3f800000u) - (hi ? 0x00800000u : 0u);
    const int e = (int)(b >> 23) - 127 + (hi ? 1 : 0);
    const float m = float_of(mb);
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    const float t = s + s;
    float p = fma_rn(z, 0x1.c71c72p-4f, 0x1.24924ap-3f);
    p = fma_rn(z, p, 0x1.99999ap-3f);
    p = fma_rn(z, p, 0x1.555556p-2f);
    const float lm = fma_rn(t * z, p, t);
    const float ef = (float)e;
    return fma_rn(ef, 0x1.62e400p-1f, fma_rn(ef, 0x1.7f7d1cp-20f, lm));
}

__host__ __device__ __forceinline__ double log_method(double x) {
    if (x == 0.0) return -double_of(0x7ff0000000000000ull);
    if (!(x > 0.0) || std::isinf(x)) return x < 0.0 ? double_of(0x7ff8000000000000ull) : x;
    uint64_t b = bits_of(x);
    int e = 0;
    if (b < 0x0010000000000000ull) {
        b = bits_of(x * 0x1p54);
        e = -54;
    }
    e += (int)(b >> 52) - 1023;
    uint64_t mb = (b & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    if (mb > 0x3ff6a09e667f3bcdull) {
        mb -= 0x0010000000000000ull;
        e += 1;
    }
    const double m = double_of(mb);
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    const double t = s + s;
    double p = fma_rn(z, 0x1.8618618618618p-5, 0x1.af286bca1af28p-5);
    p = fma_rn(z, p, 0x1.e1e1e1e1e1e1ep-5);
    p = fma_rn(z, p, 0x1.1111111111111p-4);
    p = fma_rn(z, p, 0x1.3b13b13b13b14p-4);
    p = fma_rn(z, p, 0x1.745d1745d1746p-4);
    p = fma_rn(z, p, 0x1.c71c71c71c71cp-4);
    p = fma_rn(z, p, 0x1.2492492492492p-3);
    p = fma_rn(z, p, 0x1.999999999999ap-3);
    p = fma_rn(z, p, 0x1.5555555555555p-2);
    const double lm = fma_rn(t * z, p, t);
    const double ef = (double)e;
    return fma_rn(ef, 0x1.62e42fee00000p-1, fma_rn(ef, 0x1.a39ef35793c76p-33, lm));
}

__device__ __forceinline__ double log_method_normal(double x) {
    const uint64_t b = bits_of(x);
    const bool hi = (b & 0x000fffffffffffffull) > 0x0006a09e667f3bcdull;
    const uint64_t mb =
        ((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull) - (hi ? 0x0010000000000000ull : 0ull);
    const int e = (int)(b >> 52) - 1023 + (hi ? 1 : 0);
    const double m = double_of(mb);
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    const double t = s + s;
    double p = fma_rn(z, 0x1.8618618618618p-5, 0x1.af286bca1af28p-5);
    p = fma_rn(z, p, 0x1.e1e1e1e1e1e1ep-5);
    p = fma_rn(z, p, 0x1.1111111111111p-4);
    p = fma_rn(z, p, 0x1.3b13b13b13b14p-4);
    p = fma_rn(z, p, 0x1.745d1745d1746p-4);
    p = fma_rn(z, p, 0x1.c71c71c71c71cp-4);
    p = fma_rn(z, p, 0x1.2492492492492p-3);
    p = fma_rn(z, p, 0x1.999999999999ap-3);
    p = fma_rn(z, p, 0x1.5555555555555p-2);
    const double lm = fma_rn(t * z, p, t);
    const double ef = (double)e;
    return fma_rn(ef, 0x1.62e42fee00000p-1, fma_rn(ef, 0x1.a39ef35793c76p-33, lm));
}

__device__ __forceinline__ void sincos_poly(float r, float &s, float &c) {
    const float z = r * r;
    float ps = __fmaf_rn(z, 0x1.71de3ap-19f, -0x1.a01a02p-13f);
    ps = __fmaf_rn(z, ps, 0x1.111112p-7f);
    ps = __fmaf_rn(z, ps, -0x1.555556p-3f);
    s = __fmaf_rn(r * z, ps, r);
    float pc = __fmaf_rn(z, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = __fmaf_rn(z, pc, -0x1.6c16c2p-10f);
    pc = __fmaf_rn(z, pc, 0x1.555556p-5f);
    pc = __fmaf_rn(z, pc, -0.5f);
    c = __fmaf_rn(z, pc, 1.0f);
}

__device__ __forceinline__ void sincos_poly(double r, double &s, double &c) {
    const double z = r * r;
    double ps = __fma_rn(z, 0x1.952c77030ad4ap-49, -0x1.ae7f3e733b81fp-41);
    ps = __fma_rn(z, ps, 0x1.6124613a86d09p-33);
    ps = __fma_rn(z, ps, -0x1.ae64567f544e4p-26);
    ps = __fma_rn(z, ps, 0x1.71de3a556c734p-19);
    ps = __fma_rn(z, ps, -0x1.a01a01a01a01ap-13);
    ps = __fma_rn(z, ps, 0x1.1111111111111p-7);
    ps = __fma_rn(z, ps, -0x1.5555555555555p-3);
    s = __fma_rn(r * z, ps, r);
    double pc = __fma_rn(z, -0x1.6827863b97d97p-53, 0x1.ae7f3e733b81fp-45);
    pc = __fma_rn(z, pc, -0x1.93974a8c07c9dp-37);
    pc = __fma_rn(z, pc, 0x1.1eed8eff8d898p-29);
    pc = __fma_rn(z, pc, -0x1.27e4fb7789f5cp-22);
    pc = __fma_rn(z, pc, 0x1.a01a01a01a01ap-16);
    pc = __fma_rn(z, pc, -0x1.6c16c16c16c17p-10);
    pc = __fma_rn(z, pc, 0x1.5555555555555p-5);
    pc = __fma_rn(z, pc, -0.5);
    c = __fma_rn(z, pc, 1.0);
}

template <typename T>
__device__ __forceinline__ void quadrant(int q, T sr, T cr, T &s, T &c) {
    switch (q & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}

// sin and cos of the azimuth 2*pi*t, t = a [0,1) random number.
__device__ __forceinline__ void sincos_rand(float t, float &s, float &c) {
    const float q = rintf(t * 4.0f);
    const float r = __fmaf_rn(q, -0.25f, t);
    const float th = r * 0x1.921fb6p+2f;
    float sr, cr;
    sincos_poly(th, sr, cr);
    quadrant((int)q, sr, cr, s, c);
}

__device__ __forceinline__ void sincos_rand(double t, double &s, double &c) {
    const double psi = (2.0 * 3.14159265359) * t;
    const double q = rint(psi * 0x1.45f306dc9c883p-1);
    double r = __fma_rn(-q, 0x1.921fb54442d18p+0, psi);
    r = __fma_rn(-q, 0x1.1a62633145c07p-54, r);
    double sr, cr;
    sincos_poly(r, sr, cr);
    quadrant((int)q, sr, cr, s, c);
}

// Precision-generic IEEE operations; the intrinsics are never contracted
// or approximated.
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float sqrtT(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrtT(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float rcpT(float a) { return __fdiv_rn(1.0f, a); }
__device__ __forceinline__ double rcpT(double a) { return __ddiv_rn(1.0, a); }
__device__ __forceinline__ float fabsT(float a) { return fabsf(a); }
__device__ __forceinline__ double fabsT(double a) { return fabs(a); }
__device__ __forceinline__ float fminT(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double fminT(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float fmaxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmaxT(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float copysignT(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double copysignT(double a, double b) { return copysign(a, b); }

template <typename T>
struct DevNum;

template <>
struct DevNum<float> {
    // a*b + c fused (one rounding) in the FP32 forms
    static __device__ __forceinline__ float mad(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float rand_value(uint32_t u) {
        return __uint2float_rz(u) * 0x1p-32f;
    }
    static constexpr float coszero = 0.999999f;
    static constexpr float cos90 = 1.0e-6f;
    static constexpr float weight = 1.0e-4f;
    static constexpr float chance = 0.1f;
    static constexpr float big = 1.0e10f;
};

template <>
struct DevNum<double> {
    // a*b + c with the product and the sum rounded separately, as the
    // reference's source reads without contraction
    static __device__ __forceinline__ double mad(double a, double b, double c) {
        return __dadd_rn(__dmul_rn(a, b), c);
    }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rd(a, b); }
    static __device__ __forceinline__ double rand_value(uint32_t u) {
        return (double)__uint2float_rz(u) * 0x1p-32;
    }
    static constexpr double coszero = 1.0 - 1.0e-14;
    static constexpr double cos90 = 1.0e-6;
    static constexpr double weight = 1.0e-4;
    static constexpr double chance = 0.1;
    static constexpr double big = 1.0e10;
};

// The FP32 forms (fused multiply-adds) also take a few cheaper, equally
// accurate formulations of the same quantities; the FP64 form keeps the
// reference's operations.
template <typename T>
constexpr bool kFused = sizeof(T) == sizeof(float);

// a.x + b.y + c.z as (a.x + b.y) + c.z, the reference's order.
template <typename T>
__device__ __forceinline__ T dot3(T a, T b, T c, T x, T y, T z) {
    return DevNum<T>::mad(c, z, DevNum<T>::mad(a, x, b * y));
}

// Multiply-with-carry step, src/octmps_kernel.cuh:16.
__device__ __forceinline__ uint32_t mwc_next(uint64_t &x, uint32_t a) {
    x = (x & 0xffffffffull) * (uint64_t)a + (x >> 32);
    return (uint32_t)x;
}

}  // namespace octmps

#endif
