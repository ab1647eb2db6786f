// dl_math.h — elementary functions shared by the CUDA kernels and the CPU oracle.
//
// The render and voxel pipelines turn floating-point results into integers
// (tile ranges from `ceil(radius)`, sort keys from depths, voxel bits from a
// threshold).  For those integers to agree bit-for-bit between the GPU and the
// CPU, every transcendental on the decision path must produce the same bits on
// both sides.  CUDA's and glibc's `expf` do not, so this header provides one
// implementation, built only from correctly rounded IEEE operations (+, *, /,
// sqrt, fma, rint) that compile identically for host and device.
//
// Methods (all from the public literature, constants derived here):
//   * exp (f32, f64): Cody & Waite (1980) additive argument reduction
//     x = k*ln2 + r, |r| <= ln2/2, with ln2 split into a short high part and a
//     low correction; e^r by its Taylor series in Horner form (degree 7 in f32,
//     degree 13 in f64, truncation error < 0.1 ulp), then an exact scaling by
//     2^k done in two halves so subnormal results are rounded only once.
//   * atan2 / asin (computed in f64, returned as f32): octant reduction to
//     t in [0, 1], then atan(t) = pi/6 + atan((t*sqrt3 - 1)/(t + sqrt3)) for
//     t > tan(pi/12) (Cody & Waite, ch. 14), and the odd Taylor series of atan
//     on |u| <= tan(pi/12).  asin(x) = atan2(x, sqrt((1-x)(1+x))).
//
// Reference semantics this stands in for: WGSL `exp`, `atan2`, `asin` in
// src/render/shaders/project.ts:55,77,258-259 and
// src/voxel/shaders/voxelize.ts:78-83,440, and JS `Math.exp` in
// src/spatial/aabb.ts:33-35.  WGSL only bounds their error (exp: 3+2|x| ulp),
// so any implementation within those bounds is a faithful restatement; the
// tests check this one against glibc to <= 2 ulp (f32) and <= 1 ulp (f64).
//
// Build rule: translation units including this header must be compiled with
// FMA contraction off (nvcc --fmad=false, gcc -ffp-contract=off) and without
// fast-math / flush-to-zero; the explicit dl_fma calls are the only fused ops.
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define DL_HD __host__ __device__ __forceinline__
#else
#define DL_HD static inline
#endif

DL_HD float dl_fmaf(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

DL_HD double dl_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

DL_HD uint32_t dl_f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

DL_HD float dl_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

DL_HD double dl_u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d; memcpy(&d, &u, 8); return d;
#endif
}

// 2^e for e in [-126, 127] (exact power of two).
DL_HD float dl_pow2f(int e) { return dl_u2f((uint32_t)(e + 127) << 23); }
// 2^e for e in [-1022, 1023].
DL_HD double dl_pow2(int e) { return dl_u2d((uint64_t)(e + 1023) << 52); }

// ---------------------------------------------------------------- exp (f32)
DL_HD float dl_expf(float x) {
    if (!(x == x)) return x;                       // NaN propagates
    if (x > 89.0f) return dl_u2f(0x7f800000u);     // +inf (true overflow starts at 88.7228)
    if (x < -104.0f) return 0.0f;                  // below half the smallest subnormal
    const float k = rintf(x * 1.44269502162933349609375f);   // round(x / ln2)
    // ln2 = 0.693145751953125 (16 significant bits) + 1.4286068203e-06
    float r = dl_fmaf(-k, 0.693145751953125f, x);
    r = dl_fmaf(-k, 1.42860682028622676e-06f, r);
    // Taylor coefficients 1/n!, n = 7 .. 0
    float p = 1.98412698412698413e-04f;
    p = dl_fmaf(p, r, 1.38888888888888889e-03f);
    p = dl_fmaf(p, r, 8.33333333333333333e-03f);
    p = dl_fmaf(p, r, 4.16666666666666667e-02f);
    p = dl_fmaf(p, r, 1.66666666666666667e-01f);
    p = dl_fmaf(p, r, 0.5f);
    p = dl_fmaf(p, r, 1.0f);
    p = dl_fmaf(p, r, 1.0f);
    const int ki = (int)k;
    const int k1 = ki / 2;           // both halves stay inside the normal range
    const int k2 = ki - k1;
    return (p * dl_pow2f(k1)) * dl_pow2f(k2);
}

// Logistic function 1 / (1 + e^-x) exactly as written in the shaders.
DL_HD float dl_sigmoidf(float x) { return 1.0f / (1.0f + dl_expf(-x)); }

// ---------------------------------------------------------------- exp (f64)
DL_HD double dl_exp(double x) {
    if (!(x == x)) return x;
    if (x > 710.0) return dl_u2d(0x7ff0000000000000ull);
    if (x < -746.0) return 0.0;
    const double k = rint(x * 1.4426950408889634074);
    // ln2 split: 33 significant bits + remainder
    double r = dl_fma(-k, 6.93147180369123816490e-01, x);
    r = dl_fma(-k, 1.90821492927058770002e-10, r);
    // Taylor coefficients 1/n!, n = 13 .. 0
    double p = 1.6059043836821614599e-10;
    p = dl_fma(p, r, 2.0876756987868098979e-09);
    p = dl_fma(p, r, 2.5052108385441718775e-08);
    p = dl_fma(p, r, 2.7557319223985890653e-07);
    p = dl_fma(p, r, 2.7557319223985890653e-06);
    p = dl_fma(p, r, 2.4801587301587301587e-05);
    p = dl_fma(p, r, 1.9841269841269841270e-04);
    p = dl_fma(p, r, 1.3888888888888888889e-03);
    p = dl_fma(p, r, 8.3333333333333333333e-03);
    p = dl_fma(p, r, 4.1666666666666666667e-02);
    p = dl_fma(p, r, 1.6666666666666666667e-01);
    p = dl_fma(p, r, 0.5);
    p = dl_fma(p, r, 1.0);
    p = dl_fma(p, r, 1.0);
    const int ki = (int)k;
    const int k1 = ki / 2;
    const int k2 = ki - k1;
    return (p * dl_pow2(k1)) * dl_pow2(k2);
}

// ---------------------------------------------------------------- atan (f64)
// atan(u) for |u| <= tan(pi/12) ~ 0.2679 by the odd Taylor series
// sum_{n>=0} (-1)^n u^(2n+1)/(2n+1), 15 terms (remainder < 1e-18).
DL_HD double dl_atan_small(double u) {
    const double u2 = u * u;
    double p = -1.0 / 29.0;
    p = dl_fma(p, u2,  1.0 / 27.0);
    p = dl_fma(p, u2, -1.0 / 25.0);
    p = dl_fma(p, u2,  1.0 / 23.0);
    p = dl_fma(p, u2, -1.0 / 21.0);
    p = dl_fma(p, u2,  1.0 / 19.0);
    p = dl_fma(p, u2, -1.0 / 17.0);
    p = dl_fma(p, u2,  1.0 / 15.0);
    p = dl_fma(p, u2, -1.0 / 13.0);
    p = dl_fma(p, u2,  1.0 / 11.0);
    p = dl_fma(p, u2, -1.0 / 9.0);
    p = dl_fma(p, u2,  1.0 / 7.0);
    p = dl_fma(p, u2, -1.0 / 5.0);
    p = dl_fma(p, u2,  1.0 / 3.0);
    p = dl_fma(p, u2, -1.0);
    // p = -(1 - u2/3 + u2^2/5 - ...), so atan(u) = -u * p
    return -u * p;
}

DL_HD double dl_atan01(double t) {           // t in [0, 1]
    const double kTanPi12 = 0.26794919243112270647;   // 2 - sqrt(3)
    const double kSqrt3 = 1.7320508075688772935;
    const double kPi6 = 0.52359877559829887308;
    if (t <= kTanPi12) return dl_atan_small(t);
    const double u = (t * kSqrt3 - 1.0) / (t + kSqrt3);
    return kPi6 + dl_atan_small(u);
}

DL_HD double dl_atan2(double y, double x) {
    const double kPi = 3.14159265358979323846;
    const double kPi2 = 1.57079632679489661923;
    if (!(y == y) || !(x == x)) return y + x;
    const double ay = fabs(y), ax = fabs(x);
    if (ay == 0.0 && ax == 0.0) return 0.0;
    double a;
    const double kInf = dl_u2d(0x7ff0000000000000ull);
    if (ay <= ax) {
        a = (ax == kInf) ? ((ay == ax) ? 0.78539816339744830962 : 0.0) : dl_atan01(ay / ax);
    } else {
        a = (ay == kInf) ? kPi2 : kPi2 - dl_atan01(ax / ay);
    }
    if (x < 0.0) a = kPi - a;
    return (y < 0.0) ? -a : a;
}

// f32 wrappers: evaluate in f64, round once to f32.
DL_HD float dl_atan2f(float y, float x) { return (float)dl_atan2((double)y, (double)x); }
DL_HD float dl_asinf(float x) {
    const double d = (double)x;
    if (!(d <= 1.0 && d >= -1.0)) return dl_u2f(0x7fc00000u);   // NaN outside [-1, 1]
    return (float)dl_atan2(d, sqrt((1.0 - d) * (1.0 + d)));
}

// ---------------------------------------------------------------- conversions
// WGSL u32(f32): truncate toward zero, saturate to [0, 2^32-1], NaN -> 0.
DL_HD uint32_t dl_sat_u32(float f) {
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)f;
}

// src/spatial/radix-sort.ts:20-24 — IEEE bits mapped to an order-preserving u32.
DL_HD uint32_t dl_sortable_key(float f) {
    const uint32_t u = dl_f2u(f);
    return (u & 0x80000000u) ? ~u : (u ^ 0x80000000u);
}
