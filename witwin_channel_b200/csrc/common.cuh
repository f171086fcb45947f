// Shared device math: templated 3-vectors and complex numbers.
//
// Every field/geometry routine is written once over a scalar type T so the
// same source serves the mixed-precision path (T = float), the plain FP64
// path (T = double) and the fixed-topology derivative kernels (T = Dual).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define WCB_HD __host__ __device__ __forceinline__
#define WCB_D __device__ __forceinline__
// out of line (one copy per translation unit): a helper with several call
// sites in the special-function-heavy kernels, whose inlined copies would
// overflow the instruction cache
#define WCB_HD_OOL __host__ __device__ __noinline__

namespace wcb {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kTwoPi = 6.283185307179586476925286766559005768;
constexpr double kC0 = 299792458.0;
constexpr double kEps0 = 8.8541878128e-12;
constexpr double kMu0 = 1.25663706212e-6;
constexpr double kUtdEps = 1.0e-10;       // field kernels' length floor
constexpr double kUtdSmallEps = 1.0e-6;   // field kernels' normalisation floor

// ---------------------------------------------------------------- scalars
// Out-of-line copies of the longer math-library routines.  Every call site of
// sin, cos, sincos, exp (FP64), atan2, acos or hypot would otherwise inline
// the whole routine, and the special-function-heavy kernels (the UTD and its
// dual-number derivative) then no longer fit the instruction cache; a call
// site now branches to the one copy its translation unit holds.  Device code
// only; the values are the library's own.
#ifdef __CUDA_ARCH__
namespace ool {
struct SinCosD { double s, c; };
struct SinCosF { float s, c; };
__device__ __noinline__ inline double sin_d(double x) { return ::sin(x); }
__device__ __noinline__ inline double cos_d(double x) { return ::cos(x); }
__device__ __noinline__ inline SinCosD sincos_d(double x) {
    SinCosD r;
    ::sincos(x, &r.s, &r.c);
    return r;
}
__device__ __noinline__ inline double exp_d(double x) { return ::exp(x); }
__device__ __noinline__ inline double atan2_d(double y, double x) { return ::atan2(y, x); }
__device__ __noinline__ inline double acos_d(double x) { return ::acos(x); }
__device__ __noinline__ inline double hypot_d(double a, double b) { return ::hypot(a, b); }
__device__ __noinline__ inline float sin_f(float x) { return ::sinf(x); }
__device__ __noinline__ inline float cos_f(float x) { return ::cosf(x); }
__device__ __noinline__ inline SinCosF sincos_f(float x) {
    SinCosF r;
    ::sincosf(x, &r.s, &r.c);
    return r;
}
__device__ __noinline__ inline float atan2_f(float y, float x) { return ::atan2f(y, x); }
}  // namespace ool
#define WCB_MATH(dev, host) dev
#else
#define WCB_MATH(dev, host) host
#endif
WCB_HD float s_sqrt(float x) { return sqrtf(x); }
WCB_HD double s_sqrt(double x) { return sqrt(x); }
WCB_HD float s_abs(float x) { return fabsf(x); }
WCB_HD double s_abs(double x) { return fabs(x); }
WCB_HD float s_max(float a, float b) { return fmaxf(a, b); }
WCB_HD double s_max(double a, double b) { return fmax(a, b); }
WCB_HD float s_min(float a, float b) { return fminf(a, b); }
WCB_HD double s_min(double a, double b) { return fmin(a, b); }
WCB_HD float s_exp(float x) { return expf(x); }
WCB_HD double s_exp(double x) { return WCB_MATH(ool::exp_d(x), exp(x)); }
WCB_HD float s_cos(float x) { return WCB_MATH(ool::cos_f(x), cosf(x)); }
WCB_HD double s_cos(double x) { return WCB_MATH(ool::cos_d(x), cos(x)); }
WCB_HD float s_sin(float x) { return WCB_MATH(ool::sin_f(x), sinf(x)); }
WCB_HD double s_sin(double x) { return WCB_MATH(ool::sin_d(x), sin(x)); }
WCB_HD float s_atan2(float y, float x) { return WCB_MATH(ool::atan2_f(y, x), atan2f(y, x)); }
WCB_HD double s_atan2(double y, double x) { return WCB_MATH(ool::atan2_d(y, x), atan2(y, x)); }
WCB_HD float s_hypot(float a, float b) { return hypotf(a, b); }
WCB_HD double s_hypot(double a, double b) { return WCB_MATH(ool::hypot_d(a, b), hypot(a, b)); }
WCB_HD double s_acos(double a) { return WCB_MATH(ool::acos_d(fmin(fmax(a, -1.0), 1.0)), acos(fmin(fmax(a, -1.0), 1.0))); }
WCB_HD float s_floor(float x) { return floorf(x); }
WCB_HD double s_floor(double x) { return floor(x); }
WCB_HD float s_round(float x) { return rintf(x); }
WCB_HD double s_round(double x) { return rint(x); }
WCB_HD double value_of(double x) { return x; }
WCB_HD float value_of(float x) { return x; }
WCB_HD void s_sincos(float x, float* s, float* c) {
#ifdef __CUDA_ARCH__
    const ool::SinCosF r = ool::sincos_f(x);
    *s = r.s;
    *c = r.c;
#else
    *s = sinf(x); *c = cosf(x);
#endif
}
WCB_HD void s_sincos(double x, double* s, double* c) {
#ifdef __CUDA_ARCH__
    const ool::SinCosD r = ool::sincos_d(x);
    *s = r.s;
    *c = r.c;
#else
    *s = sin(x); *c = cos(x);
#endif
}

// ---------------------------------------------------------------- vectors
template <typename T>
struct V3 {
    T x, y, z;
};

template <typename T>
WCB_HD V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T>
WCB_HD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
WCB_HD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T>
WCB_HD V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <typename T, typename S>
WCB_HD V3<T> operator*(V3<T> a, S s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T>
WCB_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
WCB_HD V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T>
WCB_HD T length(V3<T> a) { return s_sqrt(dot(a, a)); }

template <typename T, typename S>
WCB_HD V3<T> cast3(V3<S> a) { return {T(a.x), T(a.y), T(a.z)}; }

// normalize with the field kernels' rule: |v| > 1e-6 ? v/(|v|+1e-10) : fallback/(|fb|+1e-10)
template <typename T>
WCB_HD V3<T> safe_normalize(V3<T> v, V3<T> fallback) {
    T n = length(v);
    if (value_of(n) > kUtdSmallEps) {
        return v * (T(1) / (n + T(kUtdEps)));
    }
    T fn = length(fallback);
    return fallback * (T(1) / (fn + T(kUtdEps)));
}

template <typename T>
WCB_HD V3<T> transverse(V3<T> dir, V3<T> p) { return p - dir * dot(p, dir); }

template <typename T>
WCB_HD V3<T> stable_perp_basis(V3<T> dir, V3<T> preferred) {
    V3<T> proj = preferred - dir * dot(preferred, dir);
    V3<T> alt = s_abs(value_of(dir.z)) < 0.9 ? v3<T>(T(0), T(0), T(1)) : v3<T>(T(0), T(1), T(0));
    V3<T> alt_proj = alt - dir * dot(alt, dir);
    return safe_normalize(proj, alt_proj);
}

// ---------------------------------------------------------------- complex
template <typename T>
struct Cx {
    T re, im;
};
template <typename T>
WCB_HD Cx<T> cx(T re, T im) { return Cx<T>{re, im}; }
template <typename T>
WCB_HD Cx<T> operator+(Cx<T> a, Cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
WCB_HD Cx<T> operator-(Cx<T> a, Cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
WCB_HD Cx<T> operator-(Cx<T> a) { return {-a.re, -a.im}; }
template <typename T>
WCB_HD Cx<T> operator*(Cx<T> a, Cx<T> b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
template <typename T>
WCB_HD Cx<T> operator*(Cx<T> a, T s) { return {a.re * s, a.im * s}; }
template <typename T>
WCB_HD Cx<T> operator*(T s, Cx<T> a) { return {a.re * s, a.im * s}; }
template <typename T>
WCB_HD Cx<T> cconj(Cx<T> a) { return {a.re, -a.im}; }
template <typename T>
WCB_HD T cabs2(Cx<T> a) { return a.re * a.re + a.im * a.im; }
template <typename T>
WCB_HD T cabs(Cx<T> a) { return s_hypot(a.re, a.im); }
template <typename T>
WCB_HD Cx<T> operator/(Cx<T> a, Cx<T> b) {
    // scaled division (Smith) keeps the wide dynamic range of slab terms
    if (s_abs(value_of(b.re)) >= s_abs(value_of(b.im))) {
        T r = b.im / b.re;
        T den = b.re + b.im * r;
        return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    }
    T r = b.re / b.im;
    T den = b.re * r + b.im;
    return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
// principal square root (branch cut on the negative real axis).  The
// component computed from (|z| +- Re z)/2 is the one without cancellation;
// the other follows from Im z = 2 Re(w) Im(w).
template <typename T>
WCB_HD Cx<T> csqrt(Cx<T> z) {
    const T m = cabs(z);
    if (value_of(m) == 0) return {T(0), T(0)};
    if (value_of(z.re) >= 0) {
        const T re = s_sqrt(T(0.5) * (m + z.re));
        return {re, z.im / (T(2) * re)};
    }
    T im = s_sqrt(T(0.5) * (m - z.re));
    if (value_of(z.im) < 0) im = -im;
    return {z.im / (T(2) * im), im};
}
template <typename T>
WCB_HD Cx<T> cexp(Cx<T> z) {
    T e = s_exp(z.re);
    T s, c;
    s_sincos(z.im, &s, &c);
    return {e * c, e * s};
}
// exp(j*phase)
template <typename T>
WCB_HD Cx<T> cexpj(T phase) {
    T s, c;
    s_sincos(phase, &s, &c);
    return {c, s};
}

template <typename T>
struct C3 {
    Cx<T> x, y, z;
};
template <typename T>
WCB_HD C3<T> c3_from_real(V3<T> v) { return {cx(v.x, T(0)), cx(v.y, T(0)), cx(v.z, T(0))}; }
template <typename T>
WCB_HD C3<T> operator+(C3<T> a, C3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
WCB_HD C3<T> c3_scale(C3<T> a, Cx<T> s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T>
WCB_HD C3<T> c3_axis(V3<T> axis, Cx<T> s) { return {s * axis.x, s * axis.y, s * axis.z}; }
template <typename T>
WCB_HD Cx<T> c3_dot(C3<T> a, V3<T> v) {
    return {a.x.re * v.x + a.y.re * v.y + a.z.re * v.z, a.x.im * v.x + a.y.im * v.y + a.z.im * v.z};
}
template <typename T>
WCB_HD T c3_power(C3<T> a) { return cabs2(a.x) + cabs2(a.y) + cabs2(a.z); }

// FP64 phase reduction: exp(-j*k*d) with k and d in double, reduced mod 2*pi
// before the (T-precision) sincos.
template <typename T>
WCB_HD Cx<T> phasor_neg_kd(double k, double d) {
    double ph = k * d;
    ph = ph - kTwoPi * floor(ph / kTwoPi);
    return cexpj<T>(T(-ph));
}

}  // namespace wcb
