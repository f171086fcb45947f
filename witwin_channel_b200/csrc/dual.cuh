// Forward-mode dual numbers over FP64 for the fixed-topology derivative
// kernels: a value and N tangent components, propagated through the same
// templated field/geometry routines the forward solve uses (they call the
// s_* scalar functions and value_of, overloaded here).  Branches in those
// routines test value_of(), so a dual evaluation follows the forward
// evaluation's branch structure and differentiates the branch taken.
#pragma once

#include "common.cuh"

namespace wcb {

template <int N>
struct Dual {
    double v;
    double d[N];

    WCB_HD Dual() : v(0.0) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    WCB_HD Dual(double x) : v(x) {  // NOLINT: constants promote implicitly
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
};

// N = 0: no tangent lane, a plain FP64 evaluation of the same templated code
// (the tangent loops run zero times; the one-element array is never read).
template <>
struct Dual<0> {
    double v;
    double d[1];

    WCB_HD Dual() : v(0.0), d{0.0} {}
    WCB_HD Dual(double x) : v(x), d{0.0} {}  // NOLINT: constants promote implicitly
};

template <typename T>
struct is_dual {
    static constexpr bool value = false;
};
template <int N>
struct is_dual<Dual<N>> {
    static constexpr bool value = true;
};

template <int N>
WCB_HD double value_of(const Dual<N>& a) { return a.v; }

// chain rule: f(a) with f'(a) = g
template <int N>
WCB_HD Dual<N> chain(double f, double g, const Dual<N>& a) {
    Dual<N> r;
    r.v = f;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = g * a.d[i];
    return r;
}

template <int N>
WCB_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
WCB_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
WCB_HD Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
WCB_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
WCB_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    const double inv = 1.0 / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N>
WCB_HD Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
WCB_HD Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
WCB_HD Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
WCB_HD Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
WCB_HD Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N>
WCB_HD Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
WCB_HD Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N>
WCB_HD Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N>
WCB_HD bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N>
WCB_HD bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }

template <int N>
WCB_HD Dual<N> s_sqrt(const Dual<N>& a) {
    const double r = sqrt(a.v);
    return chain(r, r > 0.0 ? 0.5 / r : 0.0, a);
}
template <int N>
WCB_HD Dual<N> s_abs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
template <int N>
WCB_HD Dual<N> s_max(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v ? a : b; }
template <int N>
WCB_HD Dual<N> s_min(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v ? a : b; }
template <int N>
WCB_HD Dual<N> s_max(const Dual<N>& a, double b) { return a.v >= b ? a : Dual<N>(b); }
template <int N>
WCB_HD Dual<N> s_min(const Dual<N>& a, double b) { return a.v <= b ? a : Dual<N>(b); }
template <int N>
WCB_HD Dual<N> s_exp(const Dual<N>& a) {
    const double e = s_exp(a.v);
    return chain(e, e, a);
}
template <int N>
WCB_HD Dual<N> s_cos(const Dual<N>& a) {
    double sv, cv;
    s_sincos(a.v, &sv, &cv);
    return chain(cv, -sv, a);
}
template <int N>
WCB_HD Dual<N> s_sin(const Dual<N>& a) {
    double sv, cv;
    s_sincos(a.v, &sv, &cv);
    return chain(sv, cv, a);
}
template <int N>
WCB_HD void s_sincos(const Dual<N>& a, Dual<N>* s, Dual<N>* c) {
    double sv, cv;
    s_sincos(a.v, &sv, &cv);
    *s = chain(sv, cv, a);
    *c = chain(cv, -sv, a);
}
template <int N>
WCB_HD Dual<N> s_atan2(const Dual<N>& y, const Dual<N>& x) {
    Dual<N> r;
    r.v = s_atan2(y.v, x.v);
    const double den = x.v * x.v + y.v * y.v;
    const double gx = den > 0.0 ? -y.v / den : 0.0;
    const double gy = den > 0.0 ? x.v / den : 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = gy * y.d[i] + gx * x.d[i];
    return r;
}
template <int N>
WCB_HD Dual<N> s_hypot(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = s_hypot(a.v, b.v);
    const double ga = r.v > 0.0 ? a.v / r.v : 0.0;
    const double gb = r.v > 0.0 ? b.v / r.v : 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = ga * a.d[i] + gb * b.d[i];
    return r;
}
// piecewise-constant maps: zero derivative
template <int N>
WCB_HD Dual<N> s_floor(const Dual<N>& a) { return Dual<N>(floor(a.v)); }
template <int N>
WCB_HD Dual<N> s_round(const Dual<N>& a) { return Dual<N>(rint(a.v)); }
template <int N>
WCB_HD Dual<N> s_acos(const Dual<N>& a) {
    const double x = fmin(fmax(a.v, -1.0), 1.0);
    const double den = sqrt(fmax(1.0 - x * x, 0.0));
    return chain(s_acos(x), (den > 0.0 && fabs(a.v) < 1.0) ? -1.0 / den : 0.0, a);
}

// exp(-j k d) with the product reduced mod 2*pi on the value (a constant
// shift, so the tangents are those of -k*d).
template <int N>
WCB_HD Cx<Dual<N>> phasor_neg_kd(const Dual<N>& k, const Dual<N>& d) {
    Dual<N> ph = k * d;
    ph.v = ph.v - kTwoPi * floor(ph.v / kTwoPi);
    return cexpj<Dual<N>>(-ph);
}

}  // namespace wcb
