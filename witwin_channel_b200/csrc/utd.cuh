// First-order UTD wedge diffraction (device).
//
// The reference computes this in RayD (rayd/diffraction.cpp:405-455), whose
// source is not shipped.  This is the published Kouyoumjian-Pathak UTD with
// Luebbers' finite-conductivity face factors and the finite-edge rules the
// reference documents in docs/dev/audit/utd-continuity-fix-design.md (F1 vector
// field with unnormalised transverse Tx polarization, F2 1e-4 m distance
// guard, F3 receiver-angle clamp, F4 biased visibility point, F5e/F5f monotone
// truncation with the odd/even corner mend, C_BLEND = 0.35).
//
// Fresnel integrals C(x) + jS(x) (pi/2 convention) use the power series for
// |x| < 1.5 and, above, the continued fraction of erfc evaluated with the
// modified Lentz method (Press et al., Numerical Recipes, section 6.9):
//   C + jS = (1+j)/2 * (1 - erfc(z)),  z = sqrt(pi)/2 (1-j) x,
//   erfc(z) = (2z/sqrt(pi)) e^{-z^2} h,  h = 1/(b1 - 2/(b2 - 12/(b3 - ...))),
//   b_k = 1 - j pi x^2 + 4(k-1),  a_k = -(2k-1)(2k),
// which gives the complement (1+j)/2 - (C + jS) = x e^{j pi x^2/2} h without
// cancellation.
#pragma once

#include "common.cuh"
#include "em.cuh"

namespace wcb {

constexpr double kCBlend = 0.35;
constexpr double kGammaScale = 0.1;
constexpr double kWindowCutoff = 1.0e-3;
constexpr double kUtdGainFloor = 1.0e-30;
constexpr double kDiffractionRayBias = 1.0e-4;
constexpr double kUtdMinDistance = 1.0e-4;

template <typename T>
struct FresnelPair {
    Cx<T> value;       // C(x) + jS(x)
    Cx<T> complement;  // (1+j)/2 - (C(x) + jS(x))
    Cx<T> h;           // continued-fraction value (x >= 1.5), complement = x e^{j pi x^2/2} h
    bool has_h;
};

// Fresnel integrals for x >= 0.  For x >= 1.5 the complement is kept in the
// factored form x e^{j pi x^2/2} h so callers that need only its modulus or
// that cancel the exponential never evaluate e^{j pi x^2/2} at a large
// argument.  Out of line: its three call sites in the UTD (both truncation
// ends, the transition function) share one copy, which shortens the FP32
// batched field kernel by 23 % and the FP64 derivative kernels by 17-27 %.
template <typename T>
WCB_HD_OOL FresnelPair<T> fresnel_pos(T x, bool want_value = true) {
    FresnelPair<T> out;
    const Cx<T> half = cx(T(0.5), T(0.5));
    const T eps = sizeof(T) == 4 ? T(1e-7) : T(1e-15);
    if (value_of(x) < 1.5) {
        const T t = T(kPi / 2) * x * x;
        T sum_c = T(0), sum_s = T(0);
        T fact = T(1);  // t^k / k!
        for (int kk = 0; kk < 60; ++kk) {
            if (kk > 0) fact = fact * t / T(kk);
            const T term = fact * x / T(2 * kk + 1);
            const int r = kk & 3;
            if (r == 0) sum_c = sum_c + term;
            else if (r == 1) sum_s = sum_s + term;
            else if (r == 2) sum_c = sum_c - term;
            else sum_s = sum_s - term;
            if (kk > 2 && value_of(term) < value_of(eps) * (value_of(sum_c) + value_of(sum_s) + T(1e-30))) break;
        }
        out.value = cx(sum_c, sum_s);
        out.complement = half - out.value;
        out.has_h = false;
        return out;
    }
    const Cx<T> b1 = cx(T(1), -T(kPi) * x * x);
    Cx<T> b = b1;
    const T big = sizeof(T) == 4 ? T(1e30) : T(1e300);
    Cx<T> cc = cx(big, T(0));
    Cx<T> d = cx(T(1), T(0)) / b;
    Cx<T> h = d;
    for (int kk = 1; kk < 200; ++kk) {
        const T a = -T((2 * kk - 1) * (2 * kk));
        b = b + cx(T(4), T(0));
        d = cx(T(1), T(0)) / (d * a + b);
        cc = b + cx(a, T(0)) / cc;
        const Cx<T> del = cc * d;
        h = h * del;
        if (value_of(s_abs(del.re - T(1)) + s_abs(del.im)) < value_of(eps)) break;
    }
    out.h = h;
    out.has_h = true;
    if (want_value) {
        // the exponential argument is reduced in FP64 before the T-precision sincos
        double ph = kPi / 2 * double(value_of(x)) * double(value_of(x));
        ph = ph - kTwoPi * floor(ph / kTwoPi);
        const Cx<T> e = cexpj<T>(T(ph));
        out.complement = e * h * x;
        out.value = half - out.complement;
    }
    return out;
}

template <typename T>
WCB_HD FresnelPair<T> fresnel(T x) {
    if (value_of(x) >= 0) return fresnel_pos(x);
    FresnelPair<T> p = fresnel_pos(-x);
    // F(-x) = -F(x); complement(-x) = (1+j)/2 + F(x) = (1+j) - complement(x)
    FresnelPair<T> out;
    out.value = -p.value;
    out.complement = cx(T(1), T(1)) - p.complement;
    out.has_h = false;
    return out;
}

// |(1+j)/2 - (C(x) + jS(x))| for any real x.  The squared modulus equals
// f(x)^2 + g(x)^2 with the auxiliary functions f, g of Abramowitz & Stegun
// 7.3.5-7.3.6; for x >= 6 in FP32 their asymptotic series (A&S 7.3.27-7.3.28:
// pi x f ~ 1 - 3u^2 + 105u^4, pi x g ~ u - 15u^3 + 945u^5, u = 1/(pi x^2))
// is accurate to ~5e-9 relative and replaces the continued fraction.
template <typename T>
WCB_HD T fresnel_complement_abs(T x) {
    if (sizeof(T) == 4 && value_of(x) >= 6.0) {
        const T u = T(1) / (T(kPi) * x * x);
        const T u2 = u * u;
        const T pf = T(1) - T(3) * u2 + T(105) * u2 * u2;
        const T pg = u * (T(1) - T(15) * u2 + T(945) * u2 * u2);
        return s_sqrt(pf * pf + pg * pg) / (T(kPi) * x);
    }
    if (value_of(x) >= 0) {
        const FresnelPair<T> p = fresnel_pos(x, false);
        return p.has_h ? x * cabs(p.h) : cabs(p.complement);
    }
    const FresnelPair<T> p = fresnel_pos(-x);
    return cabs(cx(T(1), T(1)) - p.complement);
}

// KP transition function F(x) = 2j sqrt(x) e^{jx} int_{sqrt x}^inf e^{-j t^2} dt, x >= 0.
// With u = sqrt(2x/pi): int = sqrt(pi/2) conj(complement(u)); for u >= 1.5 the
// exponentials cancel exactly and F = 2j x conj(h(u)).
template <typename T>
WCB_HD Cx<T> transition(T x) {
    if (value_of(x) <= 0) return cx(T(0), T(0));
    if (value_of(x) >= (sizeof(T) == 4 ? 30.0 : 400.0)) {
        // large-argument expansion (Kouyoumjian & Pathak, Proc. IEEE 1974):
        // F(x) ~ 1 + j/(2x) - 3/(4x^2) - j 15/(8x^3) + 105/(16x^4) + j 945/(32x^5)
        const T r = T(1) / x;
        const T r2 = r * r;
        const T re = T(1) - T(0.75) * r2 + T(6.5625) * r2 * r2;
        const T im = T(0.5) * r - T(1.875) * r2 * r + T(29.53125) * r2 * r2 * r;
        return cx(re, im);
    }
    const T u = s_sqrt(T(2) * x / T(kPi));
    const FresnelPair<T> p = fresnel_pos(u, false);
    if (p.has_h) {
        const Cx<T> ch = cconj(p.h);
        return cx(-ch.im * T(2) * x, ch.re * T(2) * x);
    }
    const Cx<T> integral = cconj(p.complement) * T(s_sqrt(kPi / 2));
    const Cx<T> pre = cexpj<T>(x) * (T(2) * s_sqrt(x));
    return cx(T(0), T(1)) * pre * integral;
}

// One KP term cot((pi + s*beta)/(2n)) F(kL a^s(beta)) written in the distance
// eps to the term's own singular point: cot(eps/(2n)) F(2 kL sin^2(eps/2)).
template <typename T>
WCB_HD Cx<T> kp_term(T beta, T n, T kl, int s) {
    const T two_n_pi = T(2) * n * T(kPi);
    const T arg = T(kPi) + T(s) * beta;
    const T m = s_round(arg / two_n_pi);
    const T eps = arg - two_n_pi * m;
    const T small = sizeof(T) == 4 ? T(1e-5) : T(1e-9);
    const Cx<T> ej = cx(T(0.70710678118654752440), T(0.70710678118654752440));
    if (value_of(s_abs(eps)) < value_of(small)) {
        const T sg = value_of(eps) < 0 ? T(-1) : T(1);
        const Cx<T> inner = cx(sg * s_sqrt(T(kTwoPi) * kl), T(0)) - ej * (T(2) * kl * eps);
        return inner * ej * n;
    }
    const T half = eps / (T(2) * n);
    T sh, ch;
    s_sincos(half, &sh, &ch);
    const T se = s_sin(eps / T(2));
    return transition(T(2) * kl * se * se) * (ch / sh);
}

// One KP term with the odd/even corner mend of the monotone truncation
// (F5e/F5f): the term at beta and, inside the locality window of its corner
// b*, its odd part through the mirrored angle 2 b* - beta; t_mono and gamma
// weight the even and odd parts.  kl sets the window widths (4 and C_BLEND
// times sqrt(2 pi / kl)).
template <typename T>
WCB_HD Cx<T> mended_term(T beta, T nn, T kl, T t_mono, T gamma, int sgn, bool incident_group) {
    const T unit = s_sqrt(T(kTwoPi) / kl);
    const T delta_w = T(4) * unit;
    const T delta_b = T(kCBlend) * unit;
    T b_star;
    if (incident_group) {
        b_star = value_of(s_abs(beta - T(kPi))) <= value_of(s_abs(beta + T(kPi))) ? T(kPi) : T(-kPi);
    } else {
        const T other = (T(2) * nn - T(1)) * T(kPi);
        b_star = value_of(s_abs(beta - T(kPi))) <= value_of(s_abs(beta - other)) ? T(kPi) : other;
    }
    const T delta = beta - b_star;
    const T rw = delta / delta_w;
    T w = s_exp(-rw * rw);
    if (value_of(w) <= kWindowCutoff) w = T(0);
    // the term and, inside the locality window, its mirror through one
    // inlined copy of kp_term; outside the window the odd part vanishes
    Cx<T> value = cx(T(0), T(0)), mirrored = cx(T(0), T(0));
    const int nterms = value_of(w) > 0 ? 2 : 1;
#pragma unroll 1
    for (int m = 0; m < nterms; ++m) {
        const Cx<T> v = kp_term(m == 0 ? beta : T(2) * b_star - beta, nn, kl, sgn);
        if (m == 0) value = v;
        else mirrored = v;
    }
    if (nterms == 1) mirrored = value;
    const Cx<T> odd = (value - mirrored) * (T(0.5) * w);
    const T rb = delta / delta_b;
    const T wb = s_exp(-rb * rb);
    const T blend = wb + (T(1) - wb) * t_mono;
    return (value - odd) * t_mono + odd * (gamma * blend);
}

// One end's share of the finite-edge monotone factor
// t_mono = 1 - (|F(a_lo)| + |F(a_hi)|) / sqrt(2), F(x) = (1+j)/2 - (C(x) + jS(x)),
// from the end's FP64 argument x.  For x >= 0 it returns |F(x)| / sqrt(2) (at
// most 1/2, smooth in x).  For x = -u < 0 (the stationary point beyond this
// end) it returns 1 - |F(-u)| / sqrt(2): with c = F(u),
// |F(-u)|^2 = |(1+j) - c|^2 = 2 - 2 (Re c + Im c) + |c|^2, so the share is
// (2 (Re c + Im c) - |c|^2) / (sqrt(2) (sqrt(2) + |F(-u)|)), a small number
// 1 - (...) would form by cancellation.  It ripples with the phase pi u^2 / 2
// of c = u e^{j pi u^2/2} h(u), which FP32 cannot resolve at u ~ 100 (the
// FP32 argument alone moves it by 1e-2 rad), so that phase comes from the
// FP64 argument; h (smooth) is the T-precision continued fraction.
template <typename T>
WCB_HD T fresnel_end_share(double x) {
    const T inv_sqrt2 = T(0.70710678118654752440);
    if (x >= 0.0) return fresnel_complement_abs(T(x)) * inv_sqrt2;
    const double u = -x;
    const FresnelPair<T> p = fresnel_pos(T(u), false);
    Cx<T> c;
    if (p.has_h) {
        double ph = kPi / 2 * u * u;
        ph = ph - kTwoPi * floor(ph / kTwoPi);
        c = cexpj<T>(T(ph)) * p.h * T(u);
    } else {
        c = p.complement;
    }
    const T f = cabs(cx(T(1), T(1)) - c);
    const T sqrt2 = T(1.41421356237309504880);
    return (T(2) * (c.re + c.im) - cabs2(c)) / (sqrt2 * (sqrt2 + f));
}

// Selected diffraction edge (device layout, FP64 geometry).
struct EdgeDev {
    double pos[3];     // midpoint
    double dir[3];     // unit edge direction of the record (v0 -> v1)
    double t0[3];      // unit face-0 tangent normalize(n0 x dir)
    double n0[3];      // ordered outward normal of face 0
    double n1[3];      // ordered outward normal of face n
    double half_length;
    double n;          // exterior angle / pi
    double bisector[3];  // unit exterior bisector used for the visibility bias
    int face0, face1;    // reference face ids (visibility ignore set)
    int mat_face0, mat_face1;  // faces whose material gives R_0 and R_n
    int edge_id;         // reference edge id
    int face_n;          // 1: a second face bounds the wedge; 0: half-plane, R_n = 0
};

template <typename T>
WCB_HD T wedge_angle(V3<T> d, V3<T> t0, V3<T> n0) {
    T a = s_atan2(dot(d, n0), dot(d, t0));
    if (value_of(a) < 0) a = a + T(kTwoPi);
    return a;
}

template <typename T>
struct DiffractionResult {
    bool valid;        // source outside the wedge
    C3<T> field;       // unit-excitation field at the receiver (phase included)
    double q[3];       // unclamped stationary point (FP64)
    double q_vis[3];   // clamped + biased visibility point
    double length;     // s' + s (FP64)
};

// Edge frame in geometry type G (double in the solve, a dual number in the
// derivative kernels).
template <typename G>
struct EdgeFrame {
    V3<G> c, e, t0, n0, bisector;
    G half_length, n;
    bool face_n;  // false for a half-plane: its second face is absent (R_n = 0)
};

WCB_HD EdgeFrame<double> edge_frame(const EdgeDev& ed) {
    EdgeFrame<double> f;
    f.c = v3(ed.pos[0], ed.pos[1], ed.pos[2]);
    f.e = v3(ed.dir[0], ed.dir[1], ed.dir[2]);
    f.t0 = v3(ed.t0[0], ed.t0[1], ed.t0[2]);
    f.n0 = v3(ed.n0[0], ed.n0[1], ed.n0[2]);
    f.bisector = v3(ed.bisector[0], ed.bisector[1], ed.bisector[2]);
    f.half_length = ed.half_length;
    f.n = ed.n;
    f.face_n = ed.face_n != 0;
    return f;
}

// exp(-j k d) in the amplitude type T from geometry-typed k and d.
template <typename T>
WCB_HD Cx<T> phasor_kd(double k, double d) { return phasor_neg_kd<T>(k, d); }

// The frequency-independent part of one (source, receiver, edge) UTD
// evaluation: the Keller stationary point, lengths, wedge angles, the
// ray-fixed bases, the transmit polarisation on them and the spreading
// factor.  A caller evaluating several frequencies forms it once.
template <typename G, typename T>
struct UtdGeometry {
    bool valid;        // source outside the wedge
    bool on_face_n;    // receiver inside the wedge, its angle clamped onto face n
    V3<G> q;           // unclamped stationary point
    double q_vis[3];   // clamped + biased visibility point
    G s_p, s;          // incident and diffracted lengths (floored)
    G t_star;          // stationary parameter along the edge
    double kappa64;    // FP64 truncation curvature sin_b^2 (1/s' + 1/s) (FP32 end arguments)
    T phi_p, phi, nn, npi, sin_b, sT, spT, kappa, tsT;
    V3<T> beta_hat, phi_hat;
    T e_beta0, e_phi0;  // transmit polarisation on the incident bases (before 1/(2 k s'))
    T spread;
};

template <typename G, typename T>
WCB_HD UtdGeometry<G, T> utd_geometry(const EdgeFrame<G>& ed, V3<G> S, V3<G> R, V3<T> tx_pol) {
    UtdGeometry<G, T> g;
    g.valid = false;
    g.on_face_n = false;
    const V3<G> c = ed.c;
    const V3<G> e = ed.e;
    // Keller stationary point (unfolding)
    const V3<G> ds = S - c;
    const G ts = dot(ds, e);
    const V3<G> ps = ds - e * ts;
    const G rs = length(ps);
    const V3<G> dr = R - c;
    const G tr = dot(dr, e);
    const V3<G> pr = dr - e * tr;
    const G rr = length(pr);
    const G t_star = value_of(rs + rr) > 0.0 ? ts + (tr - ts) * rs / (rs + rr) : ts;
    const V3<G> q = c + e * t_star;
    g.q = q;
    g.t_star = t_star;
    const G tc = s_min(s_max(t_star, -ed.half_length), ed.half_length);
    const V3<G> qv = c + e * tc + ed.bisector * G(kDiffractionRayBias);
    g.q_vis[0] = value_of(qv.x); g.q_vis[1] = value_of(qv.y); g.q_vis[2] = value_of(qv.z);
    const V3<G> sp_vec = q - S;
    const V3<G> s_vec = R - q;
    const G s_p = s_max(length(sp_vec), G(kUtdMinDistance));
    const G s = s_max(length(s_vec), G(kUtdMinDistance));
    g.s_p = s_p;
    g.s = s;
    // angles in the edge frame
    const T phi_p = wedge_angle(cast3<T>(ps), cast3<T>(ed.t0), cast3<T>(ed.n0));
    T phi = wedge_angle(cast3<T>(pr), cast3<T>(ed.t0), cast3<T>(ed.n0));
    const T nn = T(ed.n);
    const T npi = nn * T(kPi);
    g.nn = nn;
    g.npi = npi;
    g.phi_p = phi_p;
    if (value_of(phi_p) > value_of(npi)) return g;
    if (value_of(phi) > value_of(npi)) {
        g.on_face_n = value_of(phi - npi) < value_of(T(kTwoPi) - phi);
        phi = g.on_face_n ? npi : T(0);
    }
    g.phi = phi;
    g.valid = true;
    const V3<T> sh_p = cast3<T>(sp_vec * (G(1) / s_p));
    const V3<T> sh = cast3<T>(s_vec * (G(1) / s));
    const V3<T> ef = cast3<T>(e);
    T cos_b = dot(sh_p, ef);
    cos_b = s_min(s_max(cos_b, T(-1)), T(1));
    const T sin_b = s_max(s_sqrt(s_max(T(1) - cos_b * cos_b, T(0))), T(1e-6));
    const T sT = T(s), spT = T(s_p);
    g.sin_b = sin_b;
    g.sT = sT;
    g.spT = spT;
    // finite-edge truncation curvature
    const T rho_p = spT * sin_b;
    const T rho = sT * sin_b;
    g.kappa = rho_p * rho_p / (spT * spT * spT) + rho * rho / (sT * sT * sT);
    g.tsT = T(t_star);
    g.kappa64 = 0.0;
    if constexpr (sizeof(T) == 4) {
        const double cb64 = fmin(fmax(value_of(dot(sp_vec, e)) / value_of(s_p), -1.0), 1.0);
        const double sb64 = fmax(sqrt(fmax(1.0 - cb64 * cb64, 0.0)), 1e-6);
        g.kappa64 = sb64 * sb64 / value_of(s_p) + sb64 * sb64 / value_of(s);
    }
    // ray-fixed bases
    V3<T> phi_hat_p = cross(ef, sh_p);
    phi_hat_p = phi_hat_p * (T(1) / s_max(length(phi_hat_p), T(1e-12)));
    const V3<T> beta_hat_p = cross(sh_p, phi_hat_p);
    V3<T> phi_hat = cross(ef, sh);
    phi_hat = phi_hat * (T(1) / s_max(length(phi_hat), T(1e-12)));
    g.beta_hat = cross(sh, phi_hat);
    g.phi_hat = phi_hat;
    const V3<T> tx_axis = transverse(sh_p, tx_pol);
    g.e_beta0 = dot(tx_axis, beta_hat_p);
    g.e_phi0 = dot(tx_axis, phi_hat_p);
    g.spread = s_sqrt(spT / (sT * (spT + sT)));
    return g;
}

// The UTD field of a valid geometry at one frequency: unit-excitation field
// at the receiver (phase included).  The face slabs give R_0 and R_n.
template <typename G, typename T>
WCB_HD C3<T> utd_field_at(const UtdGeometry<G, T>& g, const EdgeFrame<G>& ed, const Slab<T>& m0, const Slab<T>& mn,
                          G frequency) {
    const G k = G(kTwoPi) * frequency / G(kC0);
    const T phi_p = g.phi_p, phi = g.phi, nn = g.nn, npi = g.npi, sin_b = g.sin_b, sT = g.sT, spT = g.spT;
    const T kT = T(k);
    const T kl = kT * sT * spT * sin_b * sin_b / (sT + spT);
    const T sigma = s_sqrt(kT * g.kappa / T(kPi));
    const T tsT = g.tsT;
    const T tmax = T(ed.half_length), tmin = -T(ed.half_length);
    const T inv_sqrt2 = T(0.70710678118654752440);
    T t_mono;
    if constexpr (sizeof(T) == 4) {
        // both ends through one inlined copy, from their FP64 arguments (FP64
        // geometry); the end the stationary point lies beyond contributes
        // 1 - |F|/sqrt(2), so a tail factor is a difference of two small
        // numbers instead of a small residue of O(1) ones
        const double sigma64 = sqrt(value_of(k) * g.kappa64 / kPi);
        const double hl64 = value_of(ed.half_length), ts64 = value_of(g.t_star);
        const double a_hi = sigma64 * (hl64 - ts64), a_lo = sigma64 * (hl64 + ts64);
        T share_hi = T(0), share_lo = T(0);
#pragma unroll 1
        for (int e2 = 0; e2 < 2; ++e2) {
            const T v = fresnel_end_share<T>(e2 == 0 ? a_hi : a_lo);
            if (e2 == 0) share_hi = v;
            else share_lo = v;
        }
        const bool beyond_hi = a_hi < 0.0, beyond_lo = a_lo < 0.0;
        T tm;
        if (beyond_hi && beyond_lo) tm = share_hi + share_lo - T(1);
        else if (beyond_hi) tm = share_hi - share_lo;
        else if (beyond_lo) tm = share_lo - share_hi;
        else tm = T(1) - share_hi - share_lo;
        t_mono = s_min(s_max(tm, T(0)), T(1));
    } else {
        // both ends through one inlined copy of the Fresnel complement
        T hi_abs = T(0), lo_abs = T(0);
#pragma unroll 1
        for (int e2 = 0; e2 < 2; ++e2) {
            const T v = fresnel_complement_abs(e2 == 0 ? sigma * (tmax - tsT) : -(sigma * (tmin - tsT)));
            if (e2 == 0) hi_abs = v;
            else lo_abs = v;
        }
        t_mono = s_min(s_max(T(1) - inv_sqrt2 * lo_abs - inv_sqrt2 * hi_abs, T(0)), T(1));
    }
    T u;
    if (value_of(s_abs(tsT - tmax)) < value_of(s_abs(tsT - tmin))) u = sigma * (tsT - tmax);
    else u = sigma * (tmin - tsT);
    const T gamma = T(1) / (T(1) + s_exp(s_min(u / T(kGammaScale), T(80))));
    // face factors: interface (half-space) Fresnel at the wedge angles; a
    // half-plane's absent second face reflects nothing
    // (FP32 forms 1 + R without cancellation near grazing and takes R from it)
    Cx<T> r0_te, r0_tm, rn_te = cx(T(0), T(0)), rn_tm = cx(T(0), T(0));  // faces 0 and n, one inlined copy
    Cx<T> p0_te = cx(T(1), T(0)), p0_tm = p0_te, pn_te = p0_te, pn_tm = p0_te;  // 1 + R (FP32)
    const int faces = ed.face_n ? 2 : 1;
#pragma unroll 1
    for (int face = 0; face < faces; ++face) {
        Cx<T> te, tm;
        const T sin_face = s_sin(face == 0 ? phi_p : npi - phi);
        if constexpr (sizeof(T) == 4) {
            halfspace_fresnel_one_plus(sin_face, face == 0 ? m0 : mn, frequency, &te, &tm);
            if (face == 0) {
                p0_te = te;
                p0_tm = tm;
            } else {
                pn_te = te;
                pn_tm = tm;
            }
            te = te - cx(T(1), T(0));
            tm = tm - cx(T(1), T(0));
        } else {
            halfspace_fresnel(sin_face, face == 0 ? m0 : mn, frequency, &te, &tm);
        }
        if (face == 0) {
            r0_te = te;
            r0_tm = tm;
        } else {
            rn_te = te;
            rn_tm = tm;
        }
    }
    const T bm = phi - phi_p;
    const T bp = phi + phi_p;
    // FP32 with the receiver angle clamped onto face n (phi = n pi): there the
    // KP arguments of the (beta-, +) and (beta+, -) terms, and of the (beta-, -)
    // and (beta+, +) terms, differ by 2 n pi and their corner mends pair up,
    // so the sums are (1 + R_0) T0 + (1 + R_n) T1.  R_n sits at grazing
    // incidence (-1 + 1e-6) and R_0 at grazing too when the source lies near
    // face 0's plane: the direct sums are residues FP32 cannot form by
    // cancellation (cot near zero differs between the paired terms in the last
    // bits).  The paired form with 1 + R formed directly has no cancellation.
    bool merge_n = false;
    if constexpr (sizeof(T) == 4) merge_n = g.on_face_n && ed.face_n && value_of(phi_p) > 0;
    // the four KP terms: (beta-, +), (beta-, -) incident; (beta+, +) weighted by
    // R_n, (beta+, -) weighted by R_0.  One loop body (not four inlined
    // copies) keeps the kernel's instruction footprint small.
    Cx<T> sum_soft = cx(T(0), T(0)), sum_hard = cx(T(0), T(0));
    Cx<T> t0v = cx(T(0), T(0)), t1v = cx(T(0), T(0));
    const int nterms = merge_n ? 2 : 4;
#pragma unroll 1
    for (int q = 0; q < nterms; ++q) {
        const bool incident = q < 2;
        const Cx<T> term = mended_term(incident ? bm : bp, nn, kl, t_mono, gamma, (q & 1) ? -1 : +1, incident);
        if (merge_n) {
            if (q == 0) t0v = term;
            else t1v = term;
            continue;
        }
        const Cx<T> one = cx(T(1), T(0));
        const Cx<T> w_soft = incident ? one : (q == 2 ? rn_te : r0_te);
        const Cx<T> w_hard = incident ? one : (q == 2 ? rn_tm : r0_tm);
        sum_soft = sum_soft + w_soft * term;
        sum_hard = sum_hard + w_hard * term;
    }
    if (merge_n) {
        sum_soft = p0_te * t0v + pn_te * t1v;
        sum_hard = p0_tm * t0v + pn_tm * t1v;
    }
    // pre = -exp(-j pi/4) / (2 n sqrt(2 pi k) sin_b)
    const T pre_mag = T(1) / (T(2) * nn * s_sqrt(T(kTwoPi) * kT) * sin_b);
    const Cx<T> pre = cx(-inv_sqrt2 * pre_mag, inv_sqrt2 * pre_mag);
    const Cx<T> d_soft = pre * sum_soft;
    const Cx<T> d_hard = pre * sum_hard;
    const T inc_amp = T(1) / (T(2) * kT * spT);
    const T e_beta = g.e_beta0 * inc_amp;
    const T e_phi = g.e_phi0 * inc_amp;
    const Cx<T> ph = phasor_kd<T>(k, g.s_p + g.s);
    const Cx<T> cb = -(d_soft * (e_beta * g.spread)) * ph;
    const Cx<T> cf = -(d_hard * (e_phi * g.spread)) * ph;
    return c3_axis(g.beta_hat, cb) + c3_axis(g.phi_hat, cf);
}

// DiffractionResult of a geometry at one frequency (field zero when invalid).
template <typename G, typename T>
WCB_HD DiffractionResult<T> utd_result(const UtdGeometry<G, T>& g, const EdgeFrame<G>& ed, const Slab<T>& m0,
                                       const Slab<T>& mn, G frequency, V3<G>* q_out = nullptr) {
    DiffractionResult<T> out;
    out.valid = g.valid;
    if (q_out) *q_out = g.q;
    out.q[0] = value_of(g.q.x); out.q[1] = value_of(g.q.y); out.q[2] = value_of(g.q.z);
    for (int k = 0; k < 3; ++k) out.q_vis[k] = g.q_vis[k];
    out.length = value_of(g.s_p + g.s);
    if (g.valid) out.field = utd_field_at(g, ed, m0, mn, frequency);
    else out.field = C3<T>{cx(T(0), T(0)), cx(T(0), T(0)), cx(T(0), T(0))};
    return out;
}

// UTD field of one edge: geometry (stationary point, lengths, phase) in G,
// amplitudes in T.  The face slabs give R_0 and R_n.
template <typename G, typename T>
WCB_HD DiffractionResult<T> utd_field_gt(const EdgeFrame<G>& ed, V3<G> S, V3<G> R, V3<T> tx_pol, const Slab<T>& m0,
                                         const Slab<T>& mn, G frequency, V3<G>* q_out = nullptr) {
    const UtdGeometry<G, T> g = utd_geometry<G, T>(ed, S, R, tx_pol);
    return utd_result(g, ed, m0, mn, frequency, q_out);
}

// The solve's form: FP64 geometry from the precomputed edge record.
template <typename T>
WCB_HD DiffractionResult<T> utd_field(const EdgeDev& ed, V3<double> S, V3<double> R, V3<T> tx_pol, const Slab<T>& m0,
                                      const Slab<T>& mn, double frequency) {
    return utd_field_gt<double, T>(edge_frame(ed), S, R, tx_pol, m0, mn, frequency);
}

}  // namespace wcb
