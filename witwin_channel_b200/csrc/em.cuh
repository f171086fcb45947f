// Field transport: free space, thin-slab Fresnel, specular Jones chain and
// the Rouard thin-sheet stack.
//
// Restates the reference's field kernels: free space (fields.cu:36-82),
// receiver projection (fields.cu:84-105), the reflection sequence
// (fields.cu:113-204) whose per-bounce algebra the reference keeps in RayD's
// field_transport and mirrors in tests/ad/_reference_fields.py:85-186, and the
// straight thin-sheet chain (_reference_fields.py:196-337).
#pragma once

#include "common.cuh"

namespace wcb {

// Per-face slab parameters (first physical layer of the material).
template <typename T>
struct Slab {
    T eps_r, sigma_e, mu_r, gain, thickness;
};

// Thin-slab Fabry-Perot reflection r_te, r_tm (_reference_fields.py:85-115).
// F is the frequency's type: double in the solve, a dual number in the
// derivative kernels.
template <typename T, typename F = double>
WCB_HD void slab_fresnel(T cos_theta, const Slab<T>& m, F frequency, T wavelength, Cx<T>* r_te, Cx<T>* r_tm) {
    const T omega = T(s_max(kTwoPi * frequency, kUtdSmallEps));
    T ct = s_abs(cos_theta);
    ct = s_min(s_max(ct, T(kUtdSmallEps)), T(1));
    const T sin2 = s_max(T(1) - ct * ct, T(0));
    const Cx<T> eta = cx(s_max(m.eps_r, T(kUtdSmallEps)), -s_max(m.sigma_e, T(0)) / (omega * T(kEps0)));
    const T mu = s_max(m.mu_r, T(kUtdSmallEps));
    const Cx<T> root = csqrt(eta * mu - cx(sin2, T(0)));
    const Cx<T> mu_ct = cx(mu * ct, T(0));
    const Cx<T> eta_ct = eta * ct;
    const Cx<T> i_te = (mu_ct - root) / (mu_ct + root);
    const Cx<T> i_tm = (eta_ct - root) / (eta_ct + root);
    const T scale = T(kTwoPi) * s_max(m.thickness, T(0)) / s_max(wavelength, T(kUtdSmallEps));
    const Cx<T> q = root * scale;
    // exp(-2j q) = exp(2 Im q) * exp(-2j Re q)
    const Cx<T> phase = cexp(cx(T(2) * q.im, T(-2) * q.re));
    const Cx<T> one = cx(T(1), T(0));
    *r_te = ((i_te * (one - phase)) / (one - i_te * i_te * phase)) * m.gain;
    *r_tm = ((i_tm * (one - phase)) / (one - i_tm * i_tm * phase)) * m.gain;
}

// Interface (half-space) Fresnel coefficients gain * (r_te, r_tm): the slab law
// above without its Fabry-Perot layer term.  The wedge faces of first-order
// diffraction take this form at the wedge angles (the reference's design
// notes, docs/dev/plans/07-channel-native-differentiable-solver-plan.md:57).
template <typename T, typename F = double>
WCB_HD void halfspace_fresnel(T cos_theta, const Slab<T>& m, F frequency, Cx<T>* r_te, Cx<T>* r_tm) {
    const T omega = T(s_max(kTwoPi * frequency, kUtdSmallEps));
    T ct = s_abs(cos_theta);
    ct = s_min(s_max(ct, T(kUtdSmallEps)), T(1));
    const T sin2 = s_max(T(1) - ct * ct, T(0));
    const Cx<T> eta = cx(s_max(m.eps_r, T(kUtdSmallEps)), -s_max(m.sigma_e, T(0)) / (omega * T(kEps0)));
    const T mu = s_max(m.mu_r, T(kUtdSmallEps));
    const Cx<T> root = csqrt(eta * mu - cx(sin2, T(0)));
    const Cx<T> mu_ct = cx(mu * ct, T(0));
    const Cx<T> eta_ct = eta * ct;
    *r_te = ((mu_ct - root) / (mu_ct + root)) * m.gain;
    *r_tm = ((eta_ct - root) / (eta_ct + root)) * m.gain;
}

// 1 + gain * r of halfspace_fresnel, formed without the cancellation near
// grazing incidence (r -> -1): with a = mu cos, b = root (resp. eta cos, b),
// 1 + g (a - b) / (a + b) = ((1 + g) a + (1 - g) b) / (a + b).
template <typename T, typename F = double>
WCB_HD void halfspace_fresnel_one_plus(T cos_theta, const Slab<T>& m, F frequency, Cx<T>* p_te, Cx<T>* p_tm) {
    const T omega = T(s_max(kTwoPi * frequency, kUtdSmallEps));
    T ct = s_abs(cos_theta);
    ct = s_min(s_max(ct, T(kUtdSmallEps)), T(1));
    const T sin2 = s_max(T(1) - ct * ct, T(0));
    const Cx<T> eta = cx(s_max(m.eps_r, T(kUtdSmallEps)), -s_max(m.sigma_e, T(0)) / (omega * T(kEps0)));
    const T mu = s_max(m.mu_r, T(kUtdSmallEps));
    const Cx<T> root = csqrt(eta * mu - cx(sin2, T(0)));
    const Cx<T> mu_ct = cx(mu * ct, T(0));
    const Cx<T> eta_ct = eta * ct;
    const T gp = T(1) + m.gain, gm = T(1) - m.gain;
    *p_te = (mu_ct * gp + root * gm) / (mu_ct + root);
    *p_tm = (eta_ct * gp + root * gm) / (eta_ct + root);
}

// One specular bounce of the transported field (the loop body of
// _reference_fields.py:143-181).  Updates `value` and `outgoing`.
template <typename T, typename F = double>
WCB_HD void reflect_bounce(C3<T>& value, V3<T>& outgoing, V3<T> incident, V3<T> normal_in, const Slab<T>& m,
                           F frequency, T wavelength) {
    const V3<T> ez = v3<T>(T(0), T(0), T(1));
    V3<T> normal = safe_normalize(normal_in, ez);
    if (value_of(dot(incident, normal)) > 0) normal = -normal;
    const T dot_in = dot(incident, normal);
    const V3<T> reflected = safe_normalize(incident - normal * (T(2) * dot_in), -incident);
    const V3<T> s_axis = safe_normalize(cross(normal, incident), stable_perp_basis(incident, normal));
    const V3<T> p_in = safe_normalize(cross(s_axis, incident), stable_perp_basis(incident, s_axis));
    const V3<T> p_out = safe_normalize(cross(s_axis, reflected), stable_perp_basis(reflected, s_axis));
    Cx<T> r_te, r_tm;
    slab_fresnel(s_abs(dot_in), m, frequency, wavelength, &r_te, &r_tm);
    const Cx<T> e_s = c3_dot(value, s_axis);
    const Cx<T> e_p = c3_dot(value, p_in);
    value = c3_axis(s_axis, r_te * e_s) + c3_axis(p_out, r_tm * e_p);
    outgoing = reflected;
}

// Output bundle of one path evaluated at one frequency.
template <typename T>
struct PathEval {
    C3<T> field;        // unit-excitation complex 3-vector at the receiver
    Cx<T> coefficient;  // rx projection of `field`
    V3<T> direction;    // arrival direction
};

// Receiver projection onto the unnormalised transverse rx polarization.
template <typename T>
WCB_HD Cx<T> project_receiver(const C3<T>& value, V3<T> direction, V3<T> rx_pol) {
    return c3_dot(value, transverse(direction, rx_pol));
}

// Free-space LoS (fields.cu:36-82; _reference_fields.py:64-82).
// `distance` is the FP64 length used for amplitude and phase.
template <typename T>
WCB_HD PathEval<T> eval_free_space(V3<T> source, V3<T> target, V3<T> tx_pol, V3<T> rx_pol, double k, double distance) {
    const V3<T> off = target - source;
    const V3<T> dir = safe_normalize(off, v3<T>(T(0), T(0), T(1)));
    const V3<T> tx_axis = transverse(dir, tx_pol);
    const T amp = T(1) / (T(2) * T(s_max(k, kUtdSmallEps)) * T(s_max(distance, kUtdEps)));
    const Cx<T> carrier = phasor_neg_kd<T>(k, distance) * amp;
    PathEval<T> out;
    out.field = c3_axis(tx_axis, carrier);
    out.direction = dir;
    out.coefficient = project_receiver(out.field, dir, rx_pol);
    return out;
}

// Rouard stack transmission for one wall (_reference_fields.py:196-273).
// Layers ordered entry -> exit; returns t.  The layer values are stored as S
// and read as T (an FP64 solve reads the FP32 tables exactly widened).
template <typename T, typename F = double, typename S = T>
WCB_HD Cx<T> stack_t(T cos_theta, const S* thickness, const S* eps_r, const S* sigma_e, const S* mu_r, int count,
                     F frequency, int pol_tm) {
    if (count <= 0) return cx(T(1), T(0));
    const T omega = T(s_max(kTwoPi * frequency, kUtdSmallEps));
    T ct = s_min(s_max(s_abs(cos_theta), T(kUtdSmallEps)), T(1));
    const T sin2 = s_max(T(1) - ct * ct, T(0));
    const T k_entry = omega / T(kC0);
    const T k_par = k_entry * s_sqrt(sin2);
    const Cx<T> kz_entry = cx(k_entry * ct, T(0));
    const Cx<T> eps_vac = cx(T(kEps0), T(0));
    const Cx<T> mu_vac = cx(T(kMu0), T(0));
    auto admittance = [&](Cx<T> eps_abs, Cx<T> mu_abs, Cx<T> kz) -> Cx<T> {
        if (!pol_tm) return kz / (mu_abs * omega);
        return (eps_abs * omega) / kz;
    };
    auto medium = [&](int i, Cx<T>* eps_abs, Cx<T>* mu_abs, Cx<T>* kz) {
        *eps_abs = cx(T(kEps0) * s_max(T(eps_r[i]), T(kUtdSmallEps)), -s_max(T(sigma_e[i]), T(0)) / omega);
        *mu_abs = cx(T(kMu0) * s_max(T(mu_r[i]), T(kUtdSmallEps)), T(0));
        const Cx<T> kk = csqrt((*eps_abs) * (*mu_abs)) * omega;
        *kz = csqrt(kk * kk - cx(k_par * k_par, T(0)));
    };
    const Cx<T> y_entry = admittance(eps_vac, mu_vac, kz_entry);
    const Cx<T> y_exit = y_entry;
    Cx<T> eb, mb, kz_below;
    medium(count - 1, &eb, &mb, &kz_below);
    Cx<T> y_below = admittance(eb, mb, kz_below);
    Cx<T> r_total = (y_below - y_exit) / (y_below + y_exit);
    Cx<T> t_total = (y_below * T(2)) / (y_below + y_exit);
    const Cx<T> one = cx(T(1), T(0));
    for (int layer = count - 1; layer >= 0; --layer) {
        const T th = s_max(T(thickness[layer]), T(0));
        // exp(-j kz th)
        const Cx<T> phase = cexp(cx(kz_below.im * th, -kz_below.re * th));
        const Cx<T> phase2 = phase * phase;
        Cx<T> kz_above, y_above;
        if (layer > 0) {
            Cx<T> ea, ma;
            medium(layer - 1, &ea, &ma, &kz_above);
            y_above = admittance(ea, ma, kz_above);
        } else {
            kz_above = kz_entry;
            y_above = y_entry;
        }
        const Cx<T> r_top = (y_above - y_below) / (y_above + y_below);
        const Cx<T> t_top = (y_above * T(2)) / (y_above + y_below);
        const Cx<T> loop = phase2 * r_total;
        const Cx<T> den = one + r_top * loop;
        r_total = (r_top + loop) / den;
        t_total = (t_top * phase * t_total) / den;
        kz_below = kz_above;
        y_below = y_above;
    }
    return t_total;
}

// Material layer tables (CSR) at one frequency.
template <typename T>
struct LayerTable {
    const int* offset;
    const int* count;
    const T* thickness;
    const T* eps_r;
    const T* sigma_e;
    const T* mu_r;
};

// One wall of the straight thin-sheet chain (_reference_fields.py:307-333).
template <typename T, typename S>
WCB_HD void transmit_wall(C3<T>& value, T& carrier_shortening, V3<T> dir, V3<T> normal_in, int material,
                          const LayerTable<S>& lt, double frequency) {
    V3<T> n = safe_normalize(normal_in, v3<T>(T(0), T(0), T(1)));
    if (value_of(dot(dir, n)) > 0) n = -n;
    T ct = s_abs(dot(dir, n));
    ct = s_min(s_max(ct, T(kUtdSmallEps)), T(1));
    const int first = lt.offset[material];
    const int cnt = lt.count[material];
    const Cx<T> t_te = stack_t<T, double, S>(ct, lt.thickness + first, lt.eps_r + first, lt.sigma_e + first,
                                             lt.mu_r + first, cnt, frequency, 0);
    const Cx<T> t_tm = stack_t<T, double, S>(ct, lt.thickness + first, lt.eps_r + first, lt.sigma_e + first,
                                             lt.mu_r + first, cnt, frequency, 1);
    const V3<T> s_axis = safe_normalize(cross(n, dir), stable_perp_basis(dir, n));
    const V3<T> p_axis = safe_normalize(cross(s_axis, dir), stable_perp_basis(dir, s_axis));
    const Cx<T> e_s = c3_dot(value, s_axis);
    const Cx<T> e_p = c3_dot(value, p_axis);
    value = c3_axis(s_axis, t_te * e_s) + c3_axis(p_axis, t_tm * e_p);
    T wall = T(0);
    for (int i = 0; i < cnt; ++i) wall = wall + s_max(T(lt.thickness[first + i]), T(0));
    carrier_shortening = carrier_shortening + wall * ct;
}

}  // namespace wcb
