// Derivatives of one diffraction record's path field.
//
// * Dual-number overloads of the UTD special functions (the KP transition
//   function and the Fresnel complement modulus) with their analytic
//   derivatives, used by every forward-mode evaluation.
// * A hand-written reverse-mode (adjoint) evaluation of the record's receiver
//   coefficient: one FP64 forward sweep that keeps its intermediates, then one
//   reverse sweep that returns the gradient of a real loss with respect to
//   every input at once (Tx and Rx positions, the edge frame, the frequency,
//   and eps_r / sigma of both face materials).  The two subfunctions with many
//   internal branches -- a mended KP term (five inputs) and a half-space
//   Fresnel face factor (four inputs) -- give their local Jacobians through
//   dual lanes inside the forward sweep; everything else is differentiated by
//   hand.  Each branch (floors, clamps, the wedge-angle wrap, the corner
//   selection) is differentiated on the side the forward value took, the same
//   rule the dual-number evaluation follows, so both give the same
//   derivatives up to rounding.
// * The adjoint of the edge frame's construction from its vertices (end
//   points and the two faces whose normals bound the wedge).
//
// Conventions: a complex value z = a + jb carries the adjoint
// zb = dL/da + j dL/db; then for w = u v, ub = wb conj(v), and for a real
// input x of z, dL/dx = Re(zb conj(dz/dx)).
#pragma once

#include "dual.cuh"
#include "utd.cuh"

namespace wcb {

// KP transition F(x) with F'(x) = F(x) (1/(2x) + j) - j.
template <int N>
WCB_HD Cx<Dual<N>> transition(const Dual<N>& x) {
    if (x.v <= 0.0) return cx(Dual<N>(0.0), Dual<N>(0.0));
    const Cx<double> f = transition<double>(x.v);
    const double inv2x = 0.5 / x.v;
    const double dre = f.re * inv2x - f.im;
    const double dim = f.im * inv2x + f.re - 1.0;
    return cx(chain(f.re, dre, x), chain(f.im, dim, x));
}

// exp(-j k d) for dual geometry (the UTD phase).
template <typename T, int N>
WCB_HD Cx<Dual<N>> phasor_kd(const Dual<N>& k, const Dual<N>& d) {
    return phasor_neg_kd(k, d);
}

// |(1+j)/2 - (C(x) + jS(x))| with d/dx (C + jS) = exp(j pi x^2 / 2).
template <int N>
WCB_HD Dual<N> fresnel_complement_abs(const Dual<N>& x) {
    const double xv = x.v;
    Cx<double> c;
    if (xv >= 0.0) {
        c = fresnel_pos<double>(xv, true).complement;
    } else {
        c = cx(1.0, 1.0) - fresnel_pos<double>(-xv, true).complement;
    }
    const double a = hypot(c.re, c.im);
    double ph = kPi / 2 * xv * xv;
    ph = ph - kTwoPi * floor(ph / kTwoPi);
    double es, ec;
    sincos(ph, &es, &ec);
    const double g = a > 0.0 ? -(c.re * ec + c.im * es) / a : 0.0;
    return chain(a, g, x);
}

// ---------------------------------------------------------------- edge frame
// Unit normal of (b - a) x (c - a), length floored at 1e-6 (the scene
// compile's rule).
template <typename G>
WCB_HD V3<G> unit_face_normal(V3<G> a, V3<G> b, V3<G> c) {
    const V3<G> n = cross(b - a, c - a);
    return n * (G(1.0) / s_max(length(n), 1e-6));
}

// Edge frame from the edge's end vertices and the ordered unit normals of
// the faces that bound the wedge (n1 = -n0 for a half-plane), following the
// scene compile's construction.
template <typename G>
WCB_HD EdgeFrame<G> frame_from(V3<G> va, V3<G> vb, V3<G> n0, V3<G> n1, bool face_n) {
    const V3<G> vec = vb - va;
    const G L = s_max(length(vec), 1e-12);
    EdgeFrame<G> f;
    f.e = vec * (G(1.0) / L);
    f.c = (va + vb) * G(0.5);
    f.half_length = L * 0.5;
    f.n0 = n0;
    const V3<G> t = cross(f.n0, f.e);
    f.t0 = t * (G(1.0) / s_max(length(t), 1e-6));
    if (face_n) {
        G cosv = -dot(f.n0, n1);
        cosv = s_min(s_max(cosv, -1.0), 1.0);
        f.n = (G(kTwoPi) - s_acos(cosv)) / kPi;
    } else {
        f.n = G(2.0);
    }
    const V3<G> bis = f.n0 + n1;
    const G bl = length(bis);
    f.bisector = value_of(bl) > 1e-6 ? bis * (G(1.0) / bl) : -f.t0;  // feeds only the visibility point
    f.face_n = face_n;
    return f;
}

// ---------------------------------------------------------------- reverse-mode helpers
namespace rev {

using D3 = V3<double>;

WCB_HD D3 zero3() { return v3(0.0, 0.0, 0.0); }
// Re(a conj(b))
WCB_HD double rdot(Cx<double> a, Cx<double> b) { return a.re * b.re + a.im * b.im; }

// z = a x b: ab += b x zb, bb += zb x a
WCB_HD void cross_vjp(D3 a, D3 b, D3 zb, D3& ab, D3& bb) {
    ab = ab + cross(b, zb);
    bb = bb + cross(zb, a);
}

// y = v / max(|v|, floor): the adjoint of v from that of y
WCB_HD D3 normalize_floor_vjp(D3 v, double floor_len, D3 y, D3 yb) {
    const double l = length(v);
    if (l >= floor_len) return (yb - y * dot(y, yb)) * (1.0 / l);
    return yb * (1.0 / floor_len);
}

}  // namespace rev

// Inputs of one diffraction record's receiver coefficient (FP64).
struct UtdRecordIn {
    V3<double> S, R;          // Tx and Rx positions
    EdgeFrame<double> fr;     // edge frame (centre, direction, face-0 tangent and normal, half length, n)
    V3<double> tx_pol, rx_pol;
    Slab<double> m0, mn;      // face materials giving R_0 and R_n
    double f;                 // frequency (Hz)
};

// Gradient of the loss with respect to those inputs.
struct UtdRecordGrad {
    V3<double> S, R, c, e, t0, n0;
    double half_length, n, f;
    double eps0, sig0, epsn, sign;
};

// The record's path field sq * coefficient (forward) and, for the loss
// L = gg |pf|^2 + gr Re(pf) + gi Im(pf) around it, the gradient of L with
// respect to every input (reverse).  The coefficient is the receiver
// projection of the UTD field of utd_field_gt at the unclamped stationary
// point's arrival direction, as the dual-number evaluation forms it.
WCB_HD Cx<double> utd_record_vjp(const UtdRecordIn& in, double sq, double gg, double gr, double gi,
                                 UtdRecordGrad& g) {
    using rev::D3;
    using rev::rdot;
    using rev::zero3;
    g.S = g.R = g.c = g.e = g.t0 = g.n0 = zero3();
    g.half_length = g.n = g.f = g.eps0 = g.sig0 = g.epsn = g.sign = 0.0;
    const EdgeFrame<double>& fr = in.fr;
    const D3 c = fr.c, e = fr.e, t0 = fr.t0, n0 = fr.n0;
    const double hl = fr.half_length, nn = fr.n;
    constexpr double kIs2 = 0.70710678118654752440;

    // ------------------------------------------------------------ forward sweep
    const double k = kTwoPi * in.f / kC0;
    const D3 ds = in.S - c;
    const double ts = dot(ds, e);
    const D3 ps = ds - e * ts;
    const double rs = length(ps);
    const D3 dr = in.R - c;
    const double tr = dot(dr, e);
    const D3 pr = dr - e * tr;
    const double rr = length(pr);
    const double den = rs + rr;
    const bool unfold = den > 0.0;
    const double t_star = unfold ? ts + (tr - ts) * rs / den : ts;
    const D3 q = c + e * t_star;
    const D3 spv = q - in.S;
    const D3 sv = in.R - q;
    const double lp = length(spv), ls = length(sv);
    const bool lp_in = lp >= kUtdMinDistance, ls_in = ls >= kUtdMinDistance;
    const double s_p = lp_in ? lp : kUtdMinDistance;
    const double s = ls_in ? ls : kUtdMinDistance;
    const double yp = dot(ps, n0), xp = dot(ps, t0);
    double phi_p = s_atan2(yp, xp);
    if (phi_p < 0) phi_p += kTwoPi;
    const double yr = dot(pr, n0), xr = dot(pr, t0);
    double phi_raw = s_atan2(yr, xr);
    if (phi_raw < 0) phi_raw += kTwoPi;
    const double npi = nn * kPi;
    if (phi_p > npi) return cx(0.0, 0.0);  // source inside the wedge: no field, no gradient
    int phi_case = 0;  // 0: phi_raw; 1: clamped to n pi; 2: clamped to 0
    double phi = phi_raw;
    if (phi_raw > npi) {
        if (phi_raw - npi < kTwoPi - phi_raw) {
            phi = npi;
            phi_case = 1;
        } else {
            phi = 0.0;
            phi_case = 2;
        }
    }
    const D3 sh_p = spv * (1.0 / s_p);
    const D3 sh = sv * (1.0 / s);
    const double cb0 = dot(sh_p, e);
    const bool cb_in = cb0 >= -1.0 && cb0 <= 1.0;
    const double cos_b = cb_in ? cb0 : (cb0 < -1.0 ? -1.0 : 1.0);
    const double sb2 = 1.0 - cos_b * cos_b;
    const double sbr = sqrt(sb2 >= 0.0 ? sb2 : 0.0);
    const bool sb_in = sbr >= 1e-6;
    const double sin_b = sb_in ? sbr : 1e-6;
    const double kl = k * s * s_p * sin_b * sin_b / (s + s_p);
    const double rho_p = s_p * sin_b, rho = s * sin_b;
    const double kappa = rho_p * rho_p / (s_p * s_p * s_p) + rho * rho / (s * s * s);
    const double sigma = sqrt(k * kappa / kPi);
    const double a_hi = sigma * (hl - t_star);
    const double a_lo = -(sigma * (-hl - t_star));
    double hi_abs, lo_abs, dhi, dlo;
    {
        Dual<1> x(a_hi);
        x.d[0] = 1.0;
        const Dual<1> r = fresnel_complement_abs(x);
        hi_abs = r.v;
        dhi = r.d[0];
        x = Dual<1>(a_lo);
        x.d[0] = 1.0;
        const Dual<1> r2 = fresnel_complement_abs(x);
        lo_abs = r2.v;
        dlo = r2.d[0];
    }
    const double tm_raw = 1.0 - kIs2 * lo_abs - kIs2 * hi_abs;
    const bool tm_in = tm_raw >= 0.0 && tm_raw <= 1.0;
    const double t_mono = tm_in ? tm_raw : (tm_raw < 0.0 ? 0.0 : 1.0);
    const bool near_hi = fabs(t_star - hl) < fabs(t_star + hl);
    const double u = near_hi ? sigma * (t_star - hl) : sigma * (-hl - t_star);
    const double ex_raw = u / kGammaScale;
    const bool ex_in = ex_raw <= 80.0;
    const double E = s_exp(ex_in ? ex_raw : 80.0);
    const double gamma = 1.0 / (1.0 + E);
    // face factors with their Jacobians (lanes: angle, eps_r, sigma_e, frequency)
    Cx<double> r_te[2] = {cx(0.0, 0.0), cx(0.0, 0.0)}, r_tm[2] = {cx(0.0, 0.0), cx(0.0, 0.0)};
    Cx<double> dte[2][4], dtm[2][4];
    const int faces = fr.face_n ? 2 : 1;
#pragma unroll 1
    for (int face = 0; face < faces; ++face) {
        const Slab<double>& m = face == 0 ? in.m0 : in.mn;
        Dual<4> ang(face == 0 ? phi_p : npi - phi), er(m.eps_r), sg(m.sigma_e), fq(in.f);
        for (int l = 0; l < 4; ++l) ang.d[l] = er.d[l] = sg.d[l] = fq.d[l] = 0.0;
        ang.d[0] = er.d[1] = sg.d[2] = fq.d[3] = 1.0;
        const Slab<Dual<4>> md{er, sg, Dual<4>(m.mu_r), Dual<4>(m.gain), Dual<4>(m.thickness)};
        Cx<Dual<4>> te, tm;
        halfspace_fresnel(s_sin(ang), md, fq, &te, &tm);
        r_te[face] = cx(te.re.v, te.im.v);
        r_tm[face] = cx(tm.re.v, tm.im.v);
        for (int l = 0; l < 4; ++l) {
            dte[face][l] = cx(te.re.d[l], te.im.d[l]);
            dtm[face][l] = cx(tm.re.d[l], tm.im.d[l]);
        }
    }
    const double bm = phi - phi_p, bp = phi + phi_p;
    // the four mended KP terms with their Jacobians (lanes: beta, n, kl, t_mono, gamma)
    Cx<double> T[4], dT[4][5];
#pragma unroll 1
    for (int qq = 0; qq < 4; ++qq) {
        const bool incident = qq < 2;
        Dual<5> b(incident ? bm : bp), n5(nn), k5(kl), tm5(t_mono), g5(gamma);
        for (int l = 0; l < 5; ++l) b.d[l] = n5.d[l] = k5.d[l] = tm5.d[l] = g5.d[l] = 0.0;
        b.d[0] = n5.d[1] = k5.d[2] = tm5.d[3] = g5.d[4] = 1.0;
        const Cx<Dual<5>> r = mended_term(b, n5, k5, tm5, g5, (qq & 1) ? -1 : +1, incident);
        T[qq] = cx(r.re.v, r.im.v);
        for (int l = 0; l < 5; ++l) dT[qq][l] = cx(r.re.d[l], r.im.d[l]);
    }
    const Cx<double> rn_te = r_te[1], rn_tm = r_tm[1], r0_te = r_te[0], r0_tm = r_tm[0];
    const Cx<double> sum_soft = T[0] + T[1] + rn_te * T[2] + r0_te * T[3];
    const Cx<double> sum_hard = T[0] + T[1] + rn_tm * T[2] + r0_tm * T[3];
    const double pre_mag = 1.0 / (2.0 * nn * sqrt(kTwoPi * k) * sin_b);
    // ray-fixed bases
    const D3 pp_raw = cross(e, sh_p);
    const double lpp = length(pp_raw);
    const D3 phi_hat_p = pp_raw * (1.0 / (lpp >= 1e-12 ? lpp : 1e-12));
    const D3 beta_hat_p = cross(sh_p, phi_hat_p);
    const D3 ph_raw = cross(e, sh);
    const double lph = length(ph_raw);
    const D3 phi_hat = ph_raw * (1.0 / (lph >= 1e-12 ? lph : 1e-12));
    const D3 beta_hat = cross(sh, phi_hat);
    const double pt = dot(in.tx_pol, sh_p);
    const D3 tx_axis = in.tx_pol - sh_p * pt;
    const double inc_amp = 1.0 / (2.0 * k * s_p);
    const double ab = dot(tx_axis, beta_hat_p), af = dot(tx_axis, phi_hat_p);
    const double e_beta = ab * inc_amp, e_phi = af * inc_amp;
    const double sg = s_p / (s * (s_p + s));
    const double spread = sqrt(sg);
    const double Lsum = s_p + s;
    const Cx<double> ph = phasor_neg_kd<double>(k, Lsum);
    // receiver projection along the arrival direction from the unclamped stationary point
    const D3 dvec = in.R - q;
    const double ld = length(dvec);
    const bool dir_in = ld > kUtdSmallEps;
    const D3 dir = dir_in ? dvec * (1.0 / (ld + kUtdEps)) : v3(0.0, 0.0, 1.0) * (1.0 / (1.0 + kUtdEps));
    const double pd = dot(in.rx_pol, dir);
    const D3 rxt = in.rx_pol - dir * pd;
    const double Bb = dot(beta_hat, rxt), Bf = dot(phi_hat, rxt);
    const double Xb = e_beta * Bb, Xf = e_phi * Bf;
    const Cx<double> Z = sum_soft * Xb + sum_hard * Xf;
    const Cx<double> K0 = cx(kIs2, -kIs2);  // -(-1 + j)/sqrt(2)
    const double M = pre_mag * spread;
    const Cx<double> Wc = K0 * ph * M;
    const Cx<double> coef = Wc * Z;
    const Cx<double> pf = coef * sq;

    // ------------------------------------------------------------ reverse sweep
    const Cx<double> pfb = cx(2.0 * gg * pf.re + gr, 2.0 * gg * pf.im + gi);
    const Cx<double> coefb = pfb * sq;
    const Cx<double> Zb = coefb * cconj(Wc);
    const Cx<double> Wcb = coefb * cconj(Z);
    const Cx<double> phb = Wcb * cconj(K0) * M;
    const double Mb = rdot(Wcb, K0 * ph);
    const double pre_magb = Mb * spread;
    double spreadb = Mb * pre_mag;
    // ph = exp(-j k Lsum)
    const Cx<double> mjph = cx(ph.im, -ph.re);  // -j ph
    const double phr = rdot(phb, mjph);
    double kb = phr * Lsum;
    double s_pb = phr * k, sb = phr * k;
    // Z = sum_soft Xb + sum_hard Xf
    const Cx<double> ssb = Zb * Xb, shb_ = Zb * Xf;
    const double Xbb = rdot(Zb, sum_soft), Xfb = rdot(Zb, sum_hard);
    const double e_betab = Xbb * Bb, Bbb = Xbb * e_beta;
    const double e_phib = Xfb * Bf, Bfb = Xfb * e_phi;
    D3 beta_hatb = rxt * Bbb, phi_hatb = rxt * Bfb;
    const D3 rxtb = beta_hat * Bbb + phi_hat * Bfb;
    D3 dirb = rxtb * (-pd);
    dirb = dirb + in.rx_pol * (-dot(rxtb, dir));
    D3 qb = zero3(), Rb = zero3(), Sb = zero3(), cbar = zero3(), eb = zero3(), t0b = zero3(), n0b = zero3();
    if (dir_in) {
        const double inv = 1.0 / (ld + kUtdEps);
        D3 dvecb = dirb * inv;
        const double ldb = -dot(dirb, dvec) * inv * inv;
        if (ld > 0.0) dvecb = dvecb + dvec * (ldb / ld);
        Rb = Rb + dvecb;
        qb = qb - dvecb;
    }
    // spread = sqrt(sg), sg = s_p / (s (s_p + s))
    if (spread > 0.0) {
        const double sgb = spreadb * 0.5 / spread;
        const double d2 = (s_p + s) * (s_p + s);
        s_pb += sgb / d2;
        sb += sgb * (-s_p * (s_p + 2.0 * s) / (s * s * d2));
    }
    // e_beta, e_phi
    const double abb = e_betab * inc_amp, afb = e_phib * inc_amp;
    const double inc_ampb = e_betab * ab + e_phib * af;
    const D3 tx_axisb = beta_hat_p * abb + phi_hat_p * afb;
    D3 beta_hat_pb = tx_axis * abb, phi_hat_pb = tx_axis * afb;
    kb += -inc_ampb * inc_amp / k;
    s_pb += -inc_ampb * inc_amp / s_p;
    // tx_axis = tx_pol - sh_p (tx_pol . sh_p)
    D3 sh_pb = tx_axisb * (-pt);
    sh_pb = sh_pb + in.tx_pol * (-dot(tx_axisb, sh_p));
    // bases
    D3 shb = zero3();
    rev::cross_vjp(sh, phi_hat, beta_hatb, shb, phi_hatb);
    const D3 ph_rawb = rev::normalize_floor_vjp(ph_raw, 1e-12, phi_hat, phi_hatb);
    rev::cross_vjp(e, sh, ph_rawb, eb, shb);
    rev::cross_vjp(sh_p, phi_hat_p, beta_hat_pb, sh_pb, phi_hat_pb);
    const D3 pp_rawb = rev::normalize_floor_vjp(pp_raw, 1e-12, phi_hat_p, phi_hat_pb);
    rev::cross_vjp(e, sh_p, pp_rawb, eb, sh_pb);
    // pre_mag = 1 / (2 n sqrt(2 pi k) sin_b)
    double nb = -pre_magb * pre_mag / nn;
    kb += -0.5 * pre_magb * pre_mag / k;
    double sin_bb = -pre_magb * pre_mag / sin_b;
    // KP sums
    Cx<double> Tb[4];
    Tb[0] = ssb + shb_;
    Tb[1] = ssb + shb_;
    Tb[2] = ssb * cconj(rn_te) + shb_ * cconj(rn_tm);
    Tb[3] = ssb * cconj(r0_te) + shb_ * cconj(r0_tm);
    Cx<double> rteb[2], rtmb[2];
    rteb[1] = ssb * cconj(T[2]);
    rtmb[1] = shb_ * cconj(T[2]);
    rteb[0] = ssb * cconj(T[3]);
    rtmb[0] = shb_ * cconj(T[3]);
    double bmb = 0.0, bpb = 0.0, klb = 0.0, t_monob = 0.0, gammab = 0.0;
    for (int qq = 0; qq < 4; ++qq) {
        const double cbeta = rdot(Tb[qq], dT[qq][0]);
        if (qq < 2) bmb += cbeta;
        else bpb += cbeta;
        nb += rdot(Tb[qq], dT[qq][1]);
        klb += rdot(Tb[qq], dT[qq][2]);
        t_monob += rdot(Tb[qq], dT[qq][3]);
        gammab += rdot(Tb[qq], dT[qq][4]);
    }
    double phib = bmb + bpb, phi_pb = bpb - bmb;
    // face factors
    for (int face = 0; face < faces; ++face) {
        double lane[4];
        for (int l = 0; l < 4; ++l) lane[l] = rdot(rteb[face], dte[face][l]) + rdot(rtmb[face], dtm[face][l]);
        if (face == 0) {
            phi_pb += lane[0];
            g.eps0 += lane[1];
            g.sig0 += lane[2];
        } else {
            nb += lane[0] * kPi;  // angle n pi - phi
            phib -= lane[0];
            g.epsn += lane[1];
            g.sign += lane[2];
        }
        g.f += lane[3];
    }
    // gamma = 1 / (1 + exp(min(u / 0.1, 80)))
    double sigmab = 0.0, t_starb = 0.0, hlb = 0.0;
    if (ex_in) {
        const double ub = gammab * (-gamma * gamma * E) / kGammaScale;
        if (near_hi) {
            sigmab += ub * (t_star - hl);
            t_starb += ub * sigma;
            hlb -= ub * sigma;
        } else {
            sigmab += ub * (-hl - t_star);
            hlb -= ub * sigma;
            t_starb -= ub * sigma;
        }
    }
    // t_mono and the two Fresnel complements
    const double absb = tm_in ? -kIs2 * t_monob : 0.0;
    const double a_hib = absb * dhi, a_lob = absb * dlo;
    sigmab += a_hib * (hl - t_star);
    hlb += a_hib * sigma;
    t_starb -= a_hib * sigma;
    sigmab += a_lob * (hl + t_star);
    hlb += a_lob * sigma;
    t_starb += a_lob * sigma;
    // sigma = sqrt(k kappa / pi)
    double kappab = 0.0;
    if (sigma > 0.0) {
        const double wb = sigmab * 0.5 / sigma;
        kb += wb * kappa / kPi;
        kappab = wb * k / kPi;
    }
    const double sp3 = s_p * s_p * s_p, s3 = s * s * s;
    const double rho_pb = kappab * 2.0 * rho_p / sp3, rhob = kappab * 2.0 * rho / s3;
    s_pb += kappab * (-3.0 * rho_p * rho_p / (sp3 * s_p));
    sb += kappab * (-3.0 * rho * rho / (s3 * s));
    s_pb += rho_pb * sin_b;
    sin_bb += rho_pb * s_p;
    sb += rhob * sin_b;
    sin_bb += rhob * s;
    // kl = k s s_p sin_b^2 / (s + s_p)
    {
        const double ss = s + s_p;
        kb += klb * (s * s_p * sin_b * sin_b / ss);
        sin_bb += klb * 2.0 * k * s * s_p * sin_b / ss;
        sb += klb * k * sin_b * sin_b * s_p * s_p / (ss * ss);
        s_pb += klb * k * sin_b * sin_b * s * s / (ss * ss);
    }
    // sin_b = max(sqrt(max(1 - cos_b^2, 0)), 1e-6), cos_b = clamp(sh_p . e)
    double cb0b = 0.0;
    if (sb_in && sbr > 0.0 && sb2 >= 0.0 && cb_in) cb0b = -2.0 * cos_b * (sin_bb * 0.5 / sbr);
    sh_pb = sh_pb + e * cb0b;
    eb = eb + sh_p * cb0b;
    // sh_p = spv / s_p, sh = sv / s
    D3 spvb = sh_pb * (1.0 / s_p);
    s_pb += -dot(sh_pb, spv) / (s_p * s_p);
    D3 svb = shb * (1.0 / s);
    sb += -dot(shb, sv) / (s * s);
    if (lp_in && lp > 0.0) spvb = spvb + spv * (s_pb / lp);
    if (ls_in && ls > 0.0) svb = svb + sv * (sb / ls);
    // wedge angles
    double phi_rawb = 0.0;
    if (phi_case == 0) phi_rawb = phib;
    else if (phi_case == 1) nb += phib * kPi;
    D3 prb = zero3(), psb = zero3();
    {
        const double d2 = xr * xr + yr * yr;
        if (d2 > 0.0) {
            const double yb = phi_rawb * xr / d2, xb = -phi_rawb * yr / d2;
            prb = prb + n0 * yb + t0 * xb;
            n0b = n0b + pr * yb;
            t0b = t0b + pr * xb;
        }
        const double d2p = xp * xp + yp * yp;
        if (d2p > 0.0) {
            const double yb = phi_pb * xp / d2p, xb = -phi_pb * yp / d2p;
            psb = psb + n0 * yb + t0 * xb;
            n0b = n0b + ps * yb;
            t0b = t0b + ps * xb;
        }
    }
    // spv = q - S, sv = R - q, q = c + e t*
    qb = qb + spvb - svb;
    Sb = Sb - spvb;
    Rb = Rb + svb;
    cbar = cbar + qb;
    eb = eb + qb * t_star;
    t_starb += dot(qb, e);
    // t* = ts + (tr - ts) rs / (rs + rr)
    double tsb = 0.0, trb = 0.0, rsb = 0.0, rrb = 0.0;
    if (unfold) {
        tsb += t_starb * (1.0 - rs / den);
        trb += t_starb * rs / den;
        rsb += t_starb * (tr - ts) * rr / (den * den);
        rrb += -t_starb * (tr - ts) * rs / (den * den);
    } else {
        tsb += t_starb;
    }
    if (rs > 0.0) psb = psb + ps * (rsb / rs);
    if (rr > 0.0) prb = prb + pr * (rrb / rr);
    // ps = ds - e ts, ts = ds . e, ds = S - c (and the same on the Rx side)
    D3 dsb = psb;
    eb = eb - psb * ts;
    tsb -= dot(psb, e);
    dsb = dsb + e * tsb;
    eb = eb + ds * tsb;
    Sb = Sb + dsb;
    cbar = cbar - dsb;
    D3 drb = prb;
    eb = eb - prb * tr;
    trb -= dot(prb, e);
    drb = drb + e * trb;
    eb = eb + dr * trb;
    Rb = Rb + drb;
    cbar = cbar - drb;
    // k = 2 pi f / c
    g.f += kb * kTwoPi / kC0;
    g.S = Sb;
    g.R = Rb;
    g.c = cbar;
    g.e = eb;
    g.t0 = t0b;
    g.n0 = n0b;
    g.half_length = hlb;
    g.n = nb;
    return pf;
}

// Adjoint of frame_from: from the frame's gradient (c, e, t0, n0, half
// length, n) to the gradients of the end vertices and of the ordered face
// normals n0, n1 (n1 only when face_n).
WCB_HD void frame_vjp(V3<double> va, V3<double> vb, V3<double> n0, V3<double> n1, bool face_n,
                      const UtdRecordGrad& g, V3<double>& vab, V3<double>& vbb, V3<double>& n0b, V3<double>& n1b) {
    using rev::D3;
    const D3 vec = vb - va;
    const double Lr = length(vec);
    const double L = Lr >= 1e-12 ? Lr : 1e-12;
    const D3 e = vec * (1.0 / L);
    n0b = g.n0;
    n1b = rev::zero3();
    if (face_n) {
        const double cosr = -dot(n0, n1);
        const bool in_range = cosr >= -1.0 && cosr <= 1.0;
        const double x = fmin(fmax(cosr, -1.0), 1.0);
        const double den = sqrt(fmax(1.0 - x * x, 0.0));
        if (in_range && den > 0.0 && fabs(x) < 1.0) {
            const double cosb = g.n / (kPi * den);  // n = (2 pi - acos(cos)) / pi
            n0b = n0b + n1 * (-cosb);
            n1b = n1b + n0 * (-cosb);
        }
    }
    // t0 = t / max(|t|, 1e-6), t = n0 x e
    const D3 t = cross(n0, e);
    const double lt = length(t);
    const D3 t0 = t * (1.0 / (lt >= 1e-6 ? lt : 1e-6));
    const D3 tb = rev::normalize_floor_vjp(t, 1e-6, t0, g.t0);
    D3 eb = g.e;
    rev::cross_vjp(n0, e, tb, n0b, eb);
    double Lb = g.half_length * 0.5;
    vab = g.c * 0.5;
    vbb = g.c * 0.5;
    D3 vecb = eb * (1.0 / L);
    Lb += -dot(eb, vec) / (L * L);
    if (Lr >= 1e-12 && Lr > 0.0) vecb = vecb + vec * (Lb / Lr);
    vbb = vbb + vecb;
    vab = vab - vecb;
}

// Adjoint of unit_face_normal: adds the vertex gradients of one face.
WCB_HD void face_normal_vjp(V3<double> a, V3<double> b, V3<double> c, V3<double> nb, V3<double>& ab, V3<double>& bb,
                            V3<double>& cb) {
    const V3<double> B = b - a, C = c - a;
    const V3<double> m = cross(B, C);
    const double lm = length(m);
    const V3<double> n = m * (1.0 / (lm >= 1e-6 ? lm : 1e-6));
    const V3<double> mb = rev::normalize_floor_vjp(m, 1e-6, n, nb);
    const V3<double> Bb = cross(C, mb), Cb = cross(mb, B);
    ab = ab - Bb - Cb;
    bb = bb + Bb;
    cb = cb + Cb;
}

}  // namespace wcb
