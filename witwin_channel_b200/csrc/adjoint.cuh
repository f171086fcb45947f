// Shared device code of the fixed-topology VJP (see adjoint.cu): dual UTD
// pieces, the per-record parameter list and the FP64 dual re-evaluation of a
// record's path field.
#pragma once

#include <cub/cub.cuh>

#include "../../include/witwin_channel_b200.h"
#include "dual.cuh"
#include "em.cuh"
#include "internal.h"
#include "paths.cuh"
#include "solve.h"
#include "utd.cuh"

namespace wcb {

// ---------------------------------------------------------------- dual UTD pieces
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

namespace adj {

constexpr int kLanes = 4;
constexpr int kMaxParams = 192;
constexpr int kMaxLayersPerMaterial = 8;
constexpr int kBlock = 128;

enum WantBits { kWantTx = 1, kWantRx = 2, kWantFreq = 4, kWantVertices = 8, kWantMaterials = 16 };

struct AdjParams {
    SceneDev sc;
    const int* edge_slot;
    const int* edge_topo;
    const float* tx_pos;
    const float* tx_power;
    const float* tx_pol;
    int rx_kind;
    const float* rx_pos;
    float grid_origin[3], grid_x[3], grid_y[3];
    int grid_rows, grid_cols;
    float grid_spacing[2];
    const float* rx_pol;
    int rx_pol_stride;
    double freq;
    int num_materials;
    const float* eps_r;
    const float* sigma_e;
    const float* mu_r;
    const float* gain;
    const float* thickness;
    int num_layers;
    const int* layer_offset;
    const int* layer_count;
    const float* layer_thickness;
    const float* layer_eps_r;
    const float* layer_sigma_e;
    const float* layer_mu_r;
    const RowRec* rows;
    const long long* selected;
    long long count;
    const double* g_gain;
    const double* g_re;
    const double* g_im;
    const unsigned char* vertex_mask;  // per vertex: nonzero = differentiate (NULL: all)
    int want;
    // parameter id layout
    int base_meps, base_msig, base_leps, base_lsig, gid_freq, base_tx, base_rx;
    int* counts;
    int* comp_counts;          // (4) records per component: LoS, reflection, transmission, diffraction
    const int* order;          // record indices grouped by (component, depth)
    long long order_begin, order_count;
    const long long* offsets;
    unsigned* out_ids;
    double* out_vals;
    double* row_field;  // optional (K,2): FP64 re-evaluated path field
};

WCB_D int gid_vertex(int v, int c) { return 3 * v + c; }

// Per-record parameter list (global ids, deduplicated, in first-use order).
struct ParamList {
    int n;
    int id[kMaxParams];
    WCB_D void add(int g) {
        for (int i = 0; i < n; ++i)
            if (id[i] == g) return;
        if (n < kMaxParams) id[n++] = g;
    }
};

WCB_D bool vertex_wanted(const AdjParams& p, int v) {
    return (p.want & kWantVertices) && (p.vertex_mask == nullptr || p.vertex_mask[v] != 0);
}

WCB_D void add_vertex(const AdjParams& p, ParamList& pl, int v) {
    if (!vertex_wanted(p, v)) return;
    for (int c = 0; c < 3; ++c) pl.add(gid_vertex(v, c));
}

WCB_D void add_face_vertices(const AdjParams& p, ParamList& pl, int f) {
    for (int k = 0; k < 3; ++k) add_vertex(p, pl, p.sc.faces[3 * f + k]);
}

WCB_D void add_material(const AdjParams& p, ParamList& pl, int m) {
    if (!(p.want & kWantMaterials)) return;
    pl.add(p.base_meps + m);
    pl.add(p.base_msig + m);
}

WCB_D void add_layers(const AdjParams& p, ParamList& pl, int m) {
    if (!(p.want & kWantMaterials)) return;
    const int first = p.layer_offset[m];
    const int cnt = min(p.layer_count[m], kMaxLayersPerMaterial);
    for (int l = 0; l < cnt; ++l) {
        pl.add(p.base_leps + first + l);
        pl.add(p.base_lsig + first + l);
    }
}

WCB_D void build_params(const AdjParams& p, const RowRec& row, ParamList& pl) {
    pl.n = 0;
    if (p.want & kWantTx)
        for (int c = 0; c < 3; ++c) pl.add(p.base_tx + 3 * row.tx + c);
    if ((p.want & kWantRx) && p.rx_kind == 0)
        for (int c = 0; c < 3; ++c) pl.add(p.base_rx + 3 * row.rx + c);
    if (p.want & kWantFreq) pl.add(p.gid_freq);
    if (row.component == 1) {
        for (int k = 0; k < row.depth && k < kMaxDepth; ++k) {
            add_face_vertices(p, pl, row.seq[k]);
            add_material(p, pl, p.sc.face_material[row.seq[k]]);
        }
    } else if (row.component == 5) {
        for (int k = 0; k < row.depth && k < kMaxDepth; ++k) {
            add_face_vertices(p, pl, row.seq[k]);
            add_layers(p, pl, p.sc.face_material[row.seq[k]]);
        }
    } else if (row.component == 2) {
        const int slot = p.edge_slot[row.edge];
        const int* tp = p.edge_topo + 4 * slot;
        add_vertex(p, pl, tp[0]);
        add_vertex(p, pl, tp[1]);
        add_face_vertices(p, pl, tp[2]);
        if (tp[3] >= 0) add_face_vertices(p, pl, tp[3]);
        const EdgeDev& ed = p.sc.edges[slot];
        add_material(p, pl, p.sc.face_material[ed.mat_face0]);
        if (ed.face_n) add_material(p, pl, p.sc.face_material[ed.mat_face1]);
    }
}

// The ids carried as tangent lanes in this pass.
template <int N>
struct Window {
    int id[N];
    int n;
    WCB_D Dual<N> param(double value, int gid) const {
        Dual<N> d(value);
#pragma unroll
        for (int j = 0; j < N; ++j) d.d[j] = (j < n && id[j] == gid) ? 1.0 : 0.0;
        return d;
    }
};

// Forward-mode seeds: one tangent lane whose derivative of every parameter is
// that parameter's entry of a dense tangent vector (the layout of
// wcb_rows_vjp_layout).  The JVP evaluates each record once with these.
template <int N>
struct Seeds {
    const double* t;
    WCB_D Dual<N> param(double value, int gid) const {
        Dual<N> d(value);
#pragma unroll
        for (int j = 0; j < N; ++j) d.d[j] = 0.0;
        d.d[0] = t[gid];
        return d;
    }
};

// Seeds of the plain FP64 evaluation (no tangent lane).
template <int N>
struct Plain {
    WCB_D Dual<N> param(double value, int) const { return Dual<N>(value); }
};

template <template <int> class WT, int N>
WCB_D V3<Dual<N>> vertex(const AdjParams& p, const WT<N>& w, int v) {
    const float* x = p.sc.vertices + 3 * v;
    return v3(w.param(x[0], gid_vertex(v, 0)), w.param(x[1], gid_vertex(v, 1)), w.param(x[2], gid_vertex(v, 2)));
}

// unit normal of (b - a) x (c - a), length floored at 1e-6 (the scene compile's rule)
template <template <int> class WT, int N>
WCB_D V3<Dual<N>> face_unit_normal(const AdjParams& p, const WT<N>& w, int f, V3<Dual<N>>* anchor) {
    const V3<Dual<N>> a = vertex(p, w, p.sc.faces[3 * f]);
    const V3<Dual<N>> b = vertex(p, w, p.sc.faces[3 * f + 1]);
    const V3<Dual<N>> c = vertex(p, w, p.sc.faces[3 * f + 2]);
    if (anchor) *anchor = a;
    const V3<Dual<N>> n = cross(b - a, c - a);
    return n * (Dual<N>(1.0) / s_max(length(n), 1e-6));
}

template <template <int> class WT, int N>
WCB_D Slab<Dual<N>> slab(const AdjParams& p, const WT<N>& w, int m) {
    return Slab<Dual<N>>{w.param(p.eps_r[m], p.base_meps + m), w.param(p.sigma_e[m], p.base_msig + m),
                         Dual<N>(p.mu_r[m]), Dual<N>(p.gain[m]), Dual<N>(p.thickness[m])};
}

template <template <int> class WT, int N>
WCB_D V3<Dual<N>> receiver(const AdjParams& p, const WT<N>& w, int r) {
    if (p.rx_kind == 1) {
        const int row = r / p.grid_cols;
        const int col = r - row * p.grid_cols;
        const float u = __fmul_rn(float(row), p.grid_spacing[0]);
        const float v = __fmul_rn(float(col), p.grid_spacing[1]);
        const float x = __fadd_rn(__fadd_rn(p.grid_origin[0], __fmul_rn(p.grid_x[0], u)), __fmul_rn(p.grid_y[0], v));
        const float y = __fadd_rn(__fadd_rn(p.grid_origin[1], __fmul_rn(p.grid_x[1], u)), __fmul_rn(p.grid_y[1], v));
        const float z = __fadd_rn(__fadd_rn(p.grid_origin[2], __fmul_rn(p.grid_x[2], u)), __fmul_rn(p.grid_y[2], v));
        return v3(Dual<N>(x), Dual<N>(y), Dual<N>(z));
    }
    const float* x = p.rx_pos + 3 * r;
    return v3(w.param(x[0], p.base_rx + 3 * r), w.param(x[1], p.base_rx + 3 * r + 1),
              w.param(x[2], p.base_rx + 3 * r + 2));
}

// Edge frame from vertices, following the scene compile's construction.
template <template <int> class WT, int N>
WCB_D EdgeFrame<Dual<N>> edge_frame_dual(const AdjParams& p, const WT<N>& w, int slot) {
    using D = Dual<N>;
    const int* tp = p.edge_topo + 4 * slot;
    const V3<D> va = vertex(p, w, tp[0]);
    const V3<D> vb = vertex(p, w, tp[1]);
    const V3<D> vec = vb - va;
    const D L = s_max(length(vec), 1e-12);
    EdgeFrame<D> f;
    f.e = vec * (D(1.0) / L);
    f.c = (va + vb) * D(0.5);
    f.half_length = L * 0.5;
    f.n0 = face_unit_normal(p, w, tp[2], (V3<D>*)nullptr);
    const V3<D> n1 = tp[3] >= 0 ? face_unit_normal(p, w, tp[3], (V3<D>*)nullptr) : -f.n0;
    const V3<D> t = cross(f.n0, f.e);
    f.t0 = t * (D(1.0) / s_max(length(t), 1e-6));
    if (tp[3] >= 0) {
        D cosv = -dot(f.n0, n1);
        cosv = s_min(s_max(cosv, -1.0), 1.0);
        f.n = (D(kTwoPi) - s_acos(cosv)) / kPi;
    } else {
        f.n = D(2.0);
    }
    const V3<D> bis = f.n0 + n1;
    const D bl = length(bis);
    f.bisector = value_of(bl) > 1e-6 ? bis * (D(1.0) / bl) : -f.t0;  // feeds only the visibility point
    f.face_n = tp[3] >= 0;
    return f;
}

// FP64 dual re-evaluation of one record's powered path field.
template <int N, int COMP, template <int> class WT>
WCB_D Cx<Dual<N>> eval_record(const AdjParams& p, const RowRec& row, const WT<N>& w) {
    using D = Dual<N>;
    const int t = row.tx, r = row.rx;
    const V3<D> S = v3(w.param(p.tx_pos[3 * t], p.base_tx + 3 * t), w.param(p.tx_pos[3 * t + 1], p.base_tx + 3 * t + 1),
                       w.param(p.tx_pos[3 * t + 2], p.base_tx + 3 * t + 2));
    const V3<D> R = receiver(p, w, r);
    const V3<D> tx_pol = v3(D(p.tx_pol[3 * t]), D(p.tx_pol[3 * t + 1]), D(p.tx_pol[3 * t + 2]));
    const float* rp = p.rx_pol + (long long)r * p.rx_pol_stride;
    const V3<D> rx_pol = v3(D(rp[0]), D(rp[1]), D(rp[2]));
    const D f = w.param(p.freq, p.gid_freq);
    const D k = f * (kTwoPi / kC0);
    const D wl = D(kC0) / f;
    const double sq = sqrt(fmax(double(p.tx_power[t]), 0.0));
    const V3<D> ez = v3(D(0.0), D(0.0), D(1.0));
    Cx<D> coef = cx(D(0.0), D(0.0));
    if constexpr (COMP == 0) {
        const V3<D> off = R - S;
        const D dist = length(off);
        const V3<D> dir = safe_normalize(off, ez);
        const V3<D> tx_axis = transverse(dir, tx_pol);
        const D amp = D(1.0) / (D(2.0) * s_max(k, kUtdSmallEps) * s_max(dist, kUtdEps));
        const C3<D> field = c3_axis(tx_axis, phasor_neg_kd(k, dist) * amp);
        coef = project_receiver(field, dir, rx_pol);
    } else if constexpr (COMP == 1) {
        const int d = min(int(row.depth), kMaxDepth);
        V3<D> nrm[kMaxDepth], img[kMaxDepth], hit[kMaxDepth];
        D off[kMaxDepth];
        V3<D> pp = S;
        for (int q = 0; q < d; ++q) {
            V3<D> a;
            nrm[q] = face_unit_normal(p, w, row.seq[q], &a);
            off[q] = dot(nrm[q], a);
            pp = pp - nrm[q] * (D(2.0) * (dot(pp, nrm[q]) - off[q]));
            img[q] = pp;
        }
        V3<D> x = R;
        for (int q = d - 1; q >= 0; --q) {
            const D denom = dot(img[q] - x, nrm[q]);
            const D tt = (off[q] - dot(x, nrm[q])) / denom;
            x = x + (img[q] - x) * tt;
            hit[q] = x;
        }
        const D length_total = length(R - pp);
        V3<D> prev = S;
        V3<D> incident = safe_normalize(hit[0] - prev, ez);
        C3<D> value = c3_from_real(transverse(incident, tx_pol));
        V3<D> outgoing = incident;
        for (int q = 0; q < d; ++q) {
            incident = safe_normalize(hit[q] - prev, outgoing);
            reflect_bounce(value, outgoing, incident, nrm[q], slab(p, w, p.sc.face_material[row.seq[q]]), f, wl);
            prev = hit[q];
        }
        const V3<D> dir = safe_normalize(R - prev, outgoing);
        const D amp = D(1.0) / (D(2.0) * k * s_max(length_total, kUtdEps));
        value = c3_scale(value, phasor_neg_kd(k, length_total) * amp);
        coef = project_receiver(value, dir, rx_pol);
    } else if constexpr (COMP == 5) {
        const int d = min(int(row.depth), kMaxDepth);
        const V3<D> off = R - S;
        const D dist = length(off);
        const V3<D> dir = safe_normalize(off, ez);
        C3<D> value = c3_from_real(transverse(dir, tx_pol));
        D shorten(0.0);
        for (int q = 0; q < d; ++q) {
            V3<D> n = face_unit_normal(p, w, row.seq[q], (V3<D>*)nullptr);
            n = safe_normalize(n, ez);
            if (value_of(dot(dir, n)) > 0) n = -n;
            D ct = s_abs(dot(dir, n));
            ct = s_min(s_max(ct, D(kUtdSmallEps)), D(1.0));
            const int m = p.sc.face_material[row.seq[q]];
            const int first = p.layer_offset[m];
            const int cnt = min(p.layer_count[m], kMaxLayersPerMaterial);
            D th[kMaxLayersPerMaterial], er[kMaxLayersPerMaterial], sg[kMaxLayersPerMaterial],
                mu[kMaxLayersPerMaterial];
            D wall(0.0);
            for (int l = 0; l < cnt; ++l) {
                th[l] = D(p.layer_thickness[first + l]);
                er[l] = w.param(p.layer_eps_r[first + l], p.base_leps + first + l);
                sg[l] = w.param(p.layer_sigma_e[first + l], p.base_lsig + first + l);
                mu[l] = D(p.layer_mu_r[first + l]);
                wall = wall + s_max(th[l], D(0.0));
            }
            const Cx<D> t_te = stack_t<D, D>(ct, th, er, sg, mu, cnt, f, 0);
            const Cx<D> t_tm = stack_t<D, D>(ct, th, er, sg, mu, cnt, f, 1);
            const V3<D> s_axis = safe_normalize(cross(n, dir), stable_perp_basis(dir, n));
            const V3<D> p_axis = safe_normalize(cross(s_axis, dir), stable_perp_basis(dir, s_axis));
            const Cx<D> e_s = c3_dot(value, s_axis);
            const Cx<D> e_p = c3_dot(value, p_axis);
            value = c3_axis(s_axis, t_te * e_s) + c3_axis(p_axis, t_tm * e_p);
            shorten = shorten + wall * ct;
        }
        const D amp = D(1.0) / (D(2.0) * k * s_max(dist, kUtdEps));
        value = c3_scale(value, phasor_neg_kd(k, dist - shorten) * amp);
        coef = project_receiver(value, dir, rx_pol);
    } else if constexpr (COMP == 2) {
        const int slot = p.edge_slot[row.edge];
        const EdgeDev& ed = p.sc.edges[slot];
        const EdgeFrame<D> fr = edge_frame_dual(p, w, slot);
        V3<D> q;
        const DiffractionResult<D> res =
            utd_field_gt<D, D>(fr, S, R, tx_pol, slab(p, w, p.sc.face_material[ed.mat_face0]),
                               slab(p, w, p.sc.face_material[ed.mat_face1]), f, &q);
        const V3<D> dir = safe_normalize(R - q, ez);
        coef = project_receiver(res.field, dir, rx_pol);
    }
    return cx(coef.re * sq, coef.im * sq);
}


// Per-record VJP of one component: evaluate the record's path field with the
// record's parameters as dual lanes, N at a time, and write one (id,
// contribution) pair per parameter.  Records of other components are skipped.
// rank of a component in the (component, depth) grouping
WCB_HD int component_rank(int c) { return c == 0 ? 0 : c == 1 ? 1 : c == 5 ? 2 : 3; }

template <int N, int COMP>
__global__ void __launch_bounds__(kBlock) k_vjp_rows(AdjParams p) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= p.order_count) return;
    const long long i = p.order[p.order_begin + j];
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    ParamList pl;
    build_params(p, row, pl);
    const long long base = p.offsets[i];
    const double gg = p.g_gain ? p.g_gain[i] : 0.0;
    const double gr = p.g_re ? p.g_re[i] : 0.0;
    const double gi = p.g_im ? p.g_im[i] : 0.0;
    const int passes = max((pl.n + N - 1) / N, p.row_field ? 1 : 0);
    for (int pass = 0; pass < passes; ++pass) {
        Window<N> w;
        w.n = min(N, pl.n - pass * N);
#pragma unroll
        for (int j = 0; j < N; ++j) w.id[j] = j < w.n ? pl.id[pass * N + j] : -1;
        const Cx<Dual<N>> pf = eval_record<N, COMP>(p, row, w);
        if (pass == 0 && p.row_field) {
            p.row_field[2 * i] = pf.re.v;
            p.row_field[2 * i + 1] = pf.im.v;
        }
        for (int j = 0; j < w.n; ++j) {
            const double dre = pf.re.d[j], dim = pf.im.d[j];
            const double dg = 2.0 * (pf.re.v * dre + pf.im.v * dim);
            double c = gg * dg + gr * dre + gi * dim;
            if (!isfinite(c)) c = 0.0;
            p.out_ids[base + pass * N + j] = unsigned(w.id[j]);
            p.out_vals[base + pass * N + j] = c;
        }
    }
}

// The same contributions with one thread per (record, parameter): each
// thread carries a single tangent lane through the record's evaluation.  The
// lanes of a dual number never mix, so every contribution is bit-identical to
// the N-lane kernel's; the one-lane evaluation holds far fewer live values
// per thread, which pays for the repeated value part on the heavy UTD
// records.  `pair_base` is the exclusive prefix over the component's ordered
// records of their work items (parameters, or one for a parameterless record
// whose FP64 field is wanted; k_vjp_work in adjoint.cu).

template <int COMP>
__global__ void __launch_bounds__(kBlock, 4) k_vjp_pairs(AdjParams p, const int* pair_base, long long total) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    // the last ordered record whose work range starts at or before t
    long long lo = 0, hi = p.order_count - 1;
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (pair_base[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const long long i = p.order[p.order_begin + lo];
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    ParamList pl;
    build_params(p, row, pl);
    const int q = int(t - pair_base[lo]);
    Window<1> w;
    w.n = q < pl.n ? 1 : 0;
    w.id[0] = q < pl.n ? pl.id[q] : -1;
    const Cx<Dual<1>> pf = eval_record<1, COMP>(p, row, w);
    if (q == 0 && p.row_field) {
        p.row_field[2 * i] = pf.re.v;
        p.row_field[2 * i + 1] = pf.im.v;
    }
    if (q < pl.n) {
        const double gg = p.g_gain ? p.g_gain[i] : 0.0;
        const double gr = p.g_re ? p.g_re[i] : 0.0;
        const double gi = p.g_im ? p.g_im[i] : 0.0;
        const double dre = pf.re.d[0], dim = pf.im.d[0];
        const double dg = 2.0 * (pf.re.v * dre + pf.im.v * dim);
        double c = gg * dg + gr * dre + gi * dim;
        if (!isfinite(c)) c = 0.0;
        p.out_ids[p.offsets[i] + q] = unsigned(w.id[0]);
        p.out_vals[p.offsets[i] + q] = c;
    }
}

void launch_vjp_diffraction(const AdjParams& p, const int* pair_base, long long total, cudaStream_t s);
void fill_params(AdjParams& p, const SceneHandle* h, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int freq_index, const void* rows, const int64_t* selected, long long K, const int64_t* layout);

// Forward mode: each record of component COMP evaluated once with the tangent
// seeds; writes its FP64 path field and the field's tangent ((K,2) each).
template <int COMP>
__global__ void __launch_bounds__(kBlock) k_jvp_rows(AdjParams p, const double* tangent, double* field,
                                                     double* field_tangent) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= p.count) return;
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    const Seeds<1> seeds{tangent};
    const Cx<Dual<1>> pf = eval_record<1, COMP>(p, row, seeds);
    if (field) {
        field[2 * i] = pf.re.v;
        field[2 * i + 1] = pf.im.v;
    }
    const double dre = pf.re.d[0], dim = pf.im.d[0];
    field_tangent[2 * i] = isfinite(dre) ? dre : 0.0;
    field_tangent[2 * i + 1] = isfinite(dim) ? dim : 0.0;
}

void launch_jvp_diffraction(const AdjParams& p, const double* tangent, double* field, double* field_tangent,
                            cudaStream_t s);

// The records' FP64 path fields alone (the derivative kernels' primal, no
// tangent): the point the cell sums are linearised at.
template <int COMP>
__global__ void __launch_bounds__(kBlock) k_field64_rows(AdjParams p, double* field) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= p.count) return;
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    const Plain<0> seeds{};
    const Cx<Dual<0>> pf = eval_record<0, COMP>(p, row, seeds);
    field[2 * i] = pf.re.v;
    field[2 * i + 1] = pf.im.v;
}

void launch_field64_diffraction(const AdjParams& p, double* field, cudaStream_t s);

}  // namespace adj
}  // namespace wcb
