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
#include "utd_adjoint.cuh"

namespace wcb {

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

// Parameter count of a LoS, reflection or transmission record without the
// generic list (the count build_params gives): endpoint and frequency
// entries, 3 per distinct wanted vertex of its faces, and per distinct face
// material 2 (reflection: eps_r, sigma_e) or 2 per layer (transmission).
WCB_D int face_record_param_count(const AdjParams& p, const RowRec& row) {
    int n = ((p.want & kWantTx) ? 3 : 0) + (((p.want & kWantRx) && p.rx_kind == 0) ? 3 : 0) +
            ((p.want & kWantFreq) ? 1 : 0);
    if (row.component != 1 && row.component != 5) return n;
    int vids[3 * kMaxDepth], mids[kMaxDepth];
    int nv = 0, nm = 0;
    const int d = min(int(row.depth), kMaxDepth);
    for (int k = 0; k < d; ++k) {
        const int f = row.seq[k];
        for (int c = 0; c < 3; ++c) {
            const int v = p.sc.faces[3 * f + c];
            if (!vertex_wanted(p, v)) continue;
            bool seen = false;
            for (int q = 0; q < nv; ++q) seen = seen || vids[q] == v;
            if (!seen) vids[nv++] = v;
        }
        const int m = p.sc.face_material[f];
        bool seen = false;
        for (int q = 0; q < nm; ++q) seen = seen || mids[q] == m;
        if (!seen) mids[nm++] = m;
    }
    n += 3 * nv;
    if (p.want & kWantMaterials) {
        if (row.component == 1) {
            n += 2 * nm;
        } else {
            for (int q = 0; q < nm; ++q) n += 2 * min(p.layer_count[mids[q]], kMaxLayersPerMaterial);
        }
    }
    return n;
}

// The parameters of a diffraction record without the generic list (the same
// set build_params gives): the distinct wanted vertices (end points, then
// the faces' vertices), the distinct face materials, the endpoint and
// frequency entries.
struct DiffParamSet {
    int nv;
    int vid[8];
    int m0, mn;         // differentiated material ids (-1: none); mn is only a material other than m0
    bool same_material; // the second face exists and has face 0's material
    int count;
};

WCB_D DiffParamSet diffraction_params(const AdjParams& p, const RowRec& row) {
    DiffParamSet d;
    d.nv = 0;
    const int slot = p.edge_slot[row.edge];
    const int* tp = p.edge_topo + 4 * slot;
    auto addv = [&](int v) {
        if (!vertex_wanted(p, v)) return;
        for (int i = 0; i < d.nv; ++i)
            if (d.vid[i] == v) return;
        d.vid[d.nv++] = v;
    };
    addv(tp[0]);
    addv(tp[1]);
    for (int k = 0; k < 3; ++k) addv(p.sc.faces[3 * tp[2] + k]);
    if (tp[3] >= 0)
        for (int k = 0; k < 3; ++k) addv(p.sc.faces[3 * tp[3] + k]);
    const EdgeDev& ed = p.sc.edges[slot];
    d.m0 = d.mn = -1;
    d.same_material = false;
    if (p.want & kWantMaterials) {
        d.m0 = p.sc.face_material[ed.mat_face0];
        if (ed.face_n) {
            const int m = p.sc.face_material[ed.mat_face1];
            if (m != d.m0) d.mn = m;
            else d.same_material = true;
        }
    }
    d.count = ((p.want & kWantTx) ? 3 : 0) + (((p.want & kWantRx) && p.rx_kind == 0) ? 3 : 0) +
              ((p.want & kWantFreq) ? 1 : 0) + 3 * d.nv + (d.m0 >= 0 ? 2 : 0) + (d.mn >= 0 ? 2 : 0);
    return d;
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
    return unit_face_normal(a, b, c);
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
    const V3<D> n0 = face_unit_normal(p, w, tp[2], (V3<D>*)nullptr);
    const V3<D> n1 = tp[3] >= 0 ? face_unit_normal(p, w, tp[3], (V3<D>*)nullptr) : -n0;
    return frame_from(vertex(p, w, tp[0]), vertex(p, w, tp[1]), n0, n1, tp[3] >= 0);
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

// Execution-order key of a record: component rank (2 bits), depth (3 bits)
// and, for diffraction, the edge slot (26 bits), so a warp of the derivative
// kernels works on records of one component, and diffraction warps on one
// edge (shared wedge, mostly shared branches).
WCB_D int order_key(const AdjParams& p, const RowRec& row) {
    int key = (component_rank(row.component) << 29) | (min(max(int(row.depth), 0), 7) << 26);
    if (row.component == 2) key |= p.edge_slot[row.edge] & 0x3FFFFFF;
    return key;
}

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
            if (pass * N + j >= p.counts[i]) break;  // never past the record's counted slots
            const double dre = pf.re.d[j], dim = pf.im.d[j];
            const double dg = 2.0 * (pf.re.v * dre + pf.im.v * dim);
            double c = gg * dg + gr * dre + gi * dim;
            if (!isfinite(c)) c = 0.0;
            p.out_ids[base + pass * N + j] = unsigned(w.id[j]);
            p.out_vals[base + pass * N + j] = c;
        }
    }
}

// Reverse mode over the diffraction records: one thread per record.  One
// FP64 forward sweep and one reverse sweep (utd_record_vjp, then the adjoints
// of the edge frame and of the two face normals) give the contribution of
// every parameter of the record at once, where a dual-number evaluation
// would repeat the UTD (and its special functions) once per parameter lane.
// The pairs are written in the record's parameter-list order, like the
// forward-mode kernels, so the id sort and the ordered per-id sums that
// follow are unchanged.
template <int COMP>
__global__ void __launch_bounds__(kBlock) k_vjp_diffraction(AdjParams p) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= p.order_count) return;
    const long long i = p.order[p.order_begin + j];
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    const int slot = p.edge_slot[row.edge];
    const int* tp = p.edge_topo + 4 * slot;
    const EdgeDev& ed = p.sc.edges[slot];
    const bool face_n = tp[3] >= 0;
    const int t = row.tx, r = row.rx;
    auto vtx = [&](int v) {
        const float* x = p.sc.vertices + 3 * v;
        return v3(double(x[0]), double(x[1]), double(x[2]));
    };
    int fv[2][3];
    V3<double> fp[2][3];
    for (int sd = 0; sd < 2; ++sd)
        for (int k = 0; k < 3; ++k) {
            fv[sd][k] = (sd == 0 || face_n) ? p.sc.faces[3 * tp[2 + sd] + k] : -1;
            fp[sd][k] = fv[sd][k] >= 0 ? vtx(fv[sd][k]) : v3(0.0, 0.0, 0.0);
        }
    const V3<double> va = vtx(tp[0]), vb = vtx(tp[1]);
    const V3<double> n0 = unit_face_normal(fp[0][0], fp[0][1], fp[0][2]);
    const V3<double> n1 = face_n ? unit_face_normal(fp[1][0], fp[1][1], fp[1][2]) : -n0;
    UtdRecordIn in;
    in.fr = frame_from(va, vb, n0, n1, face_n);
    in.S = v3(double(p.tx_pos[3 * t]), double(p.tx_pos[3 * t + 1]), double(p.tx_pos[3 * t + 2]));
    const V3<Dual<0>> rq = receiver(p, Plain<0>{}, r);
    in.R = v3(rq.x.v, rq.y.v, rq.z.v);
    in.tx_pol = v3(double(p.tx_pol[3 * t]), double(p.tx_pol[3 * t + 1]), double(p.tx_pol[3 * t + 2]));
    const float* rp = p.rx_pol + (long long)r * p.rx_pol_stride;
    in.rx_pol = v3(double(rp[0]), double(rp[1]), double(rp[2]));
    const int m0 = p.sc.face_material[ed.mat_face0];
    const int mn = face_n ? p.sc.face_material[ed.mat_face1] : -1;
    auto slab64 = [&](int m) {
        return Slab<double>{double(p.eps_r[m]), double(p.sigma_e[m]), double(p.mu_r[m]), double(p.gain[m]),
                            double(p.thickness[m])};
    };
    in.m0 = slab64(m0);
    in.mn = slab64(face_n ? mn : m0);
    in.f = p.freq;
    const double sq = sqrt(fmax(double(p.tx_power[t]), 0.0));
    const double gg = p.g_gain ? p.g_gain[i] : 0.0;
    const double gr = p.g_re ? p.g_re[i] : 0.0;
    const double gi = p.g_im ? p.g_im[i] : 0.0;
    UtdRecordGrad g;
    const Cx<double> pf = utd_record_vjp(in, sq, gg, gr, gi, g);
    if (p.row_field) {
        p.row_field[2 * i] = pf.re;
        p.row_field[2 * i + 1] = pf.im;
    }
    V3<double> vab, vbb, n0b, n1b;
    frame_vjp(va, vb, n0, n1, face_n, g, vab, vbb, n0b, n1b);
    V3<double> fg[2][3];
    for (int sd = 0; sd < 2; ++sd)
        for (int k = 0; k < 3; ++k) fg[sd][k] = v3(0.0, 0.0, 0.0);
    face_normal_vjp(fp[0][0], fp[0][1], fp[0][2], n0b, fg[0][0], fg[0][1], fg[0][2]);
    if (face_n) face_normal_vjp(fp[1][0], fp[1][1], fp[1][2], n1b, fg[1][0], fg[1][1], fg[1][2]);
    // the contributions, in the order tx, rx, frequency, vertices, materials
    const DiffParamSet ps = diffraction_params(p, row);
    long long o = p.offsets[i];
    const long long o_end = o + p.counts[i];
    auto put = [&](int id, double c) {
        if (o >= o_end) return;  // never past the record's counted slots
        if (!isfinite(c)) c = 0.0;
        p.out_ids[o] = unsigned(id);
        p.out_vals[o] = c;
        ++o;
    };
    auto pick = [](V3<double> a, int comp) { return comp == 0 ? a.x : (comp == 1 ? a.y : a.z); };
    if (p.want & kWantTx)
        for (int k = 0; k < 3; ++k) put(p.base_tx + 3 * t + k, pick(g.S, k));
    if ((p.want & kWantRx) && p.rx_kind == 0)
        for (int k = 0; k < 3; ++k) put(p.base_rx + 3 * r + k, pick(g.R, k));
    if (p.want & kWantFreq) put(p.gid_freq, g.f);
    for (int a = 0; a < ps.nv; ++a) {
        const int v = ps.vid[a];
        V3<double> gv = v3(0.0, 0.0, 0.0);
        if (v == tp[0]) gv = gv + vab;
        if (v == tp[1]) gv = gv + vbb;
        for (int sd = 0; sd < 2; ++sd)
            for (int k = 0; k < 3; ++k)
                if (fv[sd][k] == v) gv = gv + fg[sd][k];
        for (int k = 0; k < 3; ++k) put(gid_vertex(v, k), pick(gv, k));
    }
    if (ps.m0 >= 0) {
        put(p.base_meps + ps.m0, g.eps0 + (ps.same_material ? g.epsn : 0.0));
        put(p.base_msig + ps.m0, g.sig0 + (ps.same_material ? g.sign : 0.0));
    }
    if (ps.mn >= 0) {
        put(p.base_meps + ps.mn, g.epsn);
        put(p.base_msig + ps.mn, g.sign);
    }
}

void launch_vjp_diffraction(const AdjParams& p, cudaStream_t s);
void fill_params(AdjParams& p, const SceneHandle* h, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int freq_index, const void* rows, const int64_t* selected, long long K, const int64_t* layout);

// Forward mode: each record of component COMP evaluated once with the tangent
// seeds; writes its FP64 path field and the field's tangent ((K,2) each).
template <int COMP>
__global__ void __launch_bounds__(kBlock) k_jvp_rows(AdjParams p, const double* tangent, double* field,
                                                     double* field_tangent) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= p.order_count) return;
    const long long i = p.order ? p.order[p.order_begin + j] : j;
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
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= p.order_count) return;
    const long long i = p.order ? p.order[p.order_begin + j] : j;
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != COMP) return;
    const Plain<0> seeds{};
    const Cx<Dual<0>> pf = eval_record<0, COMP>(p, row, seeds);
    field[2 * i] = pf.re.v;
    field[2 * i + 1] = pf.im.v;
}

// The frequencies of a multi-frequency plain evaluation (at most 4, the
// solve's own limit per call).
struct FreqSet {
    double f[4];
};

void launch_field64_diffraction(const AdjParams& p, double* field, cudaStream_t s);
void launch_field64_diffraction_multi(const AdjParams& p, int nf, const FreqSet& fs, double* field, cudaStream_t s);

}  // namespace adj
}  // namespace wcb
