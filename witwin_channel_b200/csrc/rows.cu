// Path records: canonical order, identity dedup, max_paths, per-row field
// evaluation from the frozen topology, and deterministic per-cell sums.
//
// Canonical order and selection follow
// native/channel/kernels/evaluated_paths.cu:76-470 and :669-710: the key is
// (rx, tx, depth, component, sequence[0..w-1], primitive, edge); rows with
// the same identity (tx, rx, per-slot event type and object id) keep the
// shortest (first on ties) and a NaN length drops the group; max_paths keeps
// a global prefix or the first max_paths rows of each (rx, tx) pair.  Here the
// key is the concatenation of its fields at the widths the input needs (one
// pass measures the largest rx, tx and object id), cut into 64-bit words and
// sorted with one stable radix pass per word, least significant first; every
// field keeps its full value, so any number of sources, sinks or ids sorts
// exactly.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "em.cuh"
#include "internal.h"
#include "paths.cuh"
#include "row_eval.cuh"
#include "solve.h"
#include "utd.cuh"

namespace wcb {

namespace {

constexpr int kB = 256;

WCB_D int row_prim(const RowRec& r) { return (r.component == 1 || r.component == 5) ? r.seq[0] : -1; }

// Canonical key fields, least significant first: edge, primitive,
// sequence[4..0], component, depth, tx, rx.  Object ids are stored +1 (so -1
// maps to 0).
constexpr int kKeyFields = 11;

struct KeyLayout {
    int offset[kKeyFields];
    int bits[kKeyFields];
    int total;
};

WCB_D unsigned long long key_field(const RowRec& r, int f) {
    switch (f) {
        case 0: return static_cast<unsigned long long>(r.edge + 1);
        case 1: return static_cast<unsigned long long>(row_prim(r) + 1);
        case 7: return static_cast<unsigned long long>(r.component & 7);
        case 8: return static_cast<unsigned long long>(r.depth & 7);
        case 9: return static_cast<unsigned long long>(r.tx);
        case 10: return static_cast<unsigned long long>(r.rx);
        default: return static_cast<unsigned long long>(r.seq[6 - f] + 1);  // f = 2..6: seq[4]..seq[0]
    }
}

// largest rx, tx and id + 1 (atomic max into m[0..2], cleared by the caller)
__global__ void k_key_max(long long n, const RowRec* rows, int* m) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int rx = 0, tx = 0, id = 0;
    if (i < n) {
        const RowRec r = rows[i];
        rx = max(r.rx, 0);
        tx = max(r.tx, 0);
        id = max(max(r.edge, row_prim(r)), 0) + 1;
#pragma unroll
        for (int k = 0; k < 5; ++k) id = max(id, r.seq[k] + 1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rx = max(rx, __shfl_xor_sync(0xffffffffu, rx, o));
        tx = max(tx, __shfl_xor_sync(0xffffffffu, tx, o));
        id = max(id, __shfl_xor_sync(0xffffffffu, id, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(m, rx);
        atomicMax(m + 1, tx);
        atomicMax(m + 2, id);
    }
}

// 64-bit word `word` of the concatenated key
__global__ void k_row_key(long long n, const RowRec* rows, const int* order, KeyLayout L, int word,
                          unsigned long long* keys) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const RowRec r = rows[order ? order[i] : i];
    const int lo = 64 * word;
    unsigned long long k = 0;
#pragma unroll
    for (int f = 0; f < kKeyFields; ++f) {
        const int off = L.offset[f], b = L.bits[f];
        if (off + b <= lo || off >= lo + 64) continue;
        const unsigned long long v = key_field(r, f) & (b >= 64 ? ~0ull : ((1ull << b) - 1ull));
        k |= off >= lo ? (v << (off - lo)) : (v >> (lo - off));
    }
    keys[i] = k;
}

__global__ void k_iota(long long n, int* v) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) v[i] = int(i);
}

WCB_D int event_type(int component, int depth, int slot) {
    if (component == 1 && slot < depth) return 1;
    if (component == 2 && depth > 0 && slot == 0) return 2;
    if (component == 5 && slot < depth) return 4;
    return 0;
}

WCB_D bool same_identity(const RowRec& a, const RowRec& b, int width) {
    if (a.tx != b.tx || a.rx != b.rx) return false;
    for (int s = 0; s < width; ++s) {
        const int ta = event_type(a.component, a.depth, s);
        const int tb = event_type(b.component, b.depth, s);
        if (ta != tb) return false;
        const int oa = ta == 0 ? -1 : (a.component == 2 && s == 0 ? a.edge : a.seq[s]);
        const int ob = tb == 0 ? -1 : (b.component == 2 && s == 0 ? b.edge : b.seq[s]);
        if (oa != ob) return false;
    }
    return true;
}

__global__ void k_group_start(long long n, const RowRec* rows, const int* order, int width, int* start) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    start[i] = (i == 0 || !same_identity(rows[order[i - 1]], rows[order[i]], width)) ? 1 : 0;
}

__global__ void k_winner(long long n, const RowRec* rows, const int* order, const int* start, int* keep) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    keep[i] = 0;
    if (!start[i]) return;
    float best = INFINITY;
    bool has_nan = false;
    long long e = i;
    while (e < n && (e == i || !start[e])) {
        const float v = rows[order[e]].length;
        if (isnan(v)) { has_nan = true; break; }
        if (v < best) best = v;
        ++e;
    }
    if (has_nan) return;
    for (long long q = i; q < e; ++q) {
        if (rows[order[q]].length == best) { keep[q] = 1; return; }
    }
}

// per (rx, tx) pair limit on the kept rows (already compacted, canonical)
__global__ void k_pair_limit(long long n, const RowRec* rows, const long long* kept, long long max_paths, int* keep2) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const RowRec r = rows[kept[i]];
    const bool pair_start = i == 0 || rows[kept[i - 1]].rx != r.rx || rows[kept[i - 1]].tx != r.tx;
    if (!pair_start) return;
    long long e = i;
    while (e < n) {
        const RowRec q = rows[kept[e]];
        if (q.rx != r.rx || q.tx != r.tx) break;
        keep2[e] = (e - i) < max_paths ? 1 : 0;
        ++e;
    }
}

__global__ void k_gather_selected(long long n, const int* order, const int* keep, const int* scan, long long* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (keep[i]) out[scan[i] - 1] = order[i];
}

__global__ void k_gather_selected64(long long n, const long long* in, const int* keep, const int* scan, long long* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (keep[i]) out[scan[i] - 1] = in[i];
}

size_t al(size_t x) { return (x + 255) & ~size_t(255); }

struct SelectLayout {
    size_t keys, keys2, idx, idx2, start, keep, scan, tmp, tmp_bytes, kept, total;
};

SelectLayout select_layout(long long n) {
    SelectLayout L;
    size_t o = 0;
    auto take = [&](size_t b) { size_t a = o; o = al(o + b); return a; };
    const size_t m = size_t(std::max<long long>(n, 1));
    L.keys = take(m * 8);
    L.keys2 = take(m * 8);
    L.idx = take(m * 4);
    L.idx2 = take(m * 4);
    L.start = take(m * 4);
    L.keep = take(m * 4);
    L.scan = take(m * 4);
    size_t a = 0, b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long*)nullptr, (unsigned long long*)nullptr, (int*)nullptr,
                                    (int*)nullptr, int(m), 0, 64);
    cub::DeviceScan::InclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, int(m));
    L.tmp_bytes = std::max(a, b);
    L.tmp = take(L.tmp_bytes);
    L.kept = take(m * 8);
    L.total = o;
    return L;
}

}  // namespace

int rows_select_workspace(int64_t n, int64_t* bytes) {
    *bytes = int64_t(select_layout(n).total);
    return 0;
}

namespace {

int bit_width(long long v) {
    int b = 1;
    while (b < 63 && (v >> b) != 0) ++b;
    return b;
}

KeyLayout key_layout(int max_rx, int max_tx, int max_id1) {
    KeyLayout L;
    const int id_bits = bit_width(max_id1);
    const int widths[kKeyFields] = {id_bits, id_bits, id_bits, id_bits, id_bits, id_bits, id_bits, 3, 3,
                                    bit_width(max_tx), bit_width(max_rx)};
    int o = 0;
    for (int f = 0; f < kKeyFields; ++f) {
        L.offset[f] = o;
        L.bits[f] = widths[f];
        o += widths[f];
    }
    L.total = o;
    return L;
}

}  // namespace

int rows_select(const void* rows_v, int64_t n, int width, int64_t max_paths, int scope, int64_t* selected,
                int64_t* num_selected, void* ws, int64_t ws_bytes, cudaStream_t stream) {
    if (n < 0 || n > INT_MAX - 1) return 1;
    const SelectLayout L = select_layout(n);
    if (ws_bytes < int64_t(L.total)) return 3;
    *num_selected = 0;
    if (n == 0) return 0;
    const RowRec* rows = static_cast<const RowRec*>(rows_v);
    char* b = static_cast<char*>(ws);
    auto* keys = reinterpret_cast<unsigned long long*>(b + L.keys);
    auto* keys2 = reinterpret_cast<unsigned long long*>(b + L.keys2);
    int* idx = reinterpret_cast<int*>(b + L.idx);
    int* idx2 = reinterpret_cast<int*>(b + L.idx2);
    int* start = reinterpret_cast<int*>(b + L.start);
    int* keep = reinterpret_cast<int*>(b + L.keep);
    int* scan = reinterpret_cast<int*>(b + L.scan);
    void* tmp = b + L.tmp;
    long long* kept = reinterpret_cast<long long*>(b + L.kept);
    const int grid = int((n + kB - 1) / kB);
    // every CUDA call and launch is checked; any failure returns WCB_ERR_CUDA (2)
    bool ok = true;
    auto chk = [&](cudaError_t e) { ok = ok && e == cudaSuccess; };
    // key widths: the largest rx, tx and id + 1 (in `scan`, free until the dedup)
    int maxima[3] = {0, 0, 0};
    chk(cudaMemsetAsync(scan, 0, 3 * sizeof(int), stream));
    k_key_max<<<grid, kB, 0, stream>>>(n, rows, scan);
    chk(cudaGetLastError());
    chk(cudaMemcpyAsync(maxima, scan, sizeof(maxima), cudaMemcpyDeviceToHost, stream));
    chk(cudaStreamSynchronize(stream));
    if (!ok) return 2;
    const KeyLayout K = key_layout(maxima[0], maxima[1], maxima[2]);
    k_iota<<<grid, kB, 0, stream>>>(n, idx);
    chk(cudaGetLastError());
    note_launch(2);
    const int words = (K.total + 63) / 64;
    for (int w = 0; w < words && ok; ++w) {
        k_row_key<<<grid, kB, 0, stream>>>(n, rows, idx, K, w, keys);
        chk(cudaGetLastError());
        size_t tb = L.tmp_bytes;
        chk(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, idx, idx2, int(n), 0,
                                            std::min(64, K.total - 64 * w), stream));
        std::swap(idx, idx2);
        note_launch(2);
    }
    k_group_start<<<grid, kB, 0, stream>>>(n, rows, idx, width, start);
    chk(cudaGetLastError());
    k_winner<<<grid, kB, 0, stream>>>(n, rows, idx, start, keep);
    chk(cudaGetLastError());
    size_t tb = L.tmp_bytes;
    chk(cub::DeviceScan::InclusiveSum(tmp, tb, keep, scan, int(n), stream));
    k_gather_selected<<<grid, kB, 0, stream>>>(n, idx, keep, scan, kept);
    chk(cudaGetLastError());
    note_launch(4);
    int count = 0;
    chk(cudaMemcpyAsync(&count, scan + n - 1, 4, cudaMemcpyDeviceToHost, stream));
    chk(cudaStreamSynchronize(stream));
    if (!ok) return 2;
    long long final_count = count;
    if (max_paths >= 0 && scope == 0) {
        final_count = std::min<long long>(count, max_paths);
        chk(cudaMemcpyAsync(selected, kept, size_t(final_count) * 8, cudaMemcpyDeviceToDevice, stream));
    } else if (max_paths >= 0 && scope == 1 && count > 0) {
        const int g2 = int((count + kB - 1) / kB);
        chk(cudaMemsetAsync(keep, 0, size_t(count) * 4, stream));
        k_pair_limit<<<g2, kB, 0, stream>>>(count, rows, kept, max_paths, keep);
        chk(cudaGetLastError());
        tb = L.tmp_bytes;
        chk(cub::DeviceScan::InclusiveSum(tmp, tb, keep, scan, int(count), stream));
        k_gather_selected64<<<g2, kB, 0, stream>>>(count, kept, keep, scan, reinterpret_cast<long long*>(selected));
        chk(cudaGetLastError());
        note_launch(3);
        int c2 = 0;
        chk(cudaMemcpyAsync(&c2, scan + count - 1, 4, cudaMemcpyDeviceToHost, stream));
        chk(cudaStreamSynchronize(stream));
        final_count = c2;
    } else {
        chk(cudaMemcpyAsync(selected, kept, size_t(count) * 8, cudaMemcpyDeviceToDevice, stream));
    }
    chk(cudaStreamSynchronize(stream));
    if (!ok) return 2;
    *num_selected = final_count;
    return 0;
}

// ------------------------------------------------------------ evaluation
namespace {

struct EvalParams {
    SceneDev sc;
    const int* edge_slot;  // reference edge id -> selected edge index
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
    double k;
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
    int width;
    wcb_row_fields out;
};

WCB_D V3<double> eval_rx(const EvalParams& p, int r) {
    if (p.rx_kind == 1) {
        const int row = r / p.grid_cols;
        const int col = r - row * p.grid_cols;
        const float u = __fmul_rn(float(row), p.grid_spacing[0]);
        const float v = __fmul_rn(float(col), p.grid_spacing[1]);
        return v3<double>(__fadd_rn(__fadd_rn(p.grid_origin[0], __fmul_rn(p.grid_x[0], u)), __fmul_rn(p.grid_y[0], v)),
                          __fadd_rn(__fadd_rn(p.grid_origin[1], __fmul_rn(p.grid_x[1], u)), __fmul_rn(p.grid_y[1], v)),
                          __fadd_rn(__fadd_rn(p.grid_origin[2], __fmul_rn(p.grid_x[2], u)), __fmul_rn(p.grid_y[2], v)));
    }
    return v3<double>(p.rx_pos[3 * r], p.rx_pos[3 * r + 1], p.rx_pos[3 * r + 2]);
}

WCB_D Slab<float> slab_of(const EvalParams& p, int face) {
    const int m = p.sc.face_material[face];
    return Slab<float>{p.eps_r[m], p.sigma_e[m], p.mu_r[m], p.gain[m], p.thickness[m]};
}

WCB_D void store_c(float* dst, long long i, Cx<float> v) {
    if (dst) { dst[2 * i] = v.re; dst[2 * i + 1] = v.im; }
}

__global__ void k_eval_rows(EvalParams p) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= p.count) return;
    const RowRec row = p.rows[p.selected[i]];
    const int t = row.tx, r = row.rx;
    const SceneDev& sc = p.sc;
    const V3<double> S = v3<double>(p.tx_pos[3 * t], p.tx_pos[3 * t + 1], p.tx_pos[3 * t + 2]);
    const V3<double> R = eval_rx(p, r);
    const V3<float> Sf = cast3<float>(S), Rf = cast3<float>(R);
    const V3<float> tx_pol = v3<float>(p.tx_pol[3 * t], p.tx_pol[3 * t + 1], p.tx_pol[3 * t + 2]);
    const float* rp = p.rx_pol + (long long)r * p.rx_pol_stride;
    const V3<float> rx_pol = v3<float>(rp[0], rp[1], rp[2]);
    const float P = fmaxf(p.tx_power[t], 0.0f);
    const float sq = sqrtf(P);
    C3<float> unit_field;
    Cx<float> coef;
    V3<float> dir;
    double length = 0.0;
    V3<double> hits[kMaxDepth];
    V3<float> normals[kMaxDepth];
    int nh = 0;
    Cx<float> path_field;
    float path_gain;
    const int W = p.width;
    if (row.component == 0) {
        length = wcb::length(R - S);
        const PathEval<float> ev = eval_free_space(Sf, Rf, tx_pol, rx_pol, p.k, length);
        unit_field = ev.field;
        coef = ev.coefficient;
        dir = ev.direction;
        path_field = coef * sq;
        path_gain = cabs2(path_field);
    } else if (row.component == 1) {
        const int d = row.depth;
        const ReflectionGeom g = reflection_geometry(sc, row.seq, d, S, R);
        for (int k = 0; k < d; ++k) hits[k] = g.hits[k];
        nh = d;
        length = g.length;
        reflection_field(sc, row.seq, d, g, Sf, Rf, tx_pol, rx_pol, [&](int f) { return slab_of(p, f); }, p.freq, p.k,
                         normals, &unit_field, &coef, &dir);
        path_field = coef * sq;
        path_gain = cabs2(path_field);
    } else if (row.component == 5) {
        const int d = row.depth;
        length = wcb::length(R - S);
        dir = safe_normalize(Rf - Sf, v3(0.f, 0.f, 1.f));
        C3<float> value = c3_from_real(transverse(dir, tx_pol));
        float shorten = 0.0f;
        const LayerTable<float> lt{p.layer_offset, p.layer_count, p.layer_thickness, p.layer_eps_r, p.layer_sigma_e, p.layer_mu_r};
        const V3<double> seg = R - S;
        for (int k = 0; k < d; ++k) {
            const int f = row.seq[k];
            const float* nf = sc.face_normal + 3 * f;
            normals[k] = v3(nf[0], nf[1], nf[2]);
            const double* pl = sc.face_plane + 4 * f;
            const V3<double> n = v3(pl[0], pl[1], pl[2]);
            const double den = dot(seg, n);
            const double tt = den != 0.0 ? (pl[3] - dot(S, n)) / den : 0.0;
            hits[k] = S + seg * tt;
            transmit_wall(value, shorten, dir, normals[k], sc.face_material[f], lt, p.freq);
        }
        nh = d;
        const float amp = 1.0f / (2.0f * float(p.k) * float(fmax(length, kUtdEps)));
        value = c3_scale(value, phasor_neg_kd<float>(p.k, length - double(shorten)) * amp);
        unit_field = value;
        coef = project_receiver(value, dir, rx_pol);
        path_field = coef * sq;
        path_gain = cabs2(path_field);
    } else {
        const int slot = p.edge_slot[row.edge];
        const EdgeDev& ed = sc.edges[slot];
        const DiffractionResult<float> res = utd_field<float>(ed, S, R, tx_pol, slab_of(p, ed.mat_face0), slab_of(p, ed.mat_face1), p.freq);
        length = res.length;
        const V3<double> q = v3(res.q[0], res.q[1], res.q[2]);
        hits[0] = q;
        normals[0] = v3(0.f, 0.f, 0.f);
        nh = 1;
        dir = safe_normalize(cast3<float>(R - q), v3(0.f, 0.f, 1.f));
        const C3<float> powered = c3_scale(res.field, cx(sq, 0.0f));
        path_field = project_receiver(powered, dir, rx_pol);
        path_gain = cabs2(path_field);
        const float amp = sqrtf(fmaxf(P, 1e-30f));
        unit_field = c3_scale(powered, cx(1.0f / amp, 0.0f));
        coef = path_field * (1.0f / amp);
    }
    const wcb_row_fields& o = p.out;
    if (o.path_length_m) o.path_length_m[i] = float(length);
    if (o.delay_s) o.delay_s[i] = float(length / kC0);
    if (o.path_gain) o.path_gain[i] = path_gain;
    store_c(o.path_field, i, path_field);
    store_c(o.coefficient, i, coef);
    if (o.field_xyz) {
        store_c(o.field_xyz, 3 * i + 0, unit_field.x);
        store_c(o.field_xyz, 3 * i + 1, unit_field.y);
        store_c(o.field_xyz, 3 * i + 2, unit_field.z);
    }
    if (o.field_direction) {
        o.field_direction[3 * i] = dir.x;
        o.field_direction[3 * i + 1] = dir.y;
        o.field_direction[3 * i + 2] = dir.z;
    }
    for (int k = 0; k < W; ++k) {
        const bool on = k < nh;
        if (o.interaction_positions) {
            float* d = o.interaction_positions + (i * W + k) * 3;
            d[0] = on ? float(hits[k].x) : 0.f;
            d[1] = on ? float(hits[k].y) : 0.f;
            d[2] = on ? float(hits[k].z) : 0.f;
        }
        if (o.interaction_normals) {
            float* d = o.interaction_normals + (i * W + k) * 3;
            d[0] = on ? normals[k].x : 0.f;
            d[1] = on ? normals[k].y : 0.f;
            d[2] = on ? normals[k].z : 0.f;
        }
    }
    if (o.phase_rad) {
        float ph = -atan2f(path_field.im, path_field.re);
        const float tp = float(kTwoPi);
        ph = fmodf(ph, tp);
        if (ph < 0.0f) ph += tp;
        o.phase_rad[i] = ph;
    }
}

// deterministic per-cell accumulation over canonical rows
__global__ void k_accumulate_rows(const RowRec* rows, const long long* sel, long long n, const float* path_gain,
                                  const float* path_field, const float* field_xyz, const float* tx_power, int num_tx,
                                  int num_rx, int coherent,
                                  float* out_pg, float* out_field, float* out_cp, float* out_cf, float* out_dv) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long cells = (long long)num_tx * num_rx;
    if (cell >= cells) return;
    const int t = int(cell / num_rx);
    const int r = int(cell - (long long)t * num_rx);
    // rows are sorted by (rx, tx): lower bound of (r, t)
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        const RowRec m = rows[sel[mid]];
        if (m.rx < r || (m.rx == r && m.tx < t)) lo = mid + 1;
        else hi = mid;
    }
    Cx<float> slot[4] = {cx(0.f, 0.f), cx(0.f, 0.f), cx(0.f, 0.f), cx(0.f, 0.f)};
    float gain[4] = {0.f, 0.f, 0.f, 0.f};
    Cx<float> dv[3] = {cx(0.f, 0.f), cx(0.f, 0.f), cx(0.f, 0.f)};
    const float amp = tx_power ? sqrtf(fmaxf(tx_power[t], 0.f)) : 1.f;
    for (long long q = lo; q < n; ++q) {
        const RowRec m = rows[sel[q]];
        if (m.rx != r || m.tx != t) break;
        const int s = m.component == 0 ? 0 : m.component == 1 ? 1 : m.component == 2 ? 2 : m.component == 5 ? 3 : -1;
        if (s < 0) continue;
        const Cx<float> pf = cx(path_field[2 * q], path_field[2 * q + 1]);
        slot[s] = slot[s] + pf;
        gain[s] += path_gain[q];
        if (s == 2 && field_xyz) {
            // field_xyz is unit excitation; the exact vector sum uses the powered field
            dv[0] = dv[0] + cx(field_xyz[6 * q + 0], field_xyz[6 * q + 1]) * amp;
            dv[1] = dv[1] + cx(field_xyz[6 * q + 2], field_xyz[6 * q + 3]) * amp;
            dv[2] = dv[2] + cx(field_xyz[6 * q + 4], field_xyz[6 * q + 5]) * amp;
        }
    }
    Cx<float> total = cx(0.f, 0.f);
    float gsum = 0.f;
    for (int s = 0; s < 4; ++s) {
        total = total + slot[s];
        gsum += gain[s];
    }
    if (out_pg) out_pg[cell] = coherent ? cabs2(total) : gsum;
    if (out_field) {
        out_field[2 * cell] = coherent ? total.re : sqrtf(fmaxf(gsum, 0.f));
        out_field[2 * cell + 1] = coherent ? total.im : 0.f;
    }
    for (int s = 0; s < 6; ++s) {
        const long long o = s * cells + cell;
        const Cx<float> v = s < 4 ? slot[s] : cx(0.f, 0.f);
        if (out_cp) out_cp[o] = s < 4 ? (coherent ? cabs2(v) : gain[s]) : 0.f;
        if (out_cf) { out_cf[2 * o] = v.re; out_cf[2 * o + 1] = v.im; }
    }
    if (out_dv) out_dv[cell] = cabs2(dv[0]) + cabs2(dv[1]) + cabs2(dv[2]);
}

// ------------------------------------------------------------ field operators
__global__ void k_field_free_space(long long n, const float* src, const float* tgt, const float* pw, const float* tpol,
                                   const float* rpol, double freq, float* fv, float* coef, float* pf, float* pg,
                                   float* plen, float* delay, float* dirout) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<double> S = v3<double>(src[3 * i], src[3 * i + 1], src[3 * i + 2]);
    const V3<double> R = v3<double>(tgt[3 * i], tgt[3 * i + 1], tgt[3 * i + 2]);
    const double k = kTwoPi * freq / kC0;
    const double dist = length(R - S);
    const PathEval<float> ev = eval_free_space(cast3<float>(S), cast3<float>(R), v3(tpol[3 * i], tpol[3 * i + 1], tpol[3 * i + 2]),
                                               v3(rpol[3 * i], rpol[3 * i + 1], rpol[3 * i + 2]), k, dist);
    const float sq = sqrtf(fmaxf(pw[i], 0.f));
    const Cx<float> p = ev.coefficient * sq;
    store_c(fv, 3 * i, ev.field.x);
    store_c(fv, 3 * i + 1, ev.field.y);
    store_c(fv, 3 * i + 2, ev.field.z);
    store_c(coef, i, ev.coefficient);
    store_c(pf, i, p);
    if (pg) pg[i] = cabs2(p);
    if (plen) plen[i] = float(dist);
    if (delay) delay[i] = float(dist / kC0);
    if (dirout) { dirout[3 * i] = ev.direction.x; dirout[3 * i + 1] = ev.direction.y; dirout[3 * i + 2] = ev.direction.z; }
}

__global__ void k_field_reflection(long long n, int depth, const float* src, const float* tgt, const float* pos,
                                   const float* nrm, const float* pw, const float* tpol, const float* rpol,
                                   const float* eps, const float* sig, const float* mu, const float* gain,
                                   const float* th, double freq, float* fv, float* coef, float* pf, float* pg,
                                   float* plen, float* delay, float* dirout) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<float> S = v3(src[3 * i], src[3 * i + 1], src[3 * i + 2]);
    const V3<float> R = v3(tgt[3 * i], tgt[3 * i + 1], tgt[3 * i + 2]);
    const V3<float> tx_pol = v3(tpol[3 * i], tpol[3 * i + 1], tpol[3 * i + 2]);
    const V3<float> rx_pol = v3(rpol[3 * i], rpol[3 * i + 1], rpol[3 * i + 2]);
    const double k = kTwoPi * freq / kC0;
    const float wl = float(kC0 / freq);
    auto hit = [&](int b) { const float* h = pos + (i * depth + b) * 3; return v3(h[0], h[1], h[2]); };
    V3<float> prev = S;
    V3<float> incident = safe_normalize(hit(0) - prev, v3(0.f, 0.f, 1.f));
    C3<float> value = c3_from_real(transverse(incident, tx_pol));
    V3<float> outgoing = incident;
    double total = 0.0;
    V3<double> prevd = cast3<double>(S);
    for (int b = 0; b < depth; ++b) {
        const V3<float> h = hit(b);
        incident = safe_normalize(h - prev, outgoing);
        total += length(cast3<double>(h) - prevd);
        const float* nn = nrm + (i * depth + b) * 3;
        const long long s = i * depth + b;
        reflect_bounce(value, outgoing, incident, v3(nn[0], nn[1], nn[2]), Slab<float>{eps[s], sig[s], mu[s], gain[s], th[s]}, freq, wl);
        prev = h;
        prevd = cast3<double>(h);
    }
    const V3<float> fdir = safe_normalize(R - prev, outgoing);
    total += length(cast3<double>(R) - prevd);
    const float amp = 1.0f / (2.0f * float(k) * float(fmax(total, kUtdEps)));
    value = c3_scale(value, phasor_neg_kd<float>(k, total) * amp);
    const Cx<float> c = project_receiver(value, fdir, rx_pol);
    const Cx<float> p = c * sqrtf(fmaxf(pw[i], 0.f));
    store_c(fv, 3 * i, value.x);
    store_c(fv, 3 * i + 1, value.y);
    store_c(fv, 3 * i + 2, value.z);
    store_c(coef, i, c);
    store_c(pf, i, p);
    if (pg) pg[i] = cabs2(p);
    if (plen) plen[i] = float(total);
    if (delay) delay[i] = float(total / kC0);
    if (dirout) { dirout[3 * i] = fdir.x; dirout[3 * i + 1] = fdir.y; dirout[3 * i + 2] = fdir.z; }
}

__global__ void k_field_transmission(long long n, int depth, const float* src, const float* tgt, const float* nrm,
                                     const int* mids, const int* counts, const float* pw, const float* tpol,
                                     const float* rpol, LayerTable<float> lt, double freq, float* fv, float* coef,
                                     float* pf, float* pg, float* plen, float* delay, float* dirout) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<double> S = v3<double>(src[3 * i], src[3 * i + 1], src[3 * i + 2]);
    const V3<double> R = v3<double>(tgt[3 * i], tgt[3 * i + 1], tgt[3 * i + 2]);
    const double k = kTwoPi * freq / kC0;
    const double dist = length(R - S);
    const V3<float> dir = safe_normalize(cast3<float>(R) - cast3<float>(S), v3(0.f, 0.f, 1.f));
    C3<float> value = c3_from_real(transverse(dir, v3(tpol[3 * i], tpol[3 * i + 1], tpol[3 * i + 2])));
    float shorten = 0.f;
    const int cnt = counts[i] < depth ? counts[i] : depth;
    for (int w = 0; w < cnt; ++w) {
        const float* nn = nrm + (i * depth + w) * 3;
        transmit_wall(value, shorten, dir, v3(nn[0], nn[1], nn[2]), mids[i * depth + w], lt, freq);
    }
    const float amp = 1.0f / (2.0f * float(k) * float(fmax(dist, kUtdEps)));
    value = c3_scale(value, phasor_neg_kd<float>(k, dist - double(shorten)) * amp);
    const Cx<float> c = project_receiver(value, dir, v3(rpol[3 * i], rpol[3 * i + 1], rpol[3 * i + 2]));
    const Cx<float> p = c * sqrtf(fmaxf(pw[i], 0.f));
    store_c(fv, 3 * i, value.x);
    store_c(fv, 3 * i + 1, value.y);
    store_c(fv, 3 * i + 2, value.z);
    store_c(coef, i, c);
    store_c(pf, i, p);
    if (pg) pg[i] = cabs2(p);
    if (plen) plen[i] = float(dist);
    if (delay) delay[i] = float(dist / kC0);
    if (dirout) { dirout[3 * i] = dir.x; dirout[3 * i + 1] = dir.y; dirout[3 * i + 2] = dir.z; }
}

__global__ void k_field_project(long long n, const float* fv, const float* dir, const float* rpol, float* coef, float* pg) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const C3<float> v = {cx(fv[6 * i], fv[6 * i + 1]), cx(fv[6 * i + 2], fv[6 * i + 3]), cx(fv[6 * i + 4], fv[6 * i + 5])};
    const Cx<float> c = project_receiver(v, v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]), v3(rpol[3 * i], rpol[3 * i + 1], rpol[3 * i + 2]));
    store_c(coef, i, c);
    if (pg) pg[i] = cabs2(c);
}

WCB_D void store_frame(float* dst, long long i, V3<float> u, V3<float> v) {
    dst[6 * i] = u.x;
    dst[6 * i + 1] = u.y;
    dst[6 * i + 2] = u.z;
    dst[6 * i + 3] = v.x;
    dst[6 * i + 4] = v.y;
    dst[6 * i + 5] = v.z;
}

// LoS Jones operator rows: row i takes pair p (source p % S, sink p / S),
// evaluates the unit-excitation free-space field of both source frame
// vectors (FP64 length and phase, as the LoS kernel) and projects each on
// both sink frame vectors: matrix[i][a][b] = response of sink vector a to
// source vector b.  A pair outside [0, S*R) writes NaN and sets status bit 0.
__global__ void k_los_jones(long long n, const long long* pair, const float* src, long long num_src, const float* snk,
                            long long num_snk, const float* src_ref, const float* snk_ref, double freq, float* matrix,
                            float* src_basis, float* snk_basis, int* status) {
    const long long stride = (long long)blockDim.x * gridDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long p = pair[i];
        if (p < 0 || p >= num_src * num_snk) {
            const float nan = __int_as_float(0x7fc00000);
            for (int j = 0; j < 8; ++j) matrix[8 * i + j] = nan;
            for (int j = 0; j < 6; ++j) {
                src_basis[6 * i + j] = nan;
                snk_basis[6 * i + j] = nan;
            }
            if (status) atomicOr(status, 1);
            continue;
        }
        const long long t = p % num_src;
        const long long r = p / num_src;
        const V3<double> S = v3<double>(src[3 * t], src[3 * t + 1], src[3 * t + 2]);
        const V3<double> R = v3<double>(snk[3 * r], snk[3 * r + 1], snk[3 * r + 2]);
        const double k = kTwoPi * freq / kC0;
        const double dist = length(R - S);
        const V3<float> Sf = cast3<float>(S);
        const V3<float> Rf = cast3<float>(R);
        const V3<float> dir = safe_normalize(Rf - Sf, v3<float>(0.f, 0.f, 1.f));
        V3<float> su, sv, ru, rv;
        endpoint_frame(src_ref, t, dir, &su, &sv);
        endpoint_frame(snk_ref, r, dir, &ru, &rv);
        const PathEval<float> eu = eval_free_space(Sf, Rf, su, ru, k, dist);
        const PathEval<float> ev = eval_free_space(Sf, Rf, sv, ru, k, dist);
        store_c(matrix, 4 * i + 0, eu.coefficient);
        store_c(matrix, 4 * i + 1, ev.coefficient);
        store_c(matrix, 4 * i + 2, project_receiver(eu.field, eu.direction, rv));
        store_c(matrix, 4 * i + 3, project_receiver(ev.field, ev.direction, rv));
        store_frame(src_basis, i, su, sv);
        store_frame(snk_basis, i, ru, rv);
    }
}

}  // namespace

int rows_evaluate(const SceneHandle* h, const wcb_solve_desc* d, const wcb_materials* m, int fi, const void* rows,
                  const int64_t* selected, int64_t count, int width, const wcb_row_fields* out, cudaStream_t stream) {
    if (count <= 0) return 0;
    if (fi < 0 || fi >= d->num_freq) return 1;
    EvalParams p;
    std::memset(&p, 0, sizeof(p));
    p.sc = h->dev;
    p.edge_slot = h->edge_slot;
    p.tx_pos = d->tx_pos;
    p.tx_power = d->tx_power;
    p.tx_pol = d->tx_pol;
    p.rx_kind = d->rx_kind;
    p.rx_pos = d->rx_pos;
    for (int k = 0; k < 3; ++k) {
        p.grid_origin[k] = d->grid_origin[k];
        p.grid_x[k] = d->grid_x_axis[k];
        p.grid_y[k] = d->grid_y_axis[k];
    }
    p.grid_rows = d->grid_rows;
    p.grid_cols = d->grid_cols;
    p.grid_spacing[0] = d->grid_spacing[0];
    p.grid_spacing[1] = d->grid_spacing[1];
    p.rx_pol = d->rx_pol;
    p.rx_pol_stride = d->rx_pol_stride;
    p.freq = d->frequency_hz[fi];
    p.k = kTwoPi * p.freq / kC0;
    const long long mo = (long long)fi * m->num_materials;
    p.num_materials = m->num_materials;
    p.eps_r = m->eps_r + mo;
    p.sigma_e = m->sigma_e + mo;
    p.mu_r = m->mu_r + mo;
    p.gain = m->gain + mo;
    p.thickness = m->thickness + mo;
    const long long lo = (long long)fi * m->num_layers;
    p.num_layers = m->num_layers;
    p.layer_offset = m->layer_offset;
    p.layer_count = m->layer_count;
    p.layer_thickness = m->layer_thickness ? m->layer_thickness + lo : nullptr;
    p.layer_eps_r = m->layer_eps_r ? m->layer_eps_r + lo : nullptr;
    p.layer_sigma_e = m->layer_sigma_e ? m->layer_sigma_e + lo : nullptr;
    p.layer_mu_r = m->layer_mu_r ? m->layer_mu_r + lo : nullptr;
    p.rows = static_cast<const RowRec*>(rows);
    p.selected = reinterpret_cast<const long long*>(selected);
    p.count = count;
    p.width = width;
    p.out = *out;
    k_eval_rows<<<int((count + kB - 1) / kB), kB, 0, stream>>>(p);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int rows_accumulate(const void* rows, const int64_t* selected, int64_t n, const float* path_gain, const float* path_field,
                    const float* field_xyz, const float* tx_power, int num_tx, int num_rx, int coherent,
                    const wcb_outputs* out, cudaStream_t stream) {
    const long long cells = (long long)num_tx * num_rx;
    if (cells <= 0) return 0;
    k_accumulate_rows<<<int((cells + kB - 1) / kB), kB, 0, stream>>>(
        static_cast<const RowRec*>(rows), reinterpret_cast<const long long*>(selected), n, path_gain, path_field, field_xyz,
        tx_power, num_tx, num_rx, coherent, static_cast<float*>(out->path_gain), static_cast<float*>(out->field),
        static_cast<float*>(out->comp_power), static_cast<float*>(out->comp_field), static_cast<float*>(out->diff_vec_power));
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int field_free_space(int64_t n, const float* s, const float* t, const float* pw, const float* tp, const float* rp, double f,
                     float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr, cudaStream_t stream) {
    if (n <= 0) return 0;
    k_field_free_space<<<int((n + kB - 1) / kB), kB, 0, stream>>>(n, s, t, pw, tp, rp, f, fv, c, pf, pg, pl, dl, dr);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int field_reflection(int64_t n, int depth, const float* s, const float* t, const float* pos, const float* nrm, const float* pw,
                     const float* tp, const float* rp, const float* eps, const float* sig, const float* mu, const float* gain,
                     const float* th, double f, float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr,
                     cudaStream_t stream) {
    if (n <= 0) return 0;
    if (depth < 1 || depth > kMaxDepth) return 1;
    k_field_reflection<<<int((n + kB - 1) / kB), kB, 0, stream>>>(n, depth, s, t, pos, nrm, pw, tp, rp, eps, sig, mu, gain, th,
                                                                   f, fv, c, pf, pg, pl, dl, dr);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int field_transmission(int64_t n, int depth, const float* s, const float* t, const float* nrm, const int* mids,
                       const int* counts, const float* pw, const float* tp, const float* rp, const wcb_materials* m,
                       double f, float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr,
                       cudaStream_t stream) {
    if (n <= 0) return 0;
    if (depth < 1 || depth > kMaxDepth) return 1;
    const LayerTable<float> lt{m->layer_offset, m->layer_count, m->layer_thickness, m->layer_eps_r, m->layer_sigma_e,
                               m->layer_mu_r};
    k_field_transmission<<<int((n + kB - 1) / kB), kB, 0, stream>>>(n, depth, s, t, nrm, mids, counts, pw, tp, rp, lt, f,
                                                                     fv, c, pf, pg, pl, dl, dr);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int field_project(int64_t n, const float* fv, const float* dir, const float* rp, float* c, float* pg, cudaStream_t stream) {
    if (n <= 0) return 0;
    k_field_project<<<int((n + kB - 1) / kB), kB, 0, stream>>>(n, fv, dir, rp, c, pg);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int los_jones(int64_t n, const int64_t* pair, const float* src, int64_t num_src, const float* snk, int64_t num_snk,
              const float* src_ref, const float* snk_ref, double f, float* matrix, float* src_basis, float* snk_basis,
              int* status, cudaStream_t stream) {
    if (n <= 0) return 0;
    // grid-stride: at most 8 blocks of 256 per SM on the 148 SMs
    const long long blocks = std::min<long long>((n + kB - 1) / kB, 148LL * 8);
    k_los_jones<<<int(blocks), kB, 0, stream>>>(n, reinterpret_cast<const long long*>(pair), src, num_src, snk, num_snk,
                                                src_ref, snk_ref, f, matrix, src_basis, snk_basis, status);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Columns of the selected records in one pass (thread per selected record):
// the records are read once, in selection order, and every column written
// contiguously.  Any output pointer may be NULL.
namespace {
__global__ void k_rows_decode(const RowRec* rows, const int64_t* selected, long long n, int* tx, int* rx, int* comp,
                              int* depth, int* seq, int* edge, float* len) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const RowRec r = rows[selected[i]];
    if (tx) tx[i] = r.tx;
    if (rx) rx[i] = r.rx;
    if (comp) comp[i] = int(r.component);
    if (depth) depth[i] = int(r.depth);
    if (seq)
        for (int k = 0; k < 5; ++k) seq[5 * i + k] = r.seq[k];
    if (edge) edge[i] = r.edge;
    if (len) len[i] = r.length;
}
}  // namespace

int rows_decode(const void* rows, const int64_t* selected, int64_t n, int32_t* tx, int32_t* rx, int32_t* component,
                int32_t* depth, int32_t* seq, int32_t* edge, float* length, cudaStream_t stream) {
    if (n < 0 || (n > 0 && (rows == nullptr || selected == nullptr))) return 1;
    if (n == 0) return 0;
    k_rows_decode<<<unsigned((n + 255) / 256), 256, 0, stream>>>(static_cast<const RowRec*>(rows), selected, n, tx, rx,
                                                                   component, depth, seq, edge, length);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace wcb
