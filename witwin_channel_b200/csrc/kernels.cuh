// Per-component solve kernels with in-warp compaction.
//
// A warp owns a tile of 32 receiver cells of one transmitter (an 8x4 patch of
// a receiver grid, or 32 consecutive points).  Lanes test candidates for
// their own cells; the survivors are appended to a per-warp queue in shared
// memory (ballot + popc) and processed 32 at a time with every lane busy.  A
// processed item's contribution is written to a per-warp buffer and gathered
// by the lane that owns the item's cell in item order, so every cell sums its
// paths in a fixed order (deterministic) and each slot of each cell is written
// once.  Each component runs in its own kernel so the code a warp executes
// stays small.
#pragma once

#include "em.cuh"
#include "paths.cuh"
#include "solve.h"
#include "utd.cuh"

namespace wcb {

constexpr int kWarpsPerBlock = 4;              // LoS/transmission: one tile per warp
constexpr int kCompBlock = kWarpsPerBlock * 32;
constexpr int kSplitWarps = 8;                 // reflection/diffraction: one tile per block,
constexpr int kSplitBlock = kSplitWarps * 32;  // its candidates interleaved over 8 warps
constexpr int kQueueCap = 64;
constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ common
template <typename T>
WCB_D Slab<T> face_slab(const MainParams& p, int f_index, int face) {
    const int m = p.sc.face_material[face];
    const long long o = (long long)f_index * p.num_materials + m;
    return Slab<T>{T(p.mat_eps_r[o]), T(p.mat_sigma_e[o]), T(p.mat_mu_r[o]), T(p.mat_gain[o]), T(p.mat_thickness[o])};
}

// Layer tables of frequency f_index (FP32 values; an FP64 solve widens them
// on load, which is exact).
WCB_D LayerTable<float> layer_table_f(const MainParams& p, int f_index) {
    const long long o = (long long)f_index * p.num_layers;
    return LayerTable<float>{p.layer_offset, p.layer_count, p.layer_thickness + o, p.layer_eps_r + o,
                             p.layer_sigma_e + o, p.layer_mu_r + o};
}

WCB_D void emit_row(const MainParams& p, int t, int r, int cid, int depth, const int* seq, int edge, float length) {
    if (p.rows == nullptr) return;
    const unsigned long long idx = atomicAdd(p.row_counter, 1ull);
    if (idx >= (unsigned long long)p.row_capacity) return;
    RowRec rec;
    rec.tx = t;
    rec.rx = r;
    rec.component = short(cid);
    rec.depth = short(depth);
    for (int k = 0; k < kMaxDepth; ++k) rec.seq[k] = k < depth && seq ? seq[k] : -1;
    rec.edge = edge;
    rec.length = length;
    rec.pad = 0;
    rec.pad2 = 0;
    p.rows[idx] = rec;
}

// receiver point (float, formed like the reference's grid kernel)
WCB_D V3<float> rx_point(const MainParams& p, int r) {
    if (p.rx_kind == 1) {
        const int row = r / p.grid_cols;
        const int col = r - row * p.grid_cols;
        const float u = __fmul_rn(float(row), p.grid_spacing[0]);
        const float v = __fmul_rn(float(col), p.grid_spacing[1]);
        return v3(__fadd_rn(__fadd_rn(p.grid_origin[0], __fmul_rn(p.grid_x[0], u)), __fmul_rn(p.grid_y[0], v)),
                  __fadd_rn(__fadd_rn(p.grid_origin[1], __fmul_rn(p.grid_x[1], u)), __fmul_rn(p.grid_y[1], v)),
                  __fadd_rn(__fadd_rn(p.grid_origin[2], __fmul_rn(p.grid_x[2], u)), __fmul_rn(p.grid_y[2], v)));
    }
    return v3(p.rx_pos[3 * r], p.rx_pos[3 * r + 1], p.rx_pos[3 * r + 2]);
}

// number of 32-cell tiles per transmitter
WCB_HD long long tiles_per_tx(const MainParams& p) {
    if (p.rx_kind == 1) return (long long)((p.grid_rows + 7) / 8) * ((p.grid_cols + 3) / 4);
    return (p.num_rx + 31) / 32;
}

// cell of (tile, lane); false for lanes past the grid edge
WCB_D bool tile_cell(const MainParams& p, long long tile_global, int lane, int* t, int* r) {
    const long long per_tx = tiles_per_tx(p);
    const long long tt = tile_global / per_tx;
    if (tt >= p.num_tx) return false;
    const long long tile = tile_global - tt * per_tx;
    *t = int(tt);
    if (p.rx_kind == 1) {
        const int tiles_c = (p.grid_cols + 3) / 4;
        const int tr = int(tile / tiles_c), tc = int(tile - (long long)tr * tiles_c);
        const int row = tr * 8 + lane / 4;
        const int col = tc * 4 + (lane & 3);
        if (row >= p.grid_rows || col >= p.grid_cols) return false;
        *r = row * p.grid_cols + col;
        return true;
    }
    const long long r64 = tile * 32 + lane;
    if (r64 >= p.num_rx) return false;
    *r = int(r64);
    return true;
}

WCB_D unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Append (lane, cand, aux) for every lane with `pass`; returns the new size.
WCB_D int queue_push(int* q, int size, bool pass, int a, int b, int c) {
    const unsigned mask = __ballot_sync(kFull, pass);
    if (pass) {
        const int pos = size + __popc(mask & lanemask_lt());
        q[3 * pos] = a;
        q[3 * pos + 1] = b;
        q[3 * pos + 2] = c;
    }
    __syncwarp();
    return size + __popc(mask);
}

// Remove the first `n` items (n <= 32) from a queue of `size` items.
WCB_D int queue_pop(int* q, int size, int n, int lane) {
    const int rem = size - n;
    int a = 0, b = 0, c = 0;
    if (lane < rem) {
        a = q[3 * (n + lane)];
        b = q[3 * (n + lane) + 1];
        c = q[3 * (n + lane) + 2];
    }
    __syncwarp();
    if (lane < rem) {
        q[3 * lane] = a;
        q[3 * lane + 1] = b;
        q[3 * lane + 2] = c;
    }
    __syncwarp();
    return rem;
}

template <typename T>
WCB_D void store_slot(const MainParams& p, int slot, int f, long long cell, Cx<T> v, T gain, bool coherent) {
    const long long cells = (long long)p.num_tx * p.num_rx;
    const long long fc = (long long)(p.freq_base + f) * cells + cell;
    const long long o = (long long)slot * p.num_freq_total * cells + fc;
    T* cp = static_cast<T*>(p.out_comp_power);
    T* cf = static_cast<T*>(p.out_comp_field);
    if (cp) cp[o] = coherent ? cabs2(v) : gain;
    if (cf) {
        cf[2 * o] = v.re;
        cf[2 * o + 1] = v.im;
    }
}

// ------------------------------------------------------------------ LoS + transmission
template <typename T, int NF>
__global__ void __launch_bounds__(kCompBlock) k_los_trans(MainParams p) {
    extern __shared__ int smem[];
    int* stack = smem;
    const int lane = threadIdx.x & 31;
    const long long tile = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    int t, r;
    if (!tile_cell(p, tile, lane, &t, &r)) return;
    const SceneDev& sc = p.sc;
    int* err = p.status;
    const V3<double> S = v3<double>(p.tx_pos[3 * t], p.tx_pos[3 * t + 1], p.tx_pos[3 * t + 2]);
    const V3<float> Rf = rx_point(p, r);
    const V3<double> R = cast3<double>(Rf);
    const V3<T> ST = cast3<T>(S), RT = cast3<T>(R);
    const V3<T> tx_pol = v3<T>(T(p.tx_pol[3 * t]), T(p.tx_pol[3 * t + 1]), T(p.tx_pol[3 * t + 2]));
    const float* rp = p.rx_pol + (long long)r * p.rx_pol_stride;
    const V3<T> rx_pol = v3<T>(T(rp[0]), T(rp[1]), T(rp[2]));
    const T sqrt_p = s_sqrt(s_max(T(p.tx_power[t]), T(0)));
    const long long cell = (long long)t * p.num_rx + r;
    unsigned long long rays = 0;
    if (p.components & 1) {
        Cx<T> acc[NF];
        T gain[NF];
        for (int f = 0; f < NF; ++f) { acc[f] = cx(T(0), T(0)); gain[f] = T(0); }
        const bool blocked = sc.num_faces > 0 && segment_blocked<T>(sc, ST, RT, ignore_none(), stack, err);
        if (sc.num_faces > 0) ++rays;
        if (!blocked) {
            const double dist = length(R - S);
#pragma unroll 1
            for (int f = 0; f < NF; ++f) {
                const PathEval<T> ev = eval_free_space(ST, RT, tx_pol, rx_pol, p.k[f], dist);
                const Cx<T> pf = ev.coefficient * sqrt_p;
                acc[f] = pf;
                gain[f] = cabs2(pf);
            }
            emit_row(p, t, r, 0, 0, nullptr, -1, float(dist));
        }
        for (int f = 0; f < NF; ++f) store_slot(p, 0, f, cell, acc[f], gain[f], p.coherent);
    }
    if ((p.components & 8) && p.max_depth >= 1) {
        Cx<T> acc[NF];
        T gain[NF];
        for (int f = 0; f < NF; ++f) { acc[f] = cx(T(0), T(0)); gain[f] = T(0); }
        if (sc.num_faces > 0) {
            HitList hl;
            ++rays;
            segment_hits<T>(sc, ST, RT, p.max_depth, &hl, stack, err);
            if (hl.count > p.max_depth) {
                if (p.overflow_counter) atomicAdd(p.overflow_counter, 1ull);
            } else if (hl.count >= 1) {
                bool ok = true;
                for (int i = 0; i < hl.count; ++i) {
                    const int m = sc.face_material[hl.face[i]];
                    if (p.mat_volumetric && p.mat_volumetric[m]) ok = false;
                }
                if (ok) {
                    const double dist = length(R - S);
                    const V3<T> dir = safe_normalize(RT - ST, v3<T>(T(0), T(0), T(1)));
#pragma unroll 1
                    for (int f = 0; f < NF; ++f) {
                        C3<T> value = c3_from_real(transverse(dir, tx_pol));
                        T shorten = T(0);
                        const LayerTable<float> lt = layer_table_f(p, f);
                        for (int i = 0; i < hl.count; ++i) {
                            const float* nf = sc.face_normal + 3 * hl.face[i];
                            transmit_wall(value, shorten, dir, v3<T>(T(nf[0]), T(nf[1]), T(nf[2])),
                                          sc.face_material[hl.face[i]], lt, p.freq[f]);
                        }
                        const T amp = T(1) / (T(2) * T(p.k[f]) * T(fmax(dist, kUtdEps)));
                        value = c3_scale(value, phasor_neg_kd<T>(p.k[f], dist - double(value_of(shorten))) * amp);
                        const Cx<T> pf = project_receiver(value, dir, rx_pol) * sqrt_p;
                        acc[f] = pf;
                        gain[f] = cabs2(pf);
                    }
                    emit_row(p, t, r, 5, hl.count, hl.face, -1, float(dist));
                }
            }
        }
        for (int f = 0; f < NF; ++f) store_slot(p, 3, f, cell, acc[f], gain[f], p.coherent);
    }
    if (p.ray_counter && p.freq_base == 0 && rays) atomicAdd(p.ray_counter, rays);
}

// ------------------------------------------------------------------ reflection
// Per-warp shared layout: queue A (3 ints/item), queue B (3 + 5 ints/item),
// queue F (3 + 5 ints/item), contribution buffer (32 items x NF x 3 floats).
template <int NF>
struct ReflShared {
    int qa[3 * kQueueCap];
    int qb[3 * kQueueCap];
    int qbf[kMaxDepth * kQueueCap];
    int qf[3 * kQueueCap];
    int qff[kMaxDepth * kQueueCap];
    float contrib[32 * NF * 3];
    int owner[32];
};

// Append the passing lanes' items (three ints plus kMaxDepth faces) to a
// queue of `size` items; returns the new size.
WCB_D int queue_push_faces(int* q, int* qfaces, int size, bool pass, int a, int b, int c,
                           const int (&faces)[kMaxDepth]) {
    const unsigned mask = __ballot_sync(kFull, pass);
    if (pass) {
        const int pos = size + __popc(mask & lanemask_lt());
        q[3 * pos] = a;
        q[3 * pos + 1] = b;
        q[3 * pos + 2] = c;
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k) qfaces[kMaxDepth * pos + k] = faces[k];
    }
    __syncwarp();
    return size + __popc(mask);
}

// Drop the first n items (n <= 32) of a queue with faces.
WCB_D int queue_pop_faces(int* q, int* qfaces, int size, int n, int lane) {
    const int rem = size - n;
    int a0 = 0, a1 = 0, a2 = 0, fb[kMaxDepth];
    if (lane < rem) {
        a0 = q[3 * (n + lane)];
        a1 = q[3 * (n + lane) + 1];
        a2 = q[3 * (n + lane) + 2];
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k) fb[k] = qfaces[kMaxDepth * (n + lane) + k];
    }
    __syncwarp();
    if (lane < rem) {
        q[3 * lane] = a0;
        q[3 * lane + 1] = a1;
        q[3 * lane + 2] = a2;
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k) qfaces[kMaxDepth * lane + k] = fb[k];
    }
    __syncwarp();
    return rem;
}

// Reflection in three queued stages per warp: A (FP64 back projection and
// containment of prefiltered candidates), B (one visibility segment per item
// and pass: an item whose segment is clear goes back to B for its next
// segment, or to F after its last), F (Jones chain and accumulation of the
// visible paths).  Testing one segment per pass keeps the warp's lanes on
// the same kind of work: most candidates are blocked on their first segment
// and leave after one traversal instead of idling while a visible path of
// the same batch traces its remaining segments and its field.
template <typename T, int NF>
__global__ void __launch_bounds__(kSplitBlock, sizeof(T) == 4 ? 3 : 2) k_reflect(MainParams p, int stack_depth) {
    extern __shared__ int smem[];
    int* stack = smem;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    ReflShared<NF>* sh = reinterpret_cast<ReflShared<NF>*>(smem + stack_depth * kSplitBlock) + warp;
    float* red = reinterpret_cast<float*>(reinterpret_cast<ReflShared<NF>*>(smem + stack_depth * kSplitBlock) + kSplitWarps);
    const long long tile = blockIdx.x;
    int t = 0, r = 0;
    const bool active = tile_cell(p, tile, lane, &t, &r);
    // the whole warp shares the tile's transmitter
    const long long per_tx = tiles_per_tx(p);
    const int tw = int(tile / per_tx);
    if (tw >= p.num_tx) return;
    t = tw;
    const SceneDev& sc = p.sc;
    int* err = p.status;
    const V3<double> S = v3<double>(p.tx_pos[3 * t], p.tx_pos[3 * t + 1], p.tx_pos[3 * t + 2]);
    const V3<T> ST = cast3<T>(S);
    const V3<T> tx_pol = v3<T>(T(p.tx_pol[3 * t]), T(p.tx_pol[3 * t + 1]), T(p.tx_pol[3 * t + 2]));
    const V3<float> Rf = active ? rx_point(p, r) : v3(0.f, 0.f, 0.f);
    const float* rp = p.rx_pol + (long long)(active ? r : 0) * p.rx_pol_stride;
    const V3<float> rpol = v3(rp[0], rp[1], rp[2]);
    const T sqrt_p = s_sqrt(s_max(T(p.tx_power[t]), T(0)));
    Cx<T> acc[NF];
    T gain[NF];
    for (int f = 0; f < NF; ++f) { acc[f] = cx(T(0), T(0)); gain[f] = T(0); }
    unsigned long long rays = 0;
    int qa = 0, qb = 0, qf = 0;

    // stage F: field of up to 32 visible paths (FP64 hits recomputed)
    auto process_f = [&](int n) __attribute__((always_inline)) {
        int it_lane = 0, c = 0, d = 1;
        if (lane < n) {
            it_lane = sh->qf[3 * lane];
            c = sh->qf[3 * lane + 1];
            d = sh->qf[3 * lane + 2];
        }
        const float rx = __shfl_sync(kFull, Rf.x, it_lane);
        const float ry = __shfl_sync(kFull, Rf.y, it_lane);
        const float rz = __shfl_sync(kFull, Rf.z, it_lane);
        const float px = __shfl_sync(kFull, rpol.x, it_lane);
        const float py = __shfl_sync(kFull, rpol.y, it_lane);
        const float pz = __shfl_sync(kFull, rpol.z, it_lane);
        const bool ok = lane < n;
        if (ok) {
            const V3<double> R = v3<double>(rx, ry, rz);
            const long long base = p.chain_offset[t * kMaxDepth + (d - 1)];
            const double* planes = p.chain_planes + (base + (long long)c * d) * 4;
            const double* images = p.chain_images + (base + (long long)c * d) * 3;
            V3<double> hits[kMaxDepth];
            back_project(R, planes, images, d, hits);
            int faces[kMaxDepth];
            for (int k = 0; k < d; ++k) faces[k] = sh->qff[kMaxDepth * lane + k];
            const V3<double> img = v3(images[3 * (d - 1)], images[3 * (d - 1) + 1], images[3 * (d - 1) + 2]);
            const double total = length(R - img);
            const V3<T> RT = cast3<T>(R);
            const V3<T> rx_pol = v3<T>(T(px), T(py), T(pz));
            // a records-only solve (no cell output requested: the
            // differentiable forward, which re-evaluates the records in FP64)
            // keeps the path and skips its field
            const int nf_fields = (p.out_comp_power || p.out_comp_field) ? NF : 0;
            for (int f = nf_fields; f < NF; ++f)
                for (int k = 0; k < 3; ++k) sh->contrib[(lane * NF + f) * 3 + k] = 0.f;
#pragma unroll 1
            for (int f = 0; f < nf_fields; ++f) {
                const double freq = p.freq[f];
                const T wl = T(kC0 / freq);
                V3<T> prev = ST;
                V3<T> incident = safe_normalize(cast3<T>(hits[0]) - prev, v3<T>(T(0), T(0), T(1)));
                C3<T> value = c3_from_real(transverse(incident, tx_pol));
                V3<T> outgoing = incident;
                for (int k = 0; k < d; ++k) {
                    const V3<T> hit = cast3<T>(hits[k]);
                    incident = safe_normalize(hit - prev, outgoing);
                    const float* nf = sc.face_normal + 3 * faces[k];
                    reflect_bounce(value, outgoing, incident, v3<T>(T(nf[0]), T(nf[1]), T(nf[2])),
                                   face_slab<T>(p, f, faces[k]), freq, wl);
                    prev = hit;
                }
                const V3<T> fdir = safe_normalize(RT - prev, outgoing);
                const T amp = T(1) / (T(2) * T(p.k[f]) * T(fmax(total, kUtdEps)));
                value = c3_scale(value, phasor_neg_kd<T>(p.k[f], total) * amp);
                const Cx<T> pf = project_receiver(value, fdir, rx_pol) * sqrt_p;
                sh->contrib[(lane * NF + f) * 3 + 0] = float(value_of(pf.re));
                sh->contrib[(lane * NF + f) * 3 + 1] = float(value_of(pf.im));
                sh->contrib[(lane * NF + f) * 3 + 2] = float(value_of(cabs2(pf)));
            }
            int tt = 0, rr = 0;
            tile_cell(p, tile, it_lane, &tt, &rr);
            emit_row(p, t, rr, 1, d, faces, -1, float(total));
        }
        sh->owner[lane] = ok ? it_lane : -1;
        __syncwarp();
        for (int i = 0; i < n; ++i) {
            if (sh->owner[i] == lane) {
                for (int f = 0; f < NF; ++f) {
                    acc[f] = acc[f] + cx(T(sh->contrib[(i * NF + f) * 3]), T(sh->contrib[(i * NF + f) * 3 + 1]));
                    gain[f] = gain[f] + T(sh->contrib[(i * NF + f) * 3 + 2]);
                }
            }
        }
        __syncwarp();
        qf = queue_pop_faces(sh->qf, sh->qff, qf, n, lane);
    };

    // stage B: segment s of up to 32 items (the third int packs d | s << 4)
    auto process_b = [&](int n) __attribute__((always_inline)) {
        int it_lane = 0, c = 0, d = 1, s = 0, faces[kMaxDepth];
        if (lane < n) {
            it_lane = sh->qb[3 * lane];
            c = sh->qb[3 * lane + 1];
            const int ds = sh->qb[3 * lane + 2];
            d = ds & 15;
            s = ds >> 4;
        }
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k) faces[k] = lane < n ? sh->qbf[kMaxDepth * lane + k] : 0;
        const float rx = __shfl_sync(kFull, Rf.x, it_lane);
        const float ry = __shfl_sync(kFull, Rf.y, it_lane);
        const float rz = __shfl_sync(kFull, Rf.z, it_lane);
        bool ok = lane < n;
        if (ok) {
            const V3<double> R = v3<double>(rx, ry, rz);
            const long long base = p.chain_offset[t * kMaxDepth + (d - 1)];
            const int* groups = p.chain_groups + base + (long long)c * d;
            const double* planes = p.chain_planes + (base + (long long)c * d) * 4;
            const double* images = p.chain_images + (base + (long long)c * d) * 3;
            V3<double> a, b;
            back_project_segment(S, R, planes, images, d, s, &a, &b);
            Ignore ig = ignore_none();
            ig.g0 = s > 0 ? groups[s - 1] : -1;
            ig.g1 = s < d ? groups[s] : -1;
            ++rays;
            ok = !segment_blocked<T>(sc, cast3<T>(a), cast3<T>(b), ig, stack, err);
        }
        qb = queue_pop_faces(sh->qb, sh->qbf, qb, n, lane);
        qb = queue_push_faces(sh->qb, sh->qbf, qb, ok && s < d, it_lane, c, d | ((s + 1) << 4), faces);
        qf = queue_push_faces(sh->qf, sh->qff, qf, ok && s == d, it_lane, c, d, faces);
    };

    // stage A: FP64 back projection + containment for up to 32 items; the
    // survivors enter queue B at segment 0
    auto process_a = [&](int n) __attribute__((always_inline)) {
        int it_lane = 0, c = 0, d = 1;
        if (lane < n) {
            it_lane = sh->qa[3 * lane];
            c = sh->qa[3 * lane + 1];
            d = sh->qa[3 * lane + 2];
        }
        const float rx = __shfl_sync(kFull, Rf.x, it_lane);
        const float ry = __shfl_sync(kFull, Rf.y, it_lane);
        const float rz = __shfl_sync(kFull, Rf.z, it_lane);
        bool ok = lane < n;
        int faces[kMaxDepth];
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k) faces[k] = 0;
        if (ok) {
            const long long base = p.chain_offset[t * kMaxDepth + (d - 1)];
            const int* groups = p.chain_groups + base + (long long)c * d;
            const double* planes = p.chain_planes + (base + (long long)c * d) * 4;
            const double* images = p.chain_images + (base + (long long)c * d) * 3;
            // hit k and its face, from the last bounce back (no hit array)
            V3<double> x = v3<double>(rx, ry, rz);
            for (int k = d - 1; k >= 0 && ok; --k) {
                ok = back_project_step(x, planes, images, k);
                const int f = ok ? resolve_in_group(sc, groups[k], x) : -1;
                ok = f >= 0;
#pragma unroll
                for (int kk = 0; kk < kMaxDepth; ++kk)
                    if (kk == k) faces[kk] = f;
            }
        }
        qa = queue_pop(sh->qa, qa, n, lane);
        qb = queue_push_faces(sh->qb, sh->qbf, qb, ok, it_lane, c, d, faces);
    };

    if ((p.components & 2) && sc.num_faces > 0) {
        // One loop drives the stages so each is inlined once.  Each pass runs
        // one step, full batches first and the latest stage first: F, then B,
        // then A, then the next candidate into queue A; partial batches only
        // once nothing upstream can fill them.  A stage runs only while the
        // queues it feeds hold fewer than 32 items, so no queue exceeds 63.
        // This warp takes every kSplitWarps-th candidate of the transmitter,
        // counted across depths.
        int d = 1, c = 0, cnt = 0, global_c = 0;
        long long base = 0;
        auto enter_depth = [&]() __attribute__((always_inline)) {
            while (d <= p.max_depth) {
                cnt = p.chain_count[t * kMaxDepth + (d - 1)];
                base = p.chain_offset[t * kMaxDepth + (d - 1)];
                c = (warp - global_c % kSplitWarps + kSplitWarps) % kSplitWarps;
                global_c += cnt;
                if (c < cnt) return;
                ++d;
            }
        };
        enter_depth();
        while (true) {
            const bool cand_left = d <= p.max_depth;
            int step;
            if (qf >= 32) step = 3;
            else if (qb >= 32) step = 2;
            else if (qa >= 32) step = 1;
            else if (cand_left) step = 0;
            else if (qa > 0) step = 1;
            else if (qb > 0) step = 2;
            else if (qf > 0) step = 3;
            else break;
            if (step == 0) {
                bool pass = active;
                if (sizeof(T) == 4 && pass) pass = back_project_prefilter(sc, Rf, p.chain_pre + (base + c) * 2);
                qa = queue_push(sh->qa, qa, pass, lane, c, d);
                c += kSplitWarps;
                if (c >= cnt) {
                    ++d;
                    enter_depth();
                }
            } else if (step == 1) {
                process_a(qa < 32 ? qa : 32);
            } else if (step == 2) {
                process_b(qb < 32 ? qb : 32);
            } else {
                process_f(qf < 32 ? qf : 32);
            }
        }
        // fixed-order reduction of the warps' partial sums, one write per cell
        for (int f = 0; f < NF; ++f) {
            float* o = red + ((warp * 32 + lane) * NF + f) * 3;
            o[0] = float(value_of(acc[f].re));
            o[1] = float(value_of(acc[f].im));
            o[2] = float(value_of(gain[f]));
        }
        __syncthreads();
        if (warp == 0 && active) {
            const long long cell = (long long)t * p.num_rx + r;
            for (int f = 0; f < NF; ++f) {
                Cx<T> sum = cx(T(0), T(0));
                T g = T(0);
                for (int w = 0; w < kSplitWarps; ++w) {
                    const float* o = red + ((w * 32 + lane) * NF + f) * 3;
                    sum = sum + cx(T(o[0]), T(o[1]));
                    g = g + T(o[2]);
                }
                store_slot(p, 1, f, cell, sum, g, p.coherent);
            }
        }
    }
    if (p.ray_counter && p.freq_base == 0 && rays) atomicAdd(p.ray_counter, rays);
}

// ------------------------------------------------------------------ diffraction
template <int NF>
struct DiffShared {
    int qv[3 * kQueueCap];
    float contrib[32 * NF * 9];
    int owner[32];
};

// Diffraction runs as two kernels per chunk of the transmitter's edge list:
// k_diffract_vis traces the two biased segments of every (cell, edge) pair and
// stores one 32-bit visibility word per (tile, edge); k_diffract_utd
// evaluates the UTD field of the visible pairs.  Apart, the traversal kernel
// runs at twice the occupancy of the field kernel and neither competes with
// the other for instruction cache.

// Visibility words of edges [j0, j0 + chunk) of each tile's transmitter: bit
// `lane` of word (tile, j - j0) is set when both Tx -> Q and Q -> Rx are clear
// for that lane's cell, Q the clamped stationary point on the edge moved by
// kDiffractionRayBias along its exterior bisector.
template <typename T>
__global__ void __launch_bounds__(kSplitBlock, 4) k_diffract_vis(MainParams p, int stack_depth, int j0, int chunk,
                                                                 unsigned* vis_words) {
    extern __shared__ int smem[];
    int* stack = smem;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = blockIdx.x;
    int t = 0, r = 0;
    const bool active = tile_cell(p, tile, lane, &t, &r);
    const long long per_tx = tiles_per_tx(p);
    const int tw = int(tile / per_tx);
    if (tw >= p.num_tx) return;
    t = tw;
    const SceneDev& sc = p.sc;
    int* err = p.status;
    const int cnt = ((p.components & 4) && p.max_depth >= 1) ? p.edge_count[t] : 0;
    const int jend = cnt < j0 + chunk ? cnt : j0 + chunk;
    if (j0 >= jend) return;
    const int* list = p.edge_list + (long long)t * sc.num_edges;
    const V3<double> S = v3<double>(p.tx_pos[3 * t], p.tx_pos[3 * t + 1], p.tx_pos[3 * t + 2]);
    const V3<T> ST = cast3<T>(S);
    const V3<float> Rf = active ? rx_point(p, r) : v3(0.f, 0.f, 0.f);
    const V3<double> R = cast3<double>(Rf);
    unsigned long long rays = 0;
    for (int j = j0 + warp; j < jend; j += kSplitWarps) {
        bool vis = false;
        if (active) {
            const EdgeDev& ed = sc.edges[list[j]];
            const V3<double> c = v3(ed.pos[0], ed.pos[1], ed.pos[2]);
            const V3<double> e = v3(ed.dir[0], ed.dir[1], ed.dir[2]);
            const V3<double> ds = S - c;
            const double ts = dot(ds, e);
            const double rs = length(ds - e * ts);
            const V3<double> dr = R - c;
            const double tr = dot(dr, e);
            const double rr = length(dr - e * tr);
            const double t_star = (rs + rr) > 0.0 ? ts + (tr - ts) * rs / (rs + rr) : ts;
            const double tc = fmin(fmax(t_star, -ed.half_length), ed.half_length);
            const V3<double> qv_pt = c + e * tc + v3(ed.bisector[0], ed.bisector[1], ed.bisector[2]) * kDiffractionRayBias;
            Ignore ig = ignore_none();
            ig.f0 = ed.face0;
            ig.f1 = ed.face1;
            ++rays;
            vis = !segment_blocked<T>(sc, ST, cast3<T>(qv_pt), ig, stack, err);
            if (vis) {
                ++rays;
                vis = !segment_blocked<T>(sc, cast3<T>(qv_pt), cast3<T>(R), ig, stack, err);
            }
        }
        const unsigned word = __ballot_sync(kFull, vis);
        if (lane == 0) vis_words[tile * chunk + (j - j0)] = word;
    }
    if (p.ray_counter && p.freq_base == 0 && rays) atomicAdd(p.ray_counter, rays);
}

// UTD fields of the visible pairs of edges [j0, j0 + chunk).  The tile's
// items are the set bits of its visibility words in (edge, lane) order; warp
// w takes the contiguous w-th eighth of them, queues them and evaluates full
// batches of 32, so the warps of a block finish together.  Per-cell sums are
// reduced over the warps in a fixed order.
// With more than one chunk the running sums (9 values per cell and
// frequency) pass between chunks through `carry`; the chunk that reaches the
// end of the transmitter's edge list writes the outputs.  Chunk 0 always
// runs, so a transmitter without visible edges still gets its zeros.
template <typename T, int NF>
__global__ void __launch_bounds__(kSplitBlock, 2) k_diffract_utd(MainParams p, int j0, int chunk,
                                                                 const unsigned* vis_words, T* carry) {
    extern __shared__ int smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    DiffShared<NF>* sh = reinterpret_cast<DiffShared<NF>*>(smem) + warp;
    float* red = reinterpret_cast<float*>(reinterpret_cast<DiffShared<NF>*>(smem) + kSplitWarps);
    const long long tile = blockIdx.x;
    int t = 0, r = 0;
    const bool active = tile_cell(p, tile, lane, &t, &r);
    const long long per_tx = tiles_per_tx(p);
    const int tw = int(tile / per_tx);
    if (tw >= p.num_tx) return;
    t = tw;
    const SceneDev& sc = p.sc;
    const int cnt = ((p.components & 4) && p.max_depth >= 1) ? p.edge_count[t] : 0;
    if (j0 > 0 && j0 >= cnt) return;
    const int jend = cnt < j0 + chunk ? cnt : j0 + chunk;
    const bool first = j0 == 0;
    const bool last = j0 + chunk >= cnt;
    const V3<double> S = v3<double>(p.tx_pos[3 * t], p.tx_pos[3 * t + 1], p.tx_pos[3 * t + 2]);
    const V3<T> tx_pol = v3<T>(T(p.tx_pol[3 * t]), T(p.tx_pol[3 * t + 1]), T(p.tx_pol[3 * t + 2]));
    const V3<float> Rf = active ? rx_point(p, r) : v3(0.f, 0.f, 0.f);
    const float* rp = p.rx_pol + (long long)(active ? r : 0) * p.rx_pol_stride;
    const V3<float> rpol = v3(rp[0], rp[1], rp[2]);
    const T sqrt_p = s_sqrt(s_max(T(p.tx_power[t]), T(0)));
    Cx<T> acc[NF];
    T gain[NF];
    Cx<T> dv[NF][3];
    for (int f = 0; f < NF; ++f) {
        acc[f] = cx(T(0), T(0));
        gain[f] = T(0);
        for (int k = 0; k < 3; ++k) dv[f][k] = cx(T(0), T(0));
    }
    int qv = 0;
    const int* list = p.edge_list + (long long)t * sc.num_edges;

    // UTD fields for up to 32 visible items
    auto process_v = [&](int n) __attribute__((always_inline)) {
        int it_lane = 0, j = 0;
        if (lane < n) {
            it_lane = sh->qv[3 * lane];
            j = sh->qv[3 * lane + 1];
        }
        const float rx = __shfl_sync(kFull, Rf.x, it_lane);
        const float ry = __shfl_sync(kFull, Rf.y, it_lane);
        const float rz = __shfl_sync(kFull, Rf.z, it_lane);
        const float px = __shfl_sync(kFull, rpol.x, it_lane);
        const float py = __shfl_sync(kFull, rpol.y, it_lane);
        const float pz = __shfl_sync(kFull, rpol.z, it_lane);
        bool any = false;
        if (lane < n) {
            const EdgeDev& ed = sc.edges[list[j]];
            const V3<double> R = v3<double>(rx, ry, rz);
            const V3<T> rx_pol = v3<T>(T(px), T(py), T(pz));
            double qx = 0, qy = 0, qz = 0, len = 0;
            // the frequency-independent geometry once, the field per frequency
            const EdgeFrame<double> fr = edge_frame(ed);
            const UtdGeometry<double, T> geo = utd_geometry<double, T>(fr, S, R, tx_pol);
#pragma unroll 1
            for (int f = 0; f < NF; ++f) {
                const DiffractionResult<T> res =
                    utd_result(geo, fr, face_slab<T>(p, f, ed.mat_face0), face_slab<T>(p, f, ed.mat_face1), p.freq[f]);
                qx = res.q[0]; qy = res.q[1]; qz = res.q[2];
                len = res.length;
                const C3<T> powered = c3_scale(res.field, cx(sqrt_p, T(0)));
                float* cb = sh->contrib + (lane * NF + f) * 9;
                if (res.valid && value_of(c3_power(powered)) >= kUtdGainFloor) {
                    any = true;
                    const V3<T> arrival = safe_normalize(cast3<T>(R - v3(qx, qy, qz)), v3<T>(T(0), T(0), T(1)));
                    const Cx<T> pf = project_receiver(powered, arrival, rx_pol);
                    cb[0] = float(value_of(pf.re));
                    cb[1] = float(value_of(pf.im));
                    cb[2] = float(value_of(cabs2(pf)));
                    cb[3] = float(value_of(powered.x.re)); cb[4] = float(value_of(powered.x.im));
                    cb[5] = float(value_of(powered.y.re)); cb[6] = float(value_of(powered.y.im));
                    cb[7] = float(value_of(powered.z.re)); cb[8] = float(value_of(powered.z.im));
                } else {
                    for (int k = 0; k < 9; ++k) cb[k] = 0.f;
                }
            }
            if (any) {
                int tt = 0, rr = 0;
                tile_cell(p, tile, it_lane, &tt, &rr);
                emit_row(p, t, rr, 2, 1, nullptr, ed.edge_id, float(len));
            }
        }
        sh->owner[lane] = any ? it_lane : -1;
        __syncwarp();
        for (int i = 0; i < n; ++i) {
            if (sh->owner[i] == lane) {
                for (int f = 0; f < NF; ++f) {
                    const float* cb = sh->contrib + (i * NF + f) * 9;
                    acc[f] = acc[f] + cx(T(cb[0]), T(cb[1]));
                    gain[f] = gain[f] + T(cb[2]);
                    dv[f][0] = dv[f][0] + cx(T(cb[3]), T(cb[4]));
                    dv[f][1] = dv[f][1] + cx(T(cb[5]), T(cb[6]));
                    dv[f][2] = dv[f][2] + cx(T(cb[7]), T(cb[8]));
                }
            }
        }
        __syncwarp();
    };

    // this warp's share [lo, hi) of the tile's items
    const unsigned* words = vis_words + tile * chunk;
    const int nw = jend > j0 ? jend - j0 : 0;
    int total = 0;
    for (int b = 0; b < nw; b += 32) {
        const int jj = b + lane;
        total += int(__reduce_add_sync(kFull, jj < nw ? unsigned(__popc(words[jj])) : 0u));
    }
    const int lo = int((long long)total * warp / kSplitWarps);
    const int hi = int((long long)total * (warp + 1) / kSplitWarps);
    // skip, 32 words at a time, the words whose items all precede lo
    int jj = 0, seen = 0;
    for (; jj < nw; jj += 32) {
        const unsigned c = jj + lane < nw ? unsigned(__popc(words[jj + lane])) : 0u;
        const int group = int(__reduce_add_sync(kFull, c));
        if (seen + group > lo) break;
        seen += group;
    }
    if (jj < nw) {
        // within this group of 32 words: the first word holding item lo
        const int word_i = jj + lane;
        const int c = word_i < nw ? __popc(words[word_i]) : 0;
        int incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        const unsigned past = __ballot_sync(kFull, seen + incl > lo);
        const int first = __ffs(past) - 1;  // past != 0: the group holds item lo
        const int before = __shfl_sync(kFull, incl - c, first);
        jj += first;
        seen += before;
    }
    // one loop walks the words and drives the queue so the UTD stage is
    // inlined once
    while (true) {
        if (jj < nw && seen < hi) {
            const unsigned word = words[jj];
            const int idx = seen + __popc(word & lanemask_lt());
            const bool mine = ((word >> lane) & 1u) && idx >= lo && idx < hi;
            qv = queue_push(sh->qv, qv, mine, lane, j0 + jj, 0);
            seen += __popc(word);
            ++jj;
        }
        const bool drained = !(jj < nw && seen < hi);
        if (qv >= 32 || (drained && qv > 0)) {
            const int n = qv < 32 ? qv : 32;
            process_v(n);
            qv = queue_pop(sh->qv, qv, n, lane);
        }
        if (drained && qv == 0) break;
    }
    // fixed-order reduction of the warps' partial sums, one write per cell
    for (int f = 0; f < NF; ++f) {
        float* o = red + ((warp * 32 + lane) * NF + f) * 9;
        o[0] = float(value_of(acc[f].re));
        o[1] = float(value_of(acc[f].im));
        o[2] = float(value_of(gain[f]));
        for (int k = 0; k < 3; ++k) {
            o[3 + 2 * k] = float(value_of(dv[f][k].re));
            o[4 + 2 * k] = float(value_of(dv[f][k].im));
        }
    }
    __syncthreads();
    if (warp == 0 && active && (p.components & 4)) {
        const long long cell = (long long)t * p.num_rx + r;
        const long long cells = (long long)p.num_tx * p.num_rx;
        for (int f = 0; f < NF; ++f) {
            Cx<T> sum = cx(T(0), T(0));
            T g = T(0);
            Cx<T> v[3] = {cx(T(0), T(0)), cx(T(0), T(0)), cx(T(0), T(0))};
            T* cr = carry ? carry + ((long long)f * cells + cell) * 9 : nullptr;
            if (!first && cr) {
                sum = cx(cr[0], cr[1]);
                g = cr[2];
                for (int k = 0; k < 3; ++k) v[k] = cx(cr[3 + 2 * k], cr[4 + 2 * k]);
            }
            for (int w = 0; w < kSplitWarps; ++w) {
                const float* o = red + ((w * 32 + lane) * NF + f) * 9;
                sum = sum + cx(T(o[0]), T(o[1]));
                g = g + T(o[2]);
                for (int k = 0; k < 3; ++k) v[k] = v[k] + cx(T(o[3 + 2 * k]), T(o[4 + 2 * k]));
            }
            if (last) {
                store_slot(p, 2, f, cell, sum, g, p.coherent);
                T* dvp = static_cast<T*>(p.out_diff_vec_power);
                if (dvp) dvp[(long long)(p.freq_base + f) * cells + cell] = cabs2(v[0]) + cabs2(v[1]) + cabs2(v[2]);
            } else if (cr) {
                cr[0] = sum.re;
                cr[1] = sum.im;
                cr[2] = g;
                for (int k = 0; k < 3; ++k) {
                    cr[3 + 2 * k] = v[k].re;
                    cr[4 + 2 * k] = v[k].im;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ totals
template <typename T>
__global__ void k_finalize(MainParams p, int nf) {
    const long long cells = (long long)p.num_tx * p.num_rx;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= cells * nf) return;
    const int f = int(i / cells);
    const long long cell = i - (long long)f * cells;
    const long long fc = (long long)(p.freq_base + f) * cells + cell;
    const long long stride = (long long)p.num_freq_total * cells;
    T* cp = static_cast<T*>(p.out_comp_power);
    T* cf = static_cast<T*>(p.out_comp_field);
    if (cp == nullptr || cf == nullptr) return;
    const int used[4] = {p.components & 1, p.components & 2, p.components & 4, p.components & 8};
    Cx<T> total = cx(T(0), T(0));
    T gsum = T(0);
    for (int s = 0; s < 6; ++s) {
        const long long o = s * stride + fc;
        if (s < 4 && used[s]) {
            total = total + cx(cf[2 * o], cf[2 * o + 1]);
            gsum = gsum + cp[o];
        } else {
            cp[o] = T(0);
            cf[2 * o] = T(0);
            cf[2 * o + 1] = T(0);
        }
    }
    T* pg = static_cast<T*>(p.out_path_gain);
    T* fl = static_cast<T*>(p.out_field);
    if (p.coherent) {
        if (pg) pg[fc] = cabs2(total);
        if (fl) { fl[2 * fc] = total.re; fl[2 * fc + 1] = total.im; }
    } else {
        if (pg) pg[fc] = gsum;
        if (fl) { fl[2 * fc] = s_sqrt(s_max(gsum, T(0))); fl[2 * fc + 1] = T(0); }
    }
    T* dvp = static_cast<T*>(p.out_diff_vec_power);
    if (dvp && !(p.components & 4)) dvp[fc] = T(0);
}

}  // namespace wcb
