// Fixed-topology replay: frozen LoS and reflection records re-evaluated at new
// endpoint positions without discovery (reference propagation/consumer.py:
// 3846-4110 reevaluate, 2375-2449 prepared_row_gather, 2734-2811 the LoS and
// reflection bucket inputs, 3029-3096 evaluate_prepared).
//
// The reference replays one (component, depth) bucket per launch and one
// launch per frequency column, after a host-side gather of the endpoint rows.
// Here one thread replays one record for every column: the endpoint gather,
// the contract validation, the visibility re-test and the image-method
// geometry are frequency-independent and done once, the per-column work is
// only the Fresnel/Jones chain.  The execution order (a permutation grouping
// records by component and depth, formed once per frozen topology) keeps a
// warp on one branch of the kernel.

#include <cuda_runtime.h>

#include <algorithm>

#include "em.cuh"
#include "internal.h"
#include "paths.cuh"
#include "row_eval.cuh"
#include "solve.h"

namespace wcb {

namespace {

constexpr int kReplayBlock = 128;

// contract bits (reference consumer.py:2261-2268) and engine bits
constexpr int kIndexBounds = 1;
constexpr int kPairOrder = 2;
constexpr int kStableId = 16;
constexpr int kSlotBlock = 32;
constexpr int kBadRecord = 2;
constexpr int kBadFace = 4;

struct ReplayParams {
    SceneDev sc;
    wcb_frozen_rows rows;
    wcb_endpoint_batch src, snk;
    long long slot_count;
    int num_columns;
    const double* freqs;
    int num_materials;
    const float* eps_r;
    const float* sigma_e;
    const float* mu_r;
    const float* gain;
    const float* thickness;
    int visibility;
    wcb_replay_outputs out;
    int* status;
};

struct PairOf {
    long long pair;
    bool in_bounds;
    bool slot_broken;
};

// Pair of frozen row i under the declared layout (reference consumer.py:
// 2339-2360 for slots, 2411 for the outer product).
WCB_D PairOf pair_of(const ReplayParams& p, long long i) {
    const long long s = p.rows.source_index[i];
    const long long r = p.rows.sink_index[i];
    PairOf o;
    o.in_bounds = s >= 0 && s < p.src.count && r >= 0 && r < p.snk.count;
    o.slot_broken = false;
    if (p.slot_count == 1) {
        o.pair = r * p.src.count + s;
        return o;
    }
    const long long ss = max(p.src.count / p.slot_count, 1LL);
    const long long ks = max(p.snk.count / p.slot_count, 1LL);
    const long long slot = s >= 0 ? s / ss : -((-s + ss - 1) / ss);  // floor division
    const long long s_in = s - slot * ss;
    const long long k_in = r - slot * ks;
    o.pair = slot * ss * ks + k_in * ss + s_in;
    o.slot_broken = k_in < 0 || k_in >= ks;
    return o;
}

WCB_D void put_c(float* dst, long long i, Cx<float> v) {
    dst[2 * i] = v.re;
    dst[2 * i + 1] = v.im;
}

WCB_D void put_c3(float* dst, long long i, const C3<float>& v) {
    put_c(dst, 3 * i + 0, v.x);
    put_c(dst, 3 * i + 1, v.y);
    put_c(dst, 3 * i + 2, v.z);
}

WCB_D void put_v(float* dst, long long i, V3<float> v) {
    dst[3 * i] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}

WCB_D void put_frame(float* dst, long long i, V3<float> u, V3<float> v) {
    put_v(dst, 2 * i, u);
    put_v(dst, 2 * i + 1, v);
}

// Every published value of row i at zero, row_valid 0.  The first nh
// interaction slots keep the positions and normals given (either may be
// NULL: zeros), the rest are zero.
WCB_D void write_inert(const ReplayParams& p, long long i, int nh, const V3<double>* hits, const V3<float>* normals) {
    const wcb_replay_outputs& o = p.out;
    const Cx<float> z = cx(0.f, 0.f);
    const C3<float> z3 = {z, z, z};
    const int extra = p.num_columns - 1;
    if (o.coefficient) put_c(o.coefficient, i, z);
    if (o.field) put_c3(o.field, i, z3);
    for (int c = 0; c < extra; ++c) {
        if (o.coefficient_offsets) put_c(o.coefficient_offsets, i * extra + c, z);
        if (o.field_offsets) put_c3(o.field_offsets, i * extra + c, z3);
    }
    if (o.path_length_m) o.path_length_m[i] = 0.f;
    if (o.delay_s) o.delay_s[i] = 0.f;
    if (o.direction) put_v(o.direction, i, v3(0.f, 0.f, 0.f));
    if (o.row_valid) o.row_valid[i] = 0;
    if (o.jones) for (int q = 0; q < 4; ++q) put_c(o.jones, 4 * i + q, z);
    if (o.source_basis) put_frame(o.source_basis, i, v3(0.f, 0.f, 0.f), v3(0.f, 0.f, 0.f));
    if (o.sink_basis) put_frame(o.sink_basis, i, v3(0.f, 0.f, 0.f), v3(0.f, 0.f, 0.f));
    const int W = p.rows.width;
    for (int k = 0; k < W; ++k) {
        const bool on = k < nh;
        if (o.interaction_positions) {
            const V3<float> h = on && hits ? cast3<float>(hits[k]) : v3(0.f, 0.f, 0.f);
            put_v(o.interaction_positions, i * W + k, h);
        }
        if (o.interaction_normals)
            put_v(o.interaction_normals, i * W + k, on && normals ? normals[k] : v3(0.f, 0.f, 0.f));
    }
}

__global__ void __launch_bounds__(kReplayBlock) k_replay_rows(ReplayParams p) {
    extern __shared__ int stack[];
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long K = p.rows.num_rows;
    if (tid >= K) return;
    long long i = tid;
    if (p.rows.order) {
        i = p.rows.order[tid];
        if (i < 0 || i >= K) {
            atomicOr(p.status + 1, kBadRecord);
            return;
        }
    }
    const wcb_frozen_rows& fr = p.rows;
    const wcb_replay_outputs& o = p.out;

    // contract validation of row i in frozen order
    const PairOf po = pair_of(p, i);
    int bits = po.in_bounds ? 0 : kIndexBounds;
    if (po.in_bounds && po.slot_broken) bits |= kSlotBlock;
    const long long s = fr.source_index[i];
    const long long r = fr.sink_index[i];
    if (po.in_bounds && ((fr.source_id && fr.source_id[i] != p.src.stable_ids[s]) ||
                         (fr.sink_id && fr.sink_id[i] != p.snk.stable_ids[r])))
        bits |= kStableId;
    if (i > 0 && po.in_bounds) {
        const PairOf prev = pair_of(p, i - 1);
        if (prev.in_bounds && po.pair < prev.pair) bits |= kPairOrder;
    }
    if (o.pair_index) o.pair_index[i] = po.pair;
    if (bits) {
        atomicOr(p.status, bits);
        write_inert(p, i, 0, nullptr, nullptr);
        return;
    }

    const int comp = fr.component_id[i];
    const int d = fr.depth[i];
    const int W = fr.width;
    const bool shape_ok = (comp == 0 && d == 0) || (comp == 1 && d >= 1 && d <= W && d <= kMaxDepth);
    if (!shape_ok) {
        atomicOr(p.status + 1, kBadRecord);
        write_inert(p, i, 0, nullptr, nullptr);
        return;
    }
    int faces[kMaxDepth];
    bool faces_ok = true;
    for (int k = 0; k < kMaxDepth; ++k) {
        faces[k] = k < d ? fr.primitive_sequence[i * W + k] : 0;
        if (k < d && (faces[k] < 0 || faces[k] >= p.sc.num_faces)) faces_ok = false;
    }
    if (!faces_ok) {
        atomicOr(p.status + 1, kBadFace);
        write_inert(p, i, 0, nullptr, nullptr);
        return;
    }

    const SceneDev& sc = p.sc;
    const V3<double> S = v3<double>(p.src.positions[3 * s], p.src.positions[3 * s + 1], p.src.positions[3 * s + 2]);
    const V3<double> R = v3<double>(p.snk.positions[3 * r], p.snk.positions[3 * r + 1], p.snk.positions[3 * r + 2]);
    const V3<float> Sf = cast3<float>(S), Rf = cast3<float>(R);
    const V3<float> tx_pol = v3<float>(p.src.polarizations[3 * s], p.src.polarizations[3 * s + 1],
                                       p.src.polarizations[3 * s + 2]);
    const V3<float> rx_pol = v3<float>(p.snk.polarizations[3 * r], p.snk.polarizations[3 * r + 1],
                                       p.snk.polarizations[3 * r + 2]);
    const float P = p.src.powers ? fmaxf(p.src.powers[s], 0.0f) : 1.0f;
    const float sq = sqrtf(P);

    // frequency-independent geometry and the visibility re-test
    ReflectionGeom g;
    V3<float> normals[kMaxDepth];
    int groups[kMaxDepth];
    bool valid = true;
    double length_m;
    if (comp == 0) {
        length_m = length(R - S);
        if (p.visibility && sc.num_faces > 0) valid = !segment_blocked<float>(sc, Sf, Rf, ignore_none(), stack, p.status + 1);
    } else {
        g = reflection_geometry(sc, faces, d, S, R);
        length_m = g.length;
        for (int k = 0; k < d; ++k) {
            groups[k] = sc.face_group[faces[k]];
            const float* nf = sc.face_normal + 3 * faces[k];
            normals[k] = v3(nf[0], nf[1], nf[2]);
        }
        if (p.visibility) {
            valid = g.solved;
            for (int k = 0; k < d && valid; ++k) valid = resolve_in_group(sc, groups[k], g.hits[k]) >= 0;
            for (int seg = 0; seg <= d && valid; ++seg) {
                const V3<double> a = seg > 0 ? g.hits[seg - 1] : S;
                const V3<double> b = seg < d ? g.hits[seg] : R;
                Ignore ig = ignore_none();
                ig.g0 = seg > 0 ? groups[seg - 1] : -1;
                ig.g1 = seg < d ? groups[seg] : -1;
                valid = !segment_blocked<float>(sc, cast3<float>(a), cast3<float>(b), ig, stack, p.status + 1);
            }
        }
    }
    if (!valid) {
        // a reflection record keeps its re-solved hits (when the back
        // projection crossed every plane) and its faces' normals
        if (comp == 1) write_inert(p, i, d, g.solved ? g.hits : nullptr, normals);
        else write_inert(p, i, 0, nullptr, nullptr);
        return;
    }

    // every frequency column
    const int extra = p.num_columns - 1;
    const int M = p.num_materials;
    V3<float> dir0 = v3(0.f, 0.f, 0.f);
#pragma unroll 1
    for (int c = 0; c < p.num_columns; ++c) {
        const double freq = p.freqs[c];
        const double k = kTwoPi * freq / kC0;
        C3<float> unit;
        Cx<float> coef;
        V3<float> dir;
        if (comp == 0) {
            const PathEval<float> ev = eval_free_space(Sf, Rf, tx_pol, rx_pol, k, length_m);
            unit = ev.field;
            coef = ev.coefficient;
            dir = ev.direction;
        } else {
            const long long mo = (long long)c * M;
            auto slab = [&](int f) {
                const int m = sc.face_material[f];
                return Slab<float>{p.eps_r[mo + m], p.sigma_e[mo + m], p.mu_r[mo + m], p.gain[mo + m],
                                   p.thickness[mo + m]};
            };
            V3<float> nb[kMaxDepth];
            reflection_field(sc, faces, d, g, Sf, Rf, tx_pol, rx_pol, slab, freq, k, nb, &unit, &coef, &dir);
        }
        const Cx<float> path_field = coef * sq;
        const C3<float> field = {unit.x * sq, unit.y * sq, unit.z * sq};
        if (c == 0) {
            dir0 = dir;
            if (o.coefficient) put_c(o.coefficient, i, path_field);
            if (o.field) put_c3(o.field, i, field);
        } else {
            if (o.coefficient_offsets) put_c(o.coefficient_offsets, i * extra + (c - 1), path_field);
            if (o.field_offsets) put_c3(o.field_offsets, i * extra + (c - 1), field);
        }
    }
    if (o.path_length_m) o.path_length_m[i] = float(length_m);
    if (o.delay_s) o.delay_s[i] = float(length_m / kC0);
    if (o.direction) put_v(o.direction, i, dir0);
    if (o.row_valid) o.row_valid[i] = 1;
    for (int k = 0; k < W; ++k) {
        const bool on = comp == 1 && k < d;
        if (o.interaction_positions)
            put_v(o.interaction_positions, i * W + k, on ? cast3<float>(g.hits[k]) : v3(0.f, 0.f, 0.f));
        if (o.interaction_normals) put_v(o.interaction_normals, i * W + k, on ? normals[k] : v3(0.f, 0.f, 0.f));
    }

    // polarimetric response at column 0: both source frame vectors through the
    // record, each projected on both sink frame vectors (reference
    // consumer.py:2898-2925 and compose_jones :2533-2579)
    if (o.jones) {
        const double freq = p.freqs[0];
        const double k = kTwoPi * freq / kC0;
        V3<float> launch, arrival;
        if (comp == 0) {
            launch = safe_normalize(Rf - Sf, v3<float>(0.f, 0.f, 1.f));
            arrival = launch;
        } else {
            launch = safe_normalize(cast3<float>(g.hits[0]) - Sf, v3<float>(0.f, 0.f, 1.f));
            arrival = safe_normalize(Rf - cast3<float>(g.hits[d - 1]), v3<float>(0.f, 0.f, 1.f));
        }
        V3<float> su, sv, ru, rv;
        endpoint_frame(p.src.polarization_basis, s, launch, &su, &sv);
        endpoint_frame(p.snk.polarization_basis, r, arrival, &ru, &rv);
        C3<float> fu, fv;
        Cx<float> cu, cv;
        V3<float> du, dv;
        if (comp == 0) {
            const PathEval<float> eu = eval_free_space(Sf, Rf, su, ru, k, length_m);
            const PathEval<float> ev = eval_free_space(Sf, Rf, sv, ru, k, length_m);
            fu = eu.field;
            fv = ev.field;
            cu = eu.coefficient;
            cv = ev.coefficient;
            du = eu.direction;
            dv = ev.direction;
        } else {
            auto slab = [&](int f) {
                const int m = sc.face_material[f];
                return Slab<float>{p.eps_r[m], p.sigma_e[m], p.mu_r[m], p.gain[m], p.thickness[m]};
            };
            V3<float> nb[kMaxDepth];
            reflection_field(sc, faces, d, g, Sf, Rf, su, ru, slab, freq, k, nb, &fu, &cu, &du);
            reflection_field(sc, faces, d, g, Sf, Rf, sv, ru, slab, freq, k, nb, &fv, &cv, &dv);
        }
        put_c(o.jones, 4 * i + 0, cu);
        put_c(o.jones, 4 * i + 1, cv);
        put_c(o.jones, 4 * i + 2, project_receiver(fu, du, rv));
        put_c(o.jones, 4 * i + 3, project_receiver(fv, dv, rv));
        if (o.source_basis) put_frame(o.source_basis, i, su, sv);
        if (o.sink_basis) put_frame(o.sink_basis, i, ru, rv);
    }
}

// pair_offsets[q] = number of rows with pair_index < q (rows in pair order)
__global__ void k_pair_offsets(const long long* pair, long long n, long long num_pairs, long long* offsets) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q > num_pairs) return;
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (pair[mid] < q) lo = mid + 1;
        else hi = mid;
    }
    offsets[q] = lo;
}

}  // namespace

int rows_replay(const SceneHandle* h, const wcb_frozen_rows* rows, const wcb_endpoint_batch* src,
                const wcb_endpoint_batch* snk, int64_t slot_count, const wcb_materials* m, const double* freqs,
                int num_columns, int visibility, const wcb_replay_outputs* out, int* status, cudaStream_t stream) {
    ReplayParams p;
    p.sc = h->dev;
    p.rows = *rows;
    p.src = *src;
    p.snk = *snk;
    p.slot_count = slot_count;
    p.num_columns = num_columns;
    p.freqs = freqs;
    p.num_materials = m->num_materials;
    p.eps_r = m->eps_r;
    p.sigma_e = m->sigma_e;
    p.mu_r = m->mu_r;
    p.gain = m->gain;
    p.thickness = m->thickness;
    p.visibility = visibility;
    p.out = *out;
    p.status = status;
    const long long K = rows->num_rows;
    if (K > 0) {
        const size_t smem = size_t(std::max(h->dev.stack_entries, 1)) * kReplayBlock * sizeof(int);
        k_replay_rows<<<int((K + kReplayBlock - 1) / kReplayBlock), kReplayBlock, smem, stream>>>(p);
        note_launch();
        if (cudaGetLastError() != cudaSuccess) return 2;
    }
    if (out->pair_offsets && (K == 0 || out->pair_index)) {
        const long long ss = src->count / slot_count, ks = snk->count / slot_count;
        const long long P = slot_count * ss * ks;
        constexpr int kB = 256;
        k_pair_offsets<<<int((P + 1 + kB - 1) / kB), kB, 0, stream>>>(reinterpret_cast<const long long*>(out->pair_index),
                                                                     K, P, reinterpret_cast<long long*>(out->pair_offsets));
        note_launch();
        if (cudaGetLastError() != cudaSuccess) return 2;
    }
    return 0;
}

}  // namespace wcb
