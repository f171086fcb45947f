// BVH traversal: any-hit segment occlusion, closest hit, and ordered
// all-hits along a segment.
//
// Each thread keeps its stack in shared memory, interleaved across the block
// (entry i of thread t lives at stack[i * blockDim.x + t]) so pushes and pops
// of a warp hit distinct banks.  Nodes are read as four 16-byte read-only
// loads and triangles as three 16-byte loads.  The triangle test is the
// watertight algorithm of Woop, Benthin and Wald (JCGT 2013): shared edges
// neither leak nor double-miss, and it falls back to double precision when an
// edge function is exactly zero.
#pragma once

#include "common.cuh"
#include "scene.cuh"

namespace wcb {

// Faces a segment query must not report: up to two coplanar groups (the
// planes a segment starts or ends on) and two faces (a diffraction wedge).
struct Ignore {
    int g0, g1, f0, f1;
};
WCB_HD Ignore ignore_none() { return Ignore{-1, -1, -1, -1}; }

// A ray with its watertight-test constants: the axis permutation (kz = the
// largest |d| component, kx and ky the next two, swapped when d[kz] < 0) and
// the shear Sx = d[kx]/d[kz], Sy = d[ky]/d[kz], Sz = 1/d[kz], computed once per
// ray instead of once per triangle test.
template <typename G>
struct Ray {
    V3<G> o, d, inv;
    G tmin, tmax;
    G Sx, Sy, Sz;
    int kx, ky, kz;
};

template <typename G>
WCB_D G comp3(const V3<G>& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : v.z);
}

template <typename G>
WCB_D Ray<G> make_ray(V3<G> o, V3<G> d, G tmin, G tmax) {
    Ray<G> r;
    r.o = o;
    r.d = d;
    const G big = sizeof(G) == 4 ? G(1e30) : G(1e300);
    r.inv.x = s_abs(d.x) > G(1e-30) ? G(1) / d.x : (d.x >= G(0) ? big : -big);
    r.inv.y = s_abs(d.y) > G(1e-30) ? G(1) / d.y : (d.y >= G(0) ? big : -big);
    r.inv.z = s_abs(d.z) > G(1e-30) ? G(1) / d.z : (d.z >= G(0) ? big : -big);
    r.tmin = tmin;
    r.tmax = tmax;
    const G adx = s_abs(d.x), ady = s_abs(d.y), adz = s_abs(d.z);
    int kz = adx > ady ? (adx > adz ? 0 : 2) : (ady > adz ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (comp3(d, kz) < G(0)) { const int t = kx; kx = ky; ky = t; }
    const G dz = comp3(d, kz);
    r.Sx = comp3(d, kx) / dz;
    r.Sy = comp3(d, ky) / dz;
    r.Sz = G(1) / dz;
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    return r;
}

// Three-operand min/max (PTX ISA, sm_100a): the same value as two nested
// two-operand ones, in one instruction.
WCB_D float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
WCB_D float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
WCB_D double fmax3(double a, double b, double c) { return fmax(fmax(a, b), c); }
WCB_D double fmin3(double a, double b, double c) { return fmin(fmin(a, b), c); }

template <typename G>
WCB_D bool box_hit(const Ray<G>& r, G lx, G ly, G lz, G hx, G hy, G hz, G tmax, G* tnear) {
    G t0x = (lx - r.o.x) * r.inv.x, t1x = (hx - r.o.x) * r.inv.x;
    G t0y = (ly - r.o.y) * r.inv.y, t1y = (hy - r.o.y) * r.inv.y;
    G t0z = (lz - r.o.z) * r.inv.z, t1z = (hz - r.o.z) * r.inv.z;
    G tn = fmax3(s_min(t0x, t1x), s_min(t0y, t1y), s_max(s_min(t0z, t1z), r.tmin));
    G tf = fmin3(s_max(t0x, t1x), s_max(t0y, t1y), s_min(s_max(t0z, t1z), tmax));
    // conservative widening (Ize, "Robust BVH ray traversal", 2013)
    tf = tf * (sizeof(G) == 4 ? G(1.0000004) : G(1.000000000000001));
    *tnear = tn;
    return tn <= tf;
}

// a*b - c*d without contraction into a fused multiply-add
WCB_D float edge_fn(float a, float b, float c, float d) { return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d)); }
WCB_D double edge_fn(double a, double b, double c, double d) { return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d)); }

// Watertight ray/triangle test.  Returns t (ray parameter) or +inf.
template <typename G>
WCB_D G tri_hit(const Ray<G>& r, float4 a4, float4 b4, float4 c4) {
    const V3<G> A0 = v3<G>(G(a4.x), G(a4.y), G(a4.z)) - r.o;
    const V3<G> B0 = v3<G>(G(b4.x), G(b4.y), G(b4.z)) - r.o;
    const V3<G> C0 = v3<G>(G(c4.x), G(c4.y), G(c4.z)) - r.o;
    const int kx = r.kx, ky = r.ky, kz = r.kz;
    const G Sx = r.Sx, Sy = r.Sy, Sz = r.Sz;
    auto comp = [](const V3<G>& v, int i) -> G { return comp3(v, i); };
    const G Ax = comp(A0, kx) - Sx * comp(A0, kz), Ay = comp(A0, ky) - Sy * comp(A0, kz);
    const G Bx = comp(B0, kx) - Sx * comp(B0, kz), By = comp(B0, ky) - Sy * comp(B0, kz);
    const G Cx_ = comp(C0, kx) - Sx * comp(C0, kz), Cy = comp(C0, ky) - Sy * comp(C0, kz);
    // Edge functions with every product rounded on its own: a shared edge's
    // function in the two adjacent triangles is then the exact negation of
    // the other (the watertightness argument), which a fused multiply-add of
    // one product into the subtraction would break (both could round to the
    // same sign and the crossing would leak between the triangles).
    G U = edge_fn(Cx_, By, Cy, Bx);
    G V = edge_fn(Ax, Cy, Ay, Cx_);
    G W = edge_fn(Bx, Ay, By, Ax);
    if (sizeof(G) == 4 && (U == G(0) || V == G(0) || W == G(0))) {
        U = G(edge_fn(double(Cx_), double(By), double(Cy), double(Bx)));
        V = G(edge_fn(double(Ax), double(Cy), double(Ay), double(Cx_)));
        W = G(edge_fn(double(Bx), double(Ay), double(By), double(Ax)));
    }
    const G inf = sizeof(G) == 4 ? G(__int_as_float(0x7f800000)) : G(__longlong_as_double(0x7ff0000000000000LL));
    if ((U < G(0) || V < G(0) || W < G(0)) && (U > G(0) || V > G(0) || W > G(0))) return inf;
    const G det = U + V + W;
    if (det == G(0)) return inf;
    const G Az = Sz * comp(A0, kz), Bz = Sz * comp(B0, kz), Cz = Sz * comp(C0, kz);
    const G Tn = U * Az + V * Bz + W * Cz;
    return Tn / det;
}

WCB_D bool ignored(const Ignore& ig, int face, int group) {
    return group == ig.g0 || group == ig.g1 || face == ig.f0 || face == ig.f1;
}

WCB_D void load_node(const BvhNode* nodes, int idx, float4& a, float4& b, float4& c, int4& d) {
    const float4* p = reinterpret_cast<const float4*>(nodes + idx);
    a = __ldg(p + 0);
    b = __ldg(p + 1);
    c = __ldg(p + 2);
    d = __ldg(reinterpret_cast<const int4*>(p + 3));
}

// Generic traversal.  MODE 0: any hit (returns true on first accepted hit).
// MODE 1: closest hit (updates *best_t / *best_face / *best_group).
// MODE 2: all hits (calls sink(t, face, group), stop when sink returns false).
template <int MODE, typename G, typename Sink>
WCB_D bool traverse(const SceneDev& sc, Ray<G> r, const Ignore& ig, int* stack, int* err, G* best_t, int* best_face,
                    int* best_group, Sink sink) {
    if (sc.num_faces == 0) return false;
    const int stride = blockDim.x;
    const int lane = threadIdx.x;
    int sp = 0;
    int node = sc.root;
    G tmax = r.tmax;
    auto leaf = [&](int ref) -> bool {  // returns true to terminate
        const int slot = ~ref;
        const float4 a = __ldg(sc.tri + 3 * slot + 0);
        const float4 b = __ldg(sc.tri + 3 * slot + 1);
        const float4 c = __ldg(sc.tri + 3 * slot + 2);
        const int face = __float_as_int(a.w);
        const int group = __float_as_int(b.w);
        if (ignored(ig, face, group)) return false;
        const G t = tri_hit(r, a, b, c);
        if (!(t >= r.tmin && t <= tmax)) return false;
        if (MODE == 0) return true;
        if (MODE == 1) {
            tmax = t;
            *best_t = t;
            *best_face = face;
            *best_group = group;
            return false;
        }
        return !sink(t, face, group);
    };
    if (node < 0) {  // single-triangle scene
        return leaf(node);
    }
    while (true) {
        float4 a, b, c;
        int4 d;
        load_node(sc.nodes, node, a, b, c, d);
        G n0, n1;
        bool h0 = box_hit(r, G(a.x), G(a.y), G(a.z), G(a.w), G(b.x), G(b.y), tmax, &n0);
        bool h1 = box_hit(r, G(b.z), G(b.w), G(c.x), G(c.y), G(c.z), G(c.w), tmax, &n1);
        int next = -1;
        bool have_next = false;
        if (h0 && d.x < 0) {
            if (leaf(d.x)) return true;
            h0 = false;
        }
        if (h1 && d.y < 0) {
            if (leaf(d.y)) return true;
            h1 = false;
        }
        if (h0 && h1) {
            const bool first0 = n0 <= n1;
            const int near_c = first0 ? d.x : d.y;
            const int far_c = first0 ? d.y : d.x;
            if (sp < sc.stack_entries) {
                stack[sp * stride + lane] = far_c;
                ++sp;
            } else {
                atomicOr(err, 1);
            }
            next = near_c;
            have_next = true;
        } else if (h0) {
            next = d.x;
            have_next = true;
        } else if (h1) {
            next = d.y;
            have_next = true;
        }
        if (!have_next) {
            if (sp == 0) break;
            --sp;
            next = stack[sp * stride + lane];
        }
        node = next;
    }
    return MODE == 1 ? (*best_face >= 0) : false;
}

struct NoSink {
    WCB_D bool operator()(float, int, int) const { return true; }
    WCB_D bool operator()(double, int, int) const { return true; }
};

// Segment p0 -> p1 blocked by any face outside `ig` at t in [1e-6, 1-1e-6].
template <typename G>
WCB_D bool segment_blocked(const SceneDev& sc, V3<G> p0, V3<G> p1, const Ignore& ig, int* stack, int* err) {
    const Ray<G> r = make_ray<G>(p0, p1 - p0, G(1e-6), G(1) - G(1e-6));
    G bt = G(0);
    int bf = -1, bg = -1;
    return traverse<0, G>(sc, r, ig, stack, err, &bt, &bf, &bg, NoSink{});
}

}  // namespace wcb
