// In-place update of a compiled scene after its vertices moved (a gradient
// loop's optimiser step), without a host round trip.
//
// The compile's discrete decisions -- coplanar face groups (quantised plane
// keys), diffraction edge selection and wedge face order, shared-boundary
// merges, the edge policy -- and the BVH topology are kept; everything
// continuous is recomputed on the device from the new vertices: face planes
// and normals, group planes and boxes, the selected edges' frames, the leaf
// triangles and the BVH boxes (bottom-up).  First, every discrete decision is
// recomputed from the new vertices with the same arithmetic as the host
// compile and compared with the decisions cached at compile time (groupings
// as partitions: a rigid move of a building changes its plane keys but not
// which faces share one); if any differs, nothing the solve reads is written
// and the caller recompiles the scene.  The result therefore equals a fresh
// compile of the moved mesh (node boxes are exact min/max values, and the
// floating-point steps mirror the host build operation for operation with
// every product and sum rounded on its own; acos and atan2 may differ from
// the host's in the last bit); only the BVH's split positions and the
// numbering of coplanar groups stay those of the original build, which
// changes no traced result.  Two small values come back to the host (the decision flag and the
// scene diagonal), one synchronisation; the mesh itself never does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/witwin_channel_b200.h"
#include "internal.h"

namespace wcb {
namespace refit {

constexpr int kB = 256;

// -------- IEEE operations without contraction (the host compile's rounding)
WCB_D double dm(double a, double b) { return __dmul_rn(a, b); }
WCB_D double da(double a, double b) { return __dadd_rn(a, b); }
WCB_D double ds(double a, double b) { return __dsub_rn(a, b); }
WCB_D double dd(double a, double b) { return __ddiv_rn(a, b); }
WCB_D float fm(float a, float b) { return __fmul_rn(a, b); }
WCB_D float fa(float a, float b) { return __fadd_rn(a, b); }
WCB_D float fs(float a, float b) { return __fsub_rn(a, b); }

struct D3 {
    double x, y, z;
};
WCB_D D3 sub3f(const float* a, const float* b) {
    return {ds(double(a[0]), double(b[0])), ds(double(a[1]), double(b[1])), ds(double(a[2]), double(b[2]))};
}
WCB_D D3 cross(D3 a, D3 b) {
    return {ds(dm(a.y, b.z), dm(a.z, b.y)), ds(dm(a.z, b.x), dm(a.x, b.z)), ds(dm(a.x, b.y), dm(a.y, b.x))};
}
WCB_D double dot(D3 a, D3 b) { return da(da(dm(a.x, b.x), dm(a.y, b.y)), dm(a.z, b.z)); }
WCB_D D3 norm(D3 a, double eps = 1e-6) {
    double l = __dsqrt_rn(dot(a, a));
    l = fmax(l, eps);
    return {dd(a.x, l), dd(a.y, l), dd(a.z, l)};
}
WCB_D D3 neg(D3 a) { return {-a.x, -a.y, -a.z}; }
WCB_D double unsigned_angle(D3 a, D3 b, D3 axis) {
    const D3 c = cross(a, b);
    const double s = dot(c, axis);
    const double sn = (s > 0 ? 1.0 : (s < 0 ? -1.0 : 0.0)) * __dsqrt_rn(dot(c, c));
    const double ang = atan2(sn, dot(a, b));
    return ang < 0 ? da(ang, 2.0 * M_PI) : ang;
}

// face plane: unit normal of (b - a) x (c - a) and offset n.a
WCB_D D3 face_normal64(const float* v, const int* faces, int f, double* offset) {
    const float* a = v + 3 * faces[3 * f];
    const float* b = v + 3 * faces[3 * f + 1];
    const float* c = v + 3 * faces[3 * f + 2];
    const D3 n = norm(cross(sub3f(b, a), sub3f(c, a)));
    if (offset) *offset = da(da(dm(n.x, double(a[0])), dm(n.y, double(a[1]))), dm(n.z, double(a[2])));
    return n;
}

// the coplanar group key of a face (fp32, as the compile forms it)
WCB_D void face_key(const float* v, const int* faces, int f, int surface, long long key[5]) {
    const float* a = v + 3 * faces[3 * f];
    const float* b = v + 3 * faces[3 * f + 1];
    const float* c = v + 3 * faces[3 * f + 2];
    const float e1[3] = {fs(b[0], a[0]), fs(b[1], a[1]), fs(b[2], a[2])};
    const float e2[3] = {fs(c[0], a[0]), fs(c[1], a[1]), fs(c[2], a[2])};
    const float cxv[3] = {fs(fm(e1[1], e2[2]), fm(e1[2], e2[1])), fs(fm(e1[2], e2[0]), fm(e1[0], e2[2])),
                          fs(fm(e1[0], e2[1]), fm(e1[1], e2[0]))};
    float l = __fsqrt_rn(fa(fa(fm(cxv[0], cxv[0]), fm(cxv[1], cxv[1])), fm(cxv[2], cxv[2])));
    l = fmaxf(l, 1e-6f);
    float nx = __fdiv_rn(cxv[0], l), ny = __fdiv_rn(cxv[1], l), nz = __fdiv_rn(cxv[2], l);
    const float nrm = __fsqrt_rn(fa(fa(fm(nx, nx), fm(ny, ny)), fm(nz, nz)));
    const float inv = nrm > 1e-6f ? __fdiv_rn(1.0f, nrm) : 0.0f;
    nx = fm(nx, inv);
    ny = fm(ny, inv);
    nz = fm(nz, inv);
    float major_abs = fabsf(nx), major = nx;
    if (fabsf(ny) > major_abs) { major_abs = fabsf(ny); major = ny; }
    if (fabsf(nz) > major_abs) { major = nz; }
    const float sgn = major < 0.0f ? -1.0f : 1.0f;
    nx = fm(nx, sgn);
    ny = fm(ny, sgn);
    nz = fm(nz, sgn);
    const float offset = fa(fa(fm(nx, a[0]), fm(ny, a[1])), fm(nz, a[2]));
    const float scale = float(1.0 / kPlaneGroupQuant);
    key[0] = surface;
    key[1] = llroundf(fm(nx, scale));
    key[2] = llroundf(fm(ny, scale));
    key[3] = llroundf(fm(nz, scale));
    key[4] = llroundf(fm(offset, scale));
}

WCB_D int opposite(const int* faces, int f, int a, int b) {
    for (int k = 0; k < 3; ++k) {
        const int v = faces[3 * f + k];
        if (v != a && v != b) return v;
    }
    return faces[3 * f + 2];
}

// One edge record's geometry and decisions, as the compile computes them.
struct EdgeCalc {
    D3 pos, dir, n0, n1, opp0;
    double len, ext;
    bool first, coplanar, sel0;
    int fn0, fn1, mat0, mat1;
};

WCB_D EdgeCalc edge_calc(const float* v, const int* faces, int v0, int v1, int f0, int f1) {
    EdgeCalc e;
    const bool bnd = f0 >= 0 && f1 < 0;
    const bool interior = f0 >= 0 && f1 >= 0;
    const int s0 = f0 >= 0 ? f0 : 0, s1 = f1 >= 0 ? f1 : 0;
    const float* st = v + 3 * v0;
    const float* en = v + 3 * v1;
    const D3 vec = sub3f(en, st);
    const double L = fmax(__dsqrt_rn(dot(vec, vec)), 1e-12);
    const D3 d = {dd(vec.x, L), dd(vec.y, L), dd(vec.z, L)};
    const D3 n0c = norm(face_normal64(v, faces, s0, nullptr));
    const D3 n1c = norm(face_normal64(v, faces, s1, nullptr));
    const D3 to1 = norm(cross(n0c, d));
    const D3 tn1 = norm(cross(n1c, d));
    const bool first = unsigned_angle(to1, tn1, d) < unsigned_angle(tn1, to1, d);
    const D3 on0 = first ? n0c : n1c;
    const D3 on1 = first ? n1c : n0c;
    const D3 out0 = interior ? on0 : n0c;
    D3 out1 = interior ? on1 : n1c;
    if (f1 < 0) out1 = neg(n0c);
    const double inter = acos(fmin(fmax(-dot(out0, out1), -1.0), 1.0));
    e.ext = interior ? ds(2.0 * M_PI, inter) : 2.0 * M_PI;
    bool coplanar = false;
    if (interior) {
        const bool aligned = fabs(dot(n0c, n1c)) >= kNormalCosTol;
        const D3 pa = sub3f(v + 3 * opposite(faces, s0, v0, v1), st);
        const D3 pb = sub3f(v + 3 * opposite(faces, s1, v0, v1), st);
        coplanar = aligned && fabs(dot(pa, n0c)) <= kEdgePlaneTol && fabs(dot(pb, n0c)) <= kEdgePlaneTol;
    }
    const bool wedge_ok = bnd || (interior && dot(n0c, n1c) < 1.0);
    e.sel0 = (interior || bnd) && !coplanar && L > 1e-6 && wedge_ok;
    e.first = first;
    e.coplanar = coplanar;
    e.pos = {dm(0.5, da(double(st[0]), double(en[0]))), dm(0.5, da(double(st[1]), double(en[1]))),
             dm(0.5, da(double(st[2]), double(en[2])))};
    e.dir = d;
    e.len = L;
    e.n0 = out0;
    e.n1 = out1;
    const bool swapped = interior && !first;
    const int of = swapped ? s1 : s0;
    const float* op = v + 3 * opposite(faces, of, v0, v1);
    e.opp0 = {double(op[0]), double(op[1]), double(op[2])};
    e.mat0 = swapped ? f1 : f0;
    e.mat1 = swapped ? f0 : f1;
    e.fn0 = interior ? (first ? s0 : s1) : s0;
    e.fn1 = interior ? (first ? s1 : s0) : -1;
    return e;
}

// merged exterior angle of a shared boundary pair (a, b) and whether the head stays selected
WCB_D double merged_exterior(D3 na, D3 nb, bool* keep) {
    const double nd = fmin(fmax(dot(na, nb), -1.0), 1.0);
    const double interior_angle = acos(fmin(fmax(-nd, -1.0), 1.0));
    const double merged = ds(2.0 * M_PI, interior_angle);
    const bool copl = fabs(nd) >= kNormalCosTol;
    *keep = (merged > M_PI * (1.0 + 1e-6)) && !copl;
    return merged;
}

WCB_D bool vertical_ok(const float* v, int v0, int v1, double ratio) {
    const D3 dv = sub3f(v + 3 * v1, v + 3 * v0);
    const double lz = fmax(__dsqrt_rn(dot(dv, dv)), 1e-6);
    return dd(fabs(dv.z), lz) > ratio;
}

// -------- decision check (writes only refit scratch and the flag)
//
// A grouping decision (coplanar face groups, shared-boundary endpoint
// classes) is kept when the moved vertices induce the same partition: every
// member still has its class head's key, and distinct classes still have
// distinct keys.  The keys' values may change (a translated or rotated
// building), so classes may sort in another order than a fresh compile
// would give them; no result depends on that order (paths are keyed by face
// and edge ids, and the representative of a class is its lowest member).

__global__ void k_face_keys(const float* v, const int* faces, const int* surface, int F, long long* keys) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    face_key(v, faces, f, surface[f], keys + 5 * size_t(f));
}

__global__ void k_check_faces(int F, const int* face_group, const int* group_rep, const long long* keys,
                              int* changed) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int r = group_rep[face_group[f]];
    for (int i = 0; i < 5; ++i)
        if (keys[5 * size_t(f) + i] != keys[5 * size_t(r) + i]) {
            atomicOr(changed, 1);
            return;
        }
}

WCB_D unsigned long long mix64(unsigned long long x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// Distinct classes keep distinct keys: each class head inserts its key into
// an open-addressing table (linear probing over at least twice as many slots
// as classes, so every insert ends within `mask + 1` probes); meeting an
// equal key of another head means two classes would merge.  Class i's head
// item is heads[i] (heads == nullptr: item i, counted only when
// head_of[i] == i).
__global__ void k_unique_keys(int n, const int* heads, const int* head_of, const long long* keys, int width,
                              int* table, int mask, int* changed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int item = i;
    if (heads != nullptr) item = heads[i];
    else if (head_of[i] != i) return;
    const long long* k = keys + size_t(width) * item;
    unsigned long long h = 0x9e3779b97f4a7c15ull;
    for (int w = 0; w < width; ++w) h = mix64(h ^ (unsigned long long)k[w]);
    int slot = int(h & (unsigned long long)mask);
    for (int probe = 0; probe <= mask; ++probe) {
        const int prev = atomicCAS(table + slot, -1, item);
        if (prev == -1) return;
        const long long* o = keys + size_t(width) * prev;
        bool same = true;
        for (int w = 0; w < width; ++w) same = same && o[w] == k[w];
        if (same) {
            atomicOr(changed, 1);
            return;
        }
        slot = (slot + 1) & mask;
    }
    atomicOr(changed, 1);  // unreachable with the table's size; a full table counts as a change
}

// every shared-boundary candidate keeps its class head's quantised endpoints
__global__ void k_check_edge_classes(int NE, const int* qhead, const long long* qkey, int* changed) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NE) return;
    const int hd = qhead[e];
    if (hd < 0 || hd == e) return;
    for (int k = 0; k < 6; ++k)
        if (qkey[6 * size_t(e) + k] != qkey[6 * size_t(hd) + k]) {
            atomicOr(changed, 1);
            return;
        }
}

__global__ void k_check_edges(const float* v, const int* faces, const int4* rec, const unsigned char* state,
                              const int* qhead, long long* qkey, const int* partner, int NE, int half_plane,
                              int vertical_only, double ratio, int* changed) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NE) return;
    const int4 r = rec[e];
    const EdgeCalc c = edge_calc(v, faces, r.x, r.y, r.z, r.w);
    const unsigned char s = state[e];
    bool ok = c.first == bool(s & 1) && c.coplanar == bool(s & 2) && c.sel0 == bool(s & 4);
    const bool boundary = r.z >= 0 && r.w < 0;
    if (qhead[e] >= 0) {
        // the quantised endpoints that pair shared boundary records (their
        // classes are checked by k_check_edge_classes and k_unique_keys)
        const float* a = v + 3 * r.x;
        const float* b = v + 3 * r.y;
        long long pa[3], pb[3];
        for (int k = 0; k < 3; ++k) {
            pa[k] = llround(dd(double(a[k]), kEndpointQuant));
            pb[k] = llround(dd(double(b[k]), kEndpointQuant));
        }
        const bool a_first = pa[0] < pb[0] || (pa[0] == pb[0] && (pa[1] < pb[1] || (pa[1] == pb[1] && pa[2] <= pb[2])));
        const long long* lo = a_first ? pa : pb;
        const long long* hi = a_first ? pb : pa;
        for (int k = 0; k < 3; ++k) {
            qkey[6 * size_t(e) + k] = lo[k];
            qkey[6 * size_t(e) + 3 + k] = hi[k];
        }
    }
    if (ok) {
        // the final selection after merges and the policy
        bool sel = c.sel0;
        bool bnd_final = boundary;
        const int p = partner[e];
        if (p >= 0) {
            const int4 rb = rec[p];
            const EdgeCalc cb = edge_calc(v, faces, rb.x, rb.y, rb.z, rb.w);
            bool keep;
            merged_exterior(c.n0, cb.n0, &keep);
            sel = keep;
            bnd_final = false;
        } else if (p <= -2) {
            sel = false;  // second or later record of a shared boundary group
        }
        if (!half_plane && bnd_final) sel = false;
        if (vertical_only && !vertical_ok(v, r.x, r.y, ratio)) sel = false;
        ok = sel == bool(s & 8);
    }
    if (!ok) atomicOr(changed, 1);
}

// -------- the update
__global__ void k_faces(const float* v, const int* faces, int F, double* plane, float* normal) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    double off;
    const D3 n = face_normal64(v, faces, f, &off);
    plane[4 * f] = n.x;
    plane[4 * f + 1] = n.y;
    plane[4 * f + 2] = n.z;
    plane[4 * f + 3] = off;
    normal[3 * f] = float(n.x);
    normal[3 * f + 1] = float(n.y);
    normal[3 * f + 2] = float(n.z);
}

__global__ void k_groups(const float* v, const int* faces, int G, const int* rep, const int* off, const int* members,
                         const double* face_plane, double* plane, float* box) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = off[g]; i < off[g + 1]; ++i) {
        const int f = members[i];
        for (int k = 0; k < 3; ++k) {
            const float* p = v + 3 * faces[3 * f + k];
            for (int ax = 0; ax < 3; ++ax) {
                lo[ax] = fminf(lo[ax], p[ax]);
                hi[ax] = fmaxf(hi[ax], p[ax]);
            }
        }
    }
    for (int ax = 0; ax < 3; ++ax) {
        const float pad = fa(float(kPlaneTolerance), fm(1e-6f, fmaxf(fabsf(lo[ax]), fabsf(hi[ax]))));
        box[6 * g + ax] = fs(lo[ax], pad);
        box[6 * g + 3 + ax] = fa(hi[ax], pad);
    }
    const int r = rep[g];
    for (int k = 0; k < 4; ++k) plane[4 * g + k] = face_plane[4 * r + k];
}

__global__ void k_edges(const float* v, const int* faces, const int4* rec, const int* partner, const int* edge_ids,
                        int E, EdgeDev* edges) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E) return;
    const int e = edge_ids[i];
    const int4 r = rec[e];
    const EdgeCalc c = edge_calc(v, faces, r.x, r.y, r.z, r.w);
    D3 n1 = c.n1;
    double ext = c.ext;
    const int p = partner[e];
    if (p >= 0) {
        const int4 rb = rec[p];
        const EdgeCalc cb = edge_calc(v, faces, rb.x, rb.y, rb.z, rb.w);
        bool keep;
        ext = merged_exterior(c.n0, cb.n0, &keep);
        n1 = cb.n0;
    }
    EdgeDev ed = edges[i];
    const D3 t0 = norm(cross(c.n0, c.dir));
    const D3 to_opp = {ds(c.opp0.x, c.pos.x), ds(c.opp0.y, c.pos.y), ds(c.opp0.z, c.pos.z)};
    const bool into_face0 = dot(to_opp, t0) >= 0.0;
    D3 bis = {da(c.n0.x, n1.x), da(c.n0.y, n1.y), da(c.n0.z, n1.z)};
    const double bl = __dsqrt_rn(dot(bis, bis));
    if (bl > 1e-6) bis = {dd(bis.x, bl), dd(bis.y, bl), dd(bis.z, bl)};
    else if (into_face0) bis = neg(t0);
    else bis = t0;
    const double pv[3] = {c.pos.x, c.pos.y, c.pos.z}, dv[3] = {c.dir.x, c.dir.y, c.dir.z};
    const double tv[3] = {t0.x, t0.y, t0.z}, n0v[3] = {c.n0.x, c.n0.y, c.n0.z}, n1v[3] = {n1.x, n1.y, n1.z};
    const double bv[3] = {bis.x, bis.y, bis.z};
    for (int k = 0; k < 3; ++k) {
        ed.pos[k] = pv[k];
        ed.dir[k] = dv[k];
        ed.t0[k] = tv[k];
        ed.n0[k] = n0v[k];
        ed.n1[k] = n1v[k];
        ed.bisector[k] = bv[k];
    }
    ed.half_length = dm(0.5, c.len);
    ed.n = dd(ext, M_PI);
    edges[i] = ed;
}

__global__ void k_leaf_tris(const float* v, const int* faces, int F, float4* tri) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= F) return;
    const float4 a0 = tri[3 * sl];
    const int f = __float_as_int(a0.w);
    const float* a = v + 3 * faces[3 * f];
    const float* b = v + 3 * faces[3 * f + 1];
    const float* c = v + 3 * faces[3 * f + 2];
    tri[3 * sl] = make_float4(a[0], a[1], a[2], a0.w);
    const float4 b0 = tri[3 * sl + 1];
    tri[3 * sl + 1] = make_float4(b[0], b[1], b[2], b0.w);
    tri[3 * sl + 2] = make_float4(c[0], c[1], c[2], 0.0f);
}

WCB_D void set_child_box(BvhNode* n, int side, const float lo[3], const float hi[3]) {
    float* w = reinterpret_cast<float*>(n);
    const int o = side == 0 ? 0 : 6;
    w[o + 0] = lo[0];
    w[o + 1] = lo[1];
    w[o + 2] = lo[2];
    w[o + 3] = hi[0];
    w[o + 4] = hi[1];
    w[o + 5] = hi[2];
}

// Bottom-up BVH boxes: one thread per leaf walks to the root; at each node
// the second child to arrive (an atomic counter) forms the node's box from
// both child boxes and carries it to the parent.
__global__ void k_bvh(const float* v, const int* faces, const float4* tri, int F, const int* leaf_parent,
                      const int* node_parent, BvhNode* nodes, int* counter) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= F) return;
    const int f = __float_as_int(tri[3 * sl].w);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 3; ++k) {
        const float* p = v + 3 * faces[3 * f + k];
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = fminf(lo[ax], p[ax]);
            hi[ax] = fmaxf(hi[ax], p[ax]);
        }
    }
    int ref = leaf_parent[sl];
    while (ref >= 0) {
        const int node = ref >> 1;
        set_child_box(nodes + node, ref & 1, lo, hi);
        __threadfence();
        if (atomicAdd(counter + node, 1) == 0) return;  // the sibling subtree finishes this node
        __threadfence();
        const volatile float* w = reinterpret_cast<const volatile float*>(nodes + node);
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = fminf(w[ax], w[6 + ax]);
            hi[ax] = fmaxf(w[3 + ax], w[9 + ax]);
        }
        ref = node_parent[node];
    }
}

__global__ void k_diagonal(const float* v, int V, double* diagonal) {
    __shared__ float slo[3][256], shi[3][256];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = threadIdx.x; i < V; i += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], v[3 * i + k]);
            hi[k] = fmaxf(hi[k], v[3 * i + k]);
        }
    for (int k = 0; k < 3; ++k) {
        slo[k][threadIdx.x] = lo[k];
        shi[k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 3; ++k) {
                slo[k][threadIdx.x] = fminf(slo[k][threadIdx.x], slo[k][threadIdx.x + s]);
                shi[k][threadIdx.x] = fmaxf(shi[k][threadIdx.x], shi[k][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double w = ds(double(shi[k][0]), double(slo[k][0]));
            s = da(s, dm(w, w));
        }
        *diagonal = V ? __dsqrt_rn(s) : 0.0;
    }
}

}  // namespace refit

// Boxes of the compiled scene's BVH from its current leaf triangles and parent
// links (bvh_counter zeroed by the caller), bottom-up.
int refit_boxes(SceneHandle* h, cudaStream_t stream) {
    using namespace refit;
    const SceneDev& sd = h->dev;
    const int F = sd.num_faces;
    if (F < 2) return 0;
    k_bvh<<<(F + kB - 1) / kB, kB, 0, stream>>>(sd.vertices, sd.faces, sd.tri, F, h->leaf_parent, h->node_parent,
                                                const_cast<BvhNode*>(sd.nodes), h->bvh_counter);
    note_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int scene_refit(SceneHandle* h, const float* d_vertices, int64_t nv, int* topology_changed, cudaStream_t stream) {
    using namespace refit;
    if (h == nullptr || topology_changed == nullptr || (nv > 0 && d_vertices == nullptr)) return 1;
    SceneDev& sd = h->dev;
    if (nv != sd.num_vertices) return 1;
    *topology_changed = 0;
    const int F = sd.num_faces, G = sd.num_groups, E = sd.num_edges, NE = h->num_edges_total, V = sd.num_vertices;
    if (V == 0) return 0;
    int* flag = h->refit_flag;
    bool ok = cudaMemsetAsync(flag, 0, sizeof(int), stream) == cudaSuccess;
    const int mask = h->key_table_slots - 1;
    int launches = 1;
    if (F > 0) {
        k_face_keys<<<(F + kB - 1) / kB, kB, 0, stream>>>(d_vertices, sd.faces, h->face_surface, F, h->face_keys);
        k_check_faces<<<(F + kB - 1) / kB, kB, 0, stream>>>(F, sd.face_group, sd.group_rep, h->face_keys, flag);
        ok = ok && cudaMemsetAsync(h->key_table, 0xff, size_t(h->key_table_slots) * sizeof(int), stream) == cudaSuccess;
        k_unique_keys<<<(G + kB - 1) / kB, kB, 0, stream>>>(G, sd.group_rep, nullptr, h->face_keys, 5, h->key_table,
                                                             mask, flag);
        launches += 3;
    }
    if (NE > 0) {
        k_check_edges<<<(NE + kB - 1) / kB, kB, 0, stream>>>(d_vertices, sd.faces, h->edge_rec, h->edge_state,
                                                             h->edge_qhead, h->edge_qkey, h->edge_partner, NE,
                                                             h->half_plane_policy, h->vertical_only_policy,
                                                             h->vertical_ratio, flag);
        k_check_edge_classes<<<(NE + kB - 1) / kB, kB, 0, stream>>>(NE, h->edge_qhead, h->edge_qkey, flag);
        ok = ok && cudaMemsetAsync(h->key_table, 0xff, size_t(h->key_table_slots) * sizeof(int), stream) == cudaSuccess;
        k_unique_keys<<<(NE + kB - 1) / kB, kB, 0, stream>>>(NE, nullptr, h->edge_qhead, h->edge_qkey, 6, h->key_table,
                                                              mask, flag);
        launches += 3;
    }
    k_diagonal<<<1, 256, 0, stream>>>(d_vertices, V, h->diagonal_dev);
    int changed = 0;
    double diagonal = 0.0;
    ok = ok && cudaGetLastError() == cudaSuccess;
    ok = ok && cudaMemcpyAsync(&changed, flag, sizeof(int), cudaMemcpyDeviceToHost, stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(&diagonal, h->diagonal_dev, sizeof(double), cudaMemcpyDeviceToHost, stream) ==
                   cudaSuccess;
    ok = ok && cudaStreamSynchronize(stream) == cudaSuccess;
    note_launch(launches);
    if (!ok) return 2;
    if (changed) {
        *topology_changed = 1;
        return 0;
    }
    float* verts = const_cast<float*>(sd.vertices);
    ok = cudaMemcpyAsync(verts, d_vertices, size_t(V) * 12, cudaMemcpyDeviceToDevice, stream) == cudaSuccess;
    if (F > 0) {
        k_faces<<<(F + kB - 1) / kB, kB, 0, stream>>>(verts, sd.faces, F, const_cast<double*>(sd.face_plane),
                                                       const_cast<float*>(sd.face_normal));
        k_groups<<<(G + kB - 1) / kB, kB, 0, stream>>>(verts, sd.faces, G, sd.group_rep, sd.group_member_off,
                                                        sd.group_members, sd.face_plane,
                                                        const_cast<double*>(sd.group_plane),
                                                        const_cast<float*>(sd.group_box));
        if (E > 0)
            k_edges<<<(E + kB - 1) / kB, kB, 0, stream>>>(verts, sd.faces, h->edge_rec, h->edge_partner, h->edge_ids,
                                                           E, const_cast<EdgeDev*>(sd.edges));
        k_leaf_tris<<<(F + kB - 1) / kB, kB, 0, stream>>>(verts, sd.faces, F, const_cast<float4*>(sd.tri));
        if (F > 1) {
            ok = ok && cudaMemsetAsync(h->bvh_counter, 0, size_t(F - 1) * sizeof(int), stream) == cudaSuccess;
            k_bvh<<<(F + kB - 1) / kB, kB, 0, stream>>>(verts, sd.faces, sd.tri, F, h->leaf_parent, h->node_parent,
                                                        const_cast<BvhNode*>(sd.nodes), h->bvh_counter);
        }
    }
    sd.diagonal = diagonal;
    ok = ok && cudaGetLastError() == cudaSuccess;
    note_launch(6);
    return ok ? 0 : 2;
}

}  // namespace wcb
