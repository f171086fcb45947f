// Scene compile: face planes, coplanar groups, diffraction edges and the
// BVH (binned SAH, built on the host and uploaded once per scene).
//
// Coplanar groups follow native/channel/kernels/paths.cu:3168-3190 (keys) and
// paths.cu:3768-3912 (ordering); edge selection follows
// native/channel/kernels/diffraction.cu:803-900 and the shared-boundary merge
// and policy filter of witwin/channel/scene/resources.py:306-405.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "internal.h"

namespace wcb {

namespace {


// ------------------------------------------------------------ BVH build
// Binned surface-area-heuristic build on the host (Wald, "On fast
// construction of SAH-based bounding volume hierarchies", 2007): each node's
// triangles are binned by centroid into kSahBins slabs along each axis and
// split where (area_left * count_left + area_right * count_right) is least;
// ranges whose centroids coincide, and every node below kSahMaxDepth, split
// at the median instead.  Leaves hold one triangle; node boxes are the exact
// fp32 min/max of their triangles' vertices.  Nodes are stored depth first
// with siblings adjacent; leaf slots follow the final triangle order.
constexpr int kSahBins = 32;
constexpr int kSahMaxDepth = kStackDepth - 8;

struct BuildBox {
    float lo[3], hi[3];
    void reset() {
        for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    }
    void grow(const BuildBox& o) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], o.lo[k]); hi[k] = std::max(hi[k], o.hi[k]); }
    }
    double area() const {
        const double dx = double(hi[0]) - lo[0], dy = double(hi[1]) - lo[1], dz = double(hi[2]) - lo[2];
        return dx < 0 ? 0.0 : 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct BuildPrim {
    BuildBox box;
    float c[3];
};

// Writes `nodes` (max(F-1, 1) entries, F > 1) and `order` (slot -> face);
// returns the largest number of internal ancestors of a leaf.
static int build_bvh(const std::vector<float>& verts, const std::vector<int>& faces, int F, std::vector<BvhNode>& nodes,
                     std::vector<int>& order) {
    std::vector<BuildPrim> prim(F);
    for (int f = 0; f < F; ++f) {
        BuildBox bx;
        bx.reset();
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < 3; ++k) {
                const float x = verts[3 * faces[3 * f + v] + k];
                bx.lo[k] = std::min(bx.lo[k], x);
                bx.hi[k] = std::max(bx.hi[k], x);
            }
        prim[f].box = bx;
        for (int k = 0; k < 3; ++k) prim[f].c[k] = 0.5f * (bx.lo[k] + bx.hi[k]);
    }
    order.resize(F);
    for (int f = 0; f < F; ++f) order[f] = f;
    nodes.assign(1, BvhNode{});
    struct Task {
        int begin, end, node, depth;
    };
    std::vector<Task> stack{{0, F, 0, 0}};
    int max_depth = 0;
    auto range_box = [&](int b, int e) {
        BuildBox bx;
        bx.reset();
        for (int i = b; i < e; ++i) bx.grow(prim[order[i]].box);
        return bx;
    };
    while (!stack.empty()) {
        const Task t = stack.back();
        stack.pop_back();
        const int n = t.end - t.begin;
        max_depth = std::max(max_depth, t.depth + 1);
        // centroid bounds
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int i = t.begin; i < t.end; ++i)
            for (int k = 0; k < 3; ++k) {
                clo[k] = std::min(clo[k], prim[order[i]].c[k]);
                chi[k] = std::max(chi[k], prim[order[i]].c[k]);
            }
        int mid = -1;
        if (t.depth < kSahMaxDepth) {
            double best = INFINITY;
            int best_axis = -1, best_split = -1;
            for (int k = 0; k < 3; ++k) {
                const float ext = chi[k] - clo[k];
                if (!(ext > 0.0f)) continue;
                BuildBox bins[kSahBins];
                int count[kSahBins] = {};
                for (int q = 0; q < kSahBins; ++q) bins[q].reset();
                const float scale = float(kSahBins) / ext;
                for (int i = t.begin; i < t.end; ++i) {
                    const BuildPrim& pr = prim[order[i]];
                    const int q = std::min(kSahBins - 1, int((pr.c[k] - clo[k]) * scale));
                    bins[q].grow(pr.box);
                    ++count[q];
                }
                double right_area[kSahBins];
                int right_count[kSahBins];
                BuildBox acc;
                acc.reset();
                int cnt = 0;
                for (int q = kSahBins - 1; q > 0; --q) {
                    acc.grow(bins[q]);
                    cnt += count[q];
                    right_area[q] = acc.area();
                    right_count[q] = cnt;
                }
                acc.reset();
                cnt = 0;
                for (int q = 1; q < kSahBins; ++q) {
                    acc.grow(bins[q - 1]);
                    cnt += count[q - 1];
                    if (cnt == 0 || right_count[q] == 0) continue;
                    const double cost = acc.area() * cnt + right_area[q] * right_count[q];
                    if (cost < best) {
                        best = cost;
                        best_axis = k;
                        best_split = q;
                    }
                }
            }
            if (best_axis >= 0) {
                const int k = best_axis;
                const float scale = float(kSahBins) / (chi[k] - clo[k]);
                auto it = std::partition(order.begin() + t.begin, order.begin() + t.end, [&](int f) {
                    return std::min(kSahBins - 1, int((prim[f].c[k] - clo[k]) * scale)) < best_split;
                });
                mid = int(it - order.begin());
            }
        }
        if (mid <= t.begin || mid >= t.end) {
            // median along the widest centroid extent (ties keep the face order)
            int k = 0;
            for (int q = 1; q < 3; ++q)
                if (chi[q] - clo[q] > chi[k] - clo[k]) k = q;
            mid = t.begin + n / 2;
            std::stable_sort(order.begin() + t.begin, order.begin() + t.end,
                             [&](int x, int y) { return prim[x].c[k] < prim[y].c[k]; });
        }
        int child[2];
        const int rb[2] = {t.begin, mid}, re[2] = {mid, t.end};
        BuildBox cb[2];
        for (int s = 0; s < 2; ++s) {
            cb[s] = range_box(rb[s], re[s]);
            if (re[s] - rb[s] == 1) {
                child[s] = ~rb[s];
            } else {
                child[s] = int(nodes.size());
                nodes.push_back(BvhNode{});
            }
        }
        BvhNode& nd = nodes[t.node];
        nd.a = make_float4(cb[0].lo[0], cb[0].lo[1], cb[0].lo[2], cb[0].hi[0]);
        nd.b = make_float4(cb[0].hi[1], cb[0].hi[2], cb[1].lo[0], cb[1].lo[1]);
        nd.c = make_float4(cb[1].lo[2], cb[1].hi[0], cb[1].hi[1], cb[1].hi[2]);
        nd.d = make_int4(child[0], child[1], 0, 0);
        // right first so the left subtree is built (and laid out) next
        for (int s = 1; s >= 0; --s)
            if (child[s] >= 0) stack.push_back({rb[s], re[s], child[s], t.depth + 1});
    }
    return max_depth;
}

// ------------------------------------------------------------ host helpers
inline long long llround_f32(float x) { return std::llround(x); }

struct HostFacePlane {
    double n[3];
    double off;
};

std::array<double, 3> sub3(const float* a, const float* b) {
    return {double(a[0]) - double(b[0]), double(a[1]) - double(b[1]), double(a[2]) - double(b[2])};
}

std::array<double, 3> cross3(const std::array<double, 3>& a, const std::array<double, 3>& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double dot3(const std::array<double, 3>& a, const std::array<double, 3>& b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
std::array<double, 3> norm3(const std::array<double, 3>& a, double eps = 1e-6) {
    double l = std::sqrt(dot3(a, a));
    l = std::max(l, eps);
    return {a[0] / l, a[1] / l, a[2] / l};
}
double unsigned_angle(const std::array<double, 3>& a, const std::array<double, 3>& b, const std::array<double, 3>& axis) {
    auto c = cross3(a, b);
    double s = dot3(c, axis);
    double sn = (s > 0 ? 1.0 : (s < 0 ? -1.0 : 0.0)) * std::sqrt(dot3(c, c));
    double ang = std::atan2(sn, dot3(a, b));
    return ang < 0 ? ang + 2.0 * M_PI : ang;
}

template <typename T>
T* upload(SceneHandle* h, const std::vector<T>& v, cudaStream_t stream) {
    T* d = nullptr;
    size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
    if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
    h->owned.push_back(d);
    if (!v.empty()) cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream);
    return d;
}

}  // namespace

int scene_create(const float* d_vertices, int64_t nv, const int32_t* d_faces, int64_t nf, const int32_t* d_surface,
                 const int32_t* d_structure, const int32_t* d_material, int boundary_half_plane, int vertical_only,
                 double vertical_ratio, cudaStream_t stream, SceneHandle** out) {
    if (nv < 0 || nf < 0 || out == nullptr) return 1;
    if (nf > INT_MAX / 3 || nv > INT_MAX / 3) return 1;
    auto* h = new SceneHandle();
    const int F = static_cast<int>(nf);
    const int V = static_cast<int>(nv);
    std::vector<float> verts(size_t(V) * 3);
    std::vector<int> faces(size_t(F) * 3), surface(F), structure(F), material(F);
    if (V) cudaMemcpyAsync(verts.data(), d_vertices, verts.size() * 4, cudaMemcpyDeviceToHost, stream);
    if (F) {
        cudaMemcpyAsync(faces.data(), d_faces, faces.size() * 4, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(surface.data(), d_surface, F * 4, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(structure.data(), d_structure, F * 4, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(material.data(), d_material, F * 4, cudaMemcpyDeviceToHost, stream);
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) { delete h; return 2; }
    for (int i = 0; i < F * 3; ++i) {
        if (faces[i] < 0 || faces[i] >= V) { delete h; return 1; }
    }
    // ---- face planes (fp64) and fp32 unit normals
    std::vector<double> face_plane(size_t(F) * 4);
    std::vector<float> face_normal(size_t(F) * 3);
    std::vector<float> nrm32(size_t(F) * 3);
    for (int f = 0; f < F; ++f) {
        const float* a = &verts[3 * faces[3 * f]];
        const float* b = &verts[3 * faces[3 * f + 1]];
        const float* c = &verts[3 * faces[3 * f + 2]];
        auto n = norm3(cross3(sub3(b, a), sub3(c, a)));
        face_plane[4 * f + 0] = n[0];
        face_plane[4 * f + 1] = n[1];
        face_plane[4 * f + 2] = n[2];
        face_plane[4 * f + 3] = n[0] * a[0] + n[1] * a[1] + n[2] * a[2];
        face_normal[3 * f + 0] = float(n[0]);
        face_normal[3 * f + 1] = float(n[1]);
        face_normal[3 * f + 2] = float(n[2]);
        // fp32 normal as the reference's group keys see it
        float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        float cxv[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        float l = std::sqrt(cxv[0] * cxv[0] + cxv[1] * cxv[1] + cxv[2] * cxv[2]);
        l = std::max(l, 1e-6f);
        for (int k = 0; k < 3; ++k) nrm32[3 * f + k] = cxv[k] / l;
    }
    // ---- coplanar groups (fp32 keys, lexicographic order, stable by face)
    std::vector<std::array<long long, 5>> keys(F);
    for (int f = 0; f < F; ++f) {
        float nx = nrm32[3 * f], ny = nrm32[3 * f + 1], nz = nrm32[3 * f + 2];
        float norm = std::sqrt(nx * nx + ny * ny + nz * nz);
        float inv = norm > 1e-6f ? 1.0f / norm : 0.0f;
        nx *= inv; ny *= inv; nz *= inv;
        float major_abs = std::fabs(nx), major = nx;
        if (std::fabs(ny) > major_abs) { major_abs = std::fabs(ny); major = ny; }
        if (std::fabs(nz) > major_abs) { major = nz; }
        float sgn = major < 0.0f ? -1.0f : 1.0f;
        nx *= sgn; ny *= sgn; nz *= sgn;
        const float* a = &verts[3 * faces[3 * f]];
        float offset = nx * a[0] + ny * a[1] + nz * a[2];
        float scale = float(1.0 / kPlaneGroupQuant);
        keys[f] = {static_cast<long long>(surface[f]), llround_f32(nx * scale), llround_f32(ny * scale),
                   llround_f32(nz * scale), llround_f32(offset * scale)};
    }
    std::vector<int> order(F);
    for (int f = 0; f < F; ++f) order[f] = f;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return keys[x] < keys[y]; });
    std::vector<int> face_group(F), group_rep;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < F; ++i) {
        const int f = order[i];
        if (i == 0 || keys[f] != keys[order[i - 1]]) {
            group_rep.push_back(f);
            members.emplace_back();
        }
        face_group[f] = int(group_rep.size()) - 1;
        members.back().push_back(f);
    }
    const int G = int(group_rep.size());
    std::vector<int> member_off(G + 1, 0), member_list;
    std::vector<double> group_plane(size_t(G) * 4);
    std::vector<float> group_box(size_t(G) * 6);
    for (int g = 0; g < G; ++g) {
        std::sort(members[g].begin(), members[g].end());
        member_off[g] = int(member_list.size());
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int f : members[g]) {
            member_list.push_back(f);
            for (int k = 0; k < 3; ++k) {
                const float* p = &verts[3 * faces[3 * f + k]];
                for (int ax = 0; ax < 3; ++ax) {
                    lo[ax] = std::min(lo[ax], p[ax]);
                    hi[ax] = std::max(hi[ax], p[ax]);
                }
            }
        }
        for (int ax = 0; ax < 3; ++ax) {
            const float pad = float(kPlaneTolerance) + 1e-6f * std::max(std::fabs(lo[ax]), std::fabs(hi[ax]));
            group_box[6 * g + ax] = lo[ax] - pad;
            group_box[6 * g + 3 + ax] = hi[ax] + pad;
        }
        const int rep = group_rep[g];
        for (int k = 0; k < 4; ++k) group_plane[4 * g + k] = face_plane[4 * rep + k];
    }
    member_off[G] = int(member_list.size());
    // ---- diffraction edges: per-structure unique undirected edges
    struct Rec { int v0, v1, f0, f1; };
    std::vector<Rec> recs;
    {
        std::vector<int> structs(structure.begin(), structure.end());
        std::sort(structs.begin(), structs.end());
        structs.erase(std::unique(structs.begin(), structs.end()), structs.end());
        std::vector<std::vector<int>> faces_of(structs.size());
        for (int f = 0; f < F; ++f) {
            auto it = std::lower_bound(structs.begin(), structs.end(), structure[f]);
            faces_of[it - structs.begin()].push_back(f);
        }
        for (auto& fl : faces_of) {
            std::map<std::pair<int, int>, std::vector<int>> table;
            for (int f : fl) {
                int vv[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
                for (int k = 0; k < 3; ++k) {
                    int u = vv[k], w = vv[(k + 1) % 3];
                    table[{std::min(u, w), std::max(u, w)}].push_back(f);
                }
            }
            for (auto& kv : table) {
                auto v = kv.second;
                std::sort(v.begin(), v.end());
                recs.push_back({kv.first.first, kv.first.second, v[0], v.size() > 1 ? v[1] : -1});
            }
        }
    }
    const int NE = int(recs.size());
    std::vector<char> sel(NE, 0), boundary(NE, 0);
    std::vector<std::array<double, 3>> epos(NE), edir(NE), n0o(NE), n1o(NE), opp0(NE);
    std::vector<double> elen(NE), ext(NE);
    std::vector<int> face0(NE), face1(NE), mat0(NE), mat1(NE);
    std::vector<int> fn0(NE), fn1(NE);  // faces whose unit normals are n0 and n1 (-1: n1 = -n0)
    std::vector<unsigned char> state(NE, 0);  // refit cache: wedge order, coplanar, selected before merges, final
    std::vector<long long> qkey(size_t(NE) * 6, 0);
    std::vector<int> partner(NE, -1);
    std::vector<int> qhead(NE, -1);  // refit cache: first record of a candidate's endpoint class
    auto fnormal = [&](int f) { return std::array<double, 3>{face_plane[4 * f], face_plane[4 * f + 1], face_plane[4 * f + 2]}; };
    auto opposite = [&](int f, int a, int b) {
        for (int k = 0; k < 3; ++k) {
            int v = faces[3 * f + k];
            if (v != a && v != b) return v;
        }
        return faces[3 * f + 2];
    };
    for (int e = 0; e < NE; ++e) {
        const Rec& r = recs[e];
        const bool bnd = r.f0 >= 0 && r.f1 < 0;
        const bool interior = r.f0 >= 0 && r.f1 >= 0;
        const int s0 = std::max(r.f0, 0), s1 = std::max(r.f1, 0);
        const float* st = &verts[3 * r.v0];
        const float* en = &verts[3 * r.v1];
        auto vec = sub3(en, st);
        double L = std::max(std::sqrt(dot3(vec, vec)), 1e-12);
        std::array<double, 3> d = {vec[0] / L, vec[1] / L, vec[2] / L};
        auto n0c = norm3(fnormal(s0));
        auto n1c = norm3(fnormal(s1));
        auto to1 = norm3(cross3(n0c, d));
        auto tn1 = norm3(cross3(n1c, d));
        const bool first = unsigned_angle(to1, tn1, d) < unsigned_angle(tn1, to1, d);
        auto on0 = first ? n0c : n1c;
        auto on1 = first ? n1c : n0c;
        auto out0 = interior ? on0 : n0c;
        auto out1 = interior ? on1 : n1c;
        if (r.f1 < 0) out1 = {-n0c[0], -n0c[1], -n0c[2]};
        double inter = std::acos(std::min(std::max(-dot3(out0, out1), -1.0), 1.0));
        ext[e] = interior ? (2.0 * M_PI - inter) : 2.0 * M_PI;
        bool coplanar = false;
        if (interior) {
            const bool aligned = std::fabs(dot3(n0c, n1c)) >= kNormalCosTol;
            auto pa = sub3(&verts[3 * opposite(s0, r.v0, r.v1)], st);
            auto pb = sub3(&verts[3 * opposite(s1, r.v0, r.v1)], st);
            coplanar = aligned && std::fabs(dot3(pa, n0c)) <= kEdgePlaneTol && std::fabs(dot3(pb, n0c)) <= kEdgePlaneTol;
        }
        const bool wedge_ok = bnd || (interior && dot3(n0c, n1c) < 1.0);
        sel[e] = (interior || bnd) && !coplanar && L > 1e-6 && wedge_ok;
        state[e] = (first ? 1 : 0) | (coplanar ? 2 : 0) | (sel[e] ? 4 : 0);
        boundary[e] = r.f1 < 0;
        epos[e] = {0.5 * (double(st[0]) + en[0]), 0.5 * (double(st[1]) + en[1]), 0.5 * (double(st[2]) + en[2])};
        edir[e] = d;
        elen[e] = L;
        n0o[e] = out0;
        n1o[e] = out1;
        const bool swapped = interior && !first;
        const int of = swapped ? s1 : s0;
        const float* op = &verts[3 * opposite(of, r.v0, r.v1)];
        opp0[e] = {double(op[0]), double(op[1]), double(op[2])};
        face0[e] = r.f0;
        face1[e] = r.f1;
        mat0[e] = swapped ? r.f1 : r.f0;
        mat1[e] = swapped ? r.f0 : r.f1;
        fn0[e] = interior ? (first ? s0 : s1) : s0;
        fn1[e] = interior ? (first ? s1 : s0) : -1;
    }
    // shared boundary merge: group boundary records by quantized endpoints
    {
        std::map<std::array<long long, 6>, std::vector<int>> groups;
        for (int e = 0; e < NE; ++e) {
            if (!(sel[e] && boundary[e])) continue;
            const float* a = &verts[3 * recs[e].v0];
            const float* b = &verts[3 * recs[e].v1];
            std::array<long long, 3> pa, pb;
            for (int k = 0; k < 3; ++k) {
                pa[k] = std::llround(double(a[k]) / kEndpointQuant);
                pb[k] = std::llround(double(b[k]) / kEndpointQuant);
            }
            std::array<long long, 6> key;
            if (pa <= pb) key = {pa[0], pa[1], pa[2], pb[0], pb[1], pb[2]};
            else key = {pb[0], pb[1], pb[2], pa[0], pa[1], pa[2]};
            for (int k = 0; k < 6; ++k) qkey[size_t(e) * 6 + k] = key[k];
            groups[key].push_back(e);
        }
        int candidates = 0;
        for (auto& kv : groups) {
            candidates += int(kv.second.size());
            for (int x : kv.second) qhead[x] = kv.second[0];
        }
        if (candidates >= 2) {
            for (auto& kv : groups) {
                auto& g = kv.second;
                if (g.size() < 2) continue;
                const int a = g[0], b = g[1];
                double nd = std::min(std::max(dot3(n0o[a], n0o[b]), -1.0), 1.0);
                double interior_angle = std::acos(std::min(std::max(-nd, -1.0), 1.0));
                double merged = 2.0 * M_PI - interior_angle;
                bool copl = std::fabs(nd) >= kNormalCosTol;
                sel[a] = (merged > M_PI * (1.0 + 1e-6)) && !copl;
                sel[b] = 0;
                n1o[a] = n0o[b];
                fn1[a] = fn0[b];
                face1[a] = face0[b];
                mat1[a] = mat0[b];
                ext[a] = merged;
                boundary[a] = 0;
                partner[a] = b;
                partner[b] = -2;
                for (size_t x = 2; x < g.size(); ++x) {
                    sel[g[x]] = 0;
                    partner[g[x]] = -2;
                }
            }
        }
    }
    std::vector<EdgeDev> edges;
    std::vector<int> edge_ids;
    std::vector<int> edge_topo;  // per selected edge: va, vb (dir = vb - va), fn0, fn1
    for (int e = 0; e < NE; ++e) {
        if (!boundary_half_plane && boundary[e]) sel[e] = 0;
        if (vertical_only) {
            auto dv = sub3(&verts[3 * recs[e].v1], &verts[3 * recs[e].v0]);
            double lz = std::max(std::sqrt(dot3(dv, dv)), 1e-6);
            if (!(std::fabs(dv[2]) / lz > vertical_ratio)) sel[e] = 0;
        }
        if (sel[e]) state[e] |= 8;
        if (!sel[e]) continue;
        EdgeDev ed;
        std::memset(&ed, 0, sizeof(ed));
        // Wedge frame of the reference's ray-tracing library: the record's own
        // direction (v0 -> v1) and t0 = normalize(n0 x dir), phi measured from t0
        // towards n0 (native/channel/kernels/diffraction.cu:450-452).  The
        // ordered normals make t0 point into face 0 of an interior wedge; a
        // half-plane's t0 may point away from its sheet.
        const auto dir = edir[e];
        const auto t0 = norm3(cross3(n0o[e], dir));
        std::array<double, 3> to_opp = {opp0[e][0] - epos[e][0], opp0[e][1] - epos[e][1], opp0[e][2] - epos[e][2]};
        const bool into_face0 = dot3(to_opp, t0) >= 0.0;
        edge_topo.push_back(recs[e].v0);
        edge_topo.push_back(recs[e].v1);
        edge_topo.push_back(fn0[e]);
        edge_topo.push_back(fn1[e]);
        // visibility offset: the exterior bisector; for a half-plane the in-plane
        // direction away from the sheet
        std::array<double, 3> bis = {n0o[e][0] + n1o[e][0], n0o[e][1] + n1o[e][1], n0o[e][2] + n1o[e][2]};
        double bl = std::sqrt(dot3(bis, bis));
        if (bl > 1e-6) bis = {bis[0] / bl, bis[1] / bl, bis[2] / bl};
        else if (into_face0) bis = {-t0[0], -t0[1], -t0[2]};
        else bis = t0;
        for (int k = 0; k < 3; ++k) {
            ed.pos[k] = epos[e][k];
            ed.dir[k] = dir[k];
            ed.t0[k] = t0[k];
            ed.n0[k] = n0o[e][k];
            ed.n1[k] = n1o[e][k];
            ed.bisector[k] = bis[k];
        }
        ed.half_length = 0.5 * elen[e];
        ed.n = ext[e] / M_PI;
        ed.face0 = face0[e];
        ed.face1 = face1[e];
        ed.mat_face0 = mat0[e];
        ed.mat_face1 = mat1[e] >= 0 ? mat1[e] : mat0[e];
        ed.face_n = face1[e] >= 0 ? 1 : 0;
        ed.edge_id = e;
        edges.push_back(ed);
        edge_ids.push_back(e);
    }
    // ---- upload tables
    SceneDev& sd = h->dev;
    std::memset(&sd, 0, sizeof(sd));
    sd.num_vertices = V;
    sd.num_faces = F;
    sd.num_groups = G;
    sd.num_edges = int(edges.size());
    sd.vertices = upload(h, verts, stream);
    sd.faces = upload(h, faces, stream);
    sd.face_normal = upload(h, face_normal, stream);
    sd.face_plane = upload(h, face_plane, stream);
    sd.face_group = upload(h, face_group, stream);
    sd.face_material = upload(h, material, stream);
    sd.group_rep = upload(h, group_rep, stream);
    sd.group_member_off = upload(h, member_off, stream);
    sd.group_members = upload(h, member_list, stream);
    sd.group_plane = upload(h, group_plane, stream);
    sd.group_box = upload(h, group_box, stream);
    sd.edges = upload(h, edges, stream);
    h->edge_ids = upload(h, edge_ids, stream);
    h->edge_topo = upload(h, edge_topo, stream);
    {
        std::vector<int> slot(std::max(NE, 1), -1);
        for (size_t i = 0; i < edge_ids.size(); ++i) slot[edge_ids[i]] = int(i);
        h->edge_slot = upload(h, slot, stream);
    }
    h->group_rep_host = group_rep;
    h->face_group_host = face_group;
    h->num_edges_total = NE;
    // caches of the discrete decisions for scene_refit
    {
        std::vector<long long> fkeys(size_t(F) * 5);
        for (int f = 0; f < F; ++f)
            for (int k = 0; k < 5; ++k) fkeys[size_t(f) * 5 + k] = keys[f][k];
        std::vector<int4> erec(NE);
        for (int e = 0; e < NE; ++e) erec[e] = make_int4(recs[e].v0, recs[e].v1, recs[e].f0, recs[e].f1);
        h->face_surface = upload(h, surface, stream);
        h->face_keys = upload(h, fkeys, stream);
        h->edge_rec = upload(h, erec, stream);
        h->edge_state = upload(h, state, stream);
        h->edge_qkey = upload(h, qkey, stream);
        h->edge_partner = upload(h, partner, stream);
        h->edge_qhead = upload(h, qhead, stream);
        int slots = 1;
        while (slots < 2 * std::max(std::max(G, NE), 1)) slots <<= 1;
        h->key_table = upload(h, std::vector<int>(slots, -1), stream);
        h->key_table_slots = slots;
        h->refit_flag = upload(h, std::vector<int>(1, 0), stream);
        h->diagonal_dev = upload(h, std::vector<double>(1, 0.0), stream);
        h->half_plane_policy = boundary_half_plane;
        h->vertical_only_policy = vertical_only;
        h->vertical_ratio = vertical_ratio;
    }
    // bounds
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < V; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], verts[3 * i + k]);
            hi[k] = std::max(hi[k], verts[3 * i + k]);
        }
    sd.diagonal = V ? std::sqrt(double(hi[0] - lo[0]) * (hi[0] - lo[0]) + double(hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                double(hi[2] - lo[2]) * (hi[2] - lo[2]))
                    : 0.0;
    // ---- BVH (host binned SAH) and triangles in leaf order
    sd.root = INT_MIN;
    sd.max_depth = 0;
    sd.stack_entries = 8;
    if (F > 0) {
        std::vector<BvhNode> host_nodes;
        std::vector<int> slot_face;
        int hdepth = 0;
        if (F > 1) {
            hdepth = build_bvh(verts, faces, F, host_nodes, slot_face);
        } else {
            slot_face.assign(1, 0);
            host_nodes.assign(1, BvhNode{});
        }
        if (hdepth >= kStackDepth) { scene_destroy(h); return 4; }
        std::vector<float4> tri(size_t(F) * 3);
        for (int sl = 0; sl < F; ++sl) {
            const int f = slot_face[sl];
            const float* a = &verts[3 * faces[3 * f]];
            const float* b = &verts[3 * faces[3 * f + 1]];
            const float* c = &verts[3 * faces[3 * f + 2]];
            float fbits, gbits;
            std::memcpy(&fbits, &f, 4);
            std::memcpy(&gbits, &face_group[f], 4);
            tri[3 * sl + 0] = make_float4(a[0], a[1], a[2], fbits);
            tri[3 * sl + 1] = make_float4(b[0], b[1], b[2], gbits);
            tri[3 * sl + 2] = make_float4(c[0], c[1], c[2], 0.0f);
        }
        // parent links for the refit: node << 1 | side (-1 at the root)
        std::vector<int> leaf_parent(F, -1), node_parent(std::max(F - 1, 1), -1);
        if (F > 1)
            for (int i = 0; i < int(host_nodes.size()); ++i) {
                const int ch[2] = {host_nodes[i].d.x, host_nodes[i].d.y};
                for (int side = 0; side < 2; ++side) {
                    if (ch[side] >= 0) node_parent[ch[side]] = (i << 1) | side;
                    else leaf_parent[~ch[side]] = (i << 1) | side;
                }
            }
        h->leaf_parent = upload(h, leaf_parent, stream);
        h->node_parent = upload(h, node_parent, stream);
        h->bvh_counter = upload(h, std::vector<int>(std::max(F - 1, 1), 0), stream);
        sd.tri = upload(h, tri, stream);
        sd.nodes = upload(h, host_nodes, stream);
        if (sd.tri == nullptr || sd.nodes == nullptr) { scene_destroy(h); return 2; }
        sd.root = F > 1 ? 0 : ~0;
        sd.max_depth = hdepth;
        sd.stack_entries = std::max(8, std::min(kStackDepth, hdepth + 2));
        h->num_nodes = std::max(F - 1, 0);
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) { scene_destroy(h); return 2; }
    *out = h;
    return 0;
}

void scene_destroy(SceneHandle* h) {
    if (!h) return;
    for (void* p : h->owned) cudaFree(p);
    delete h;
}

}  // namespace wcb
