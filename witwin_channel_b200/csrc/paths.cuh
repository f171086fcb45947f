// Per-path geometry shared by the fused solve kernel and the per-row
// evaluation kernels: image-method back projection, containment in a
// coplanar group, and the straight-segment penetration list.
#pragma once

#include "common.cuh"
#include "scene.cuh"
#include "traverse.cuh"

namespace wcb {

constexpr int kMaxDepth = 5;
constexpr double kPlaneTol = 1.0e-3;   // rayd/reflection.cpp:50 plane_tolerance
constexpr double kBaryEps = 1.0e-7;
constexpr double kSegEps = 1.0e-6;

// Point-in-face test in FP64: within the plane tolerance of the face plane
// and inside the triangle (edges inclusive, 1e-7 barycentric slack).
WCB_D bool point_in_face(const SceneDev& sc, int f, V3<double> p) {
    const double* pl = sc.face_plane + 4 * f;
    const V3<double> n = v3(pl[0], pl[1], pl[2]);
    const int ia = sc.faces[3 * f], ib = sc.faces[3 * f + 1], ic = sc.faces[3 * f + 2];
    const V3<double> a = v3<double>(sc.vertices[3 * ia], sc.vertices[3 * ia + 1], sc.vertices[3 * ia + 2]);
    const double dist = dot(p - a, n);
    if (fabs(dist) > kPlaneTol) return false;
    const V3<double> b = v3<double>(sc.vertices[3 * ib], sc.vertices[3 * ib + 1], sc.vertices[3 * ib + 2]);
    const V3<double> c = v3<double>(sc.vertices[3 * ic], sc.vertices[3 * ic + 1], sc.vertices[3 * ic + 2]);
    const V3<double> q = p - n * dist;
    const V3<double> e1 = b - a, e2 = c - a, w = q - a;
    const double d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
    const double w1 = dot(w, e1), w2 = dot(w, e2);
    const double den = d11 * d22 - d12 * d12;
    if (!(den > 0.0)) return false;
    const double v = (d22 * w1 - d12 * w2) / den;
    const double u = (d11 * w2 - d12 * w1) / den;
    return v >= -kBaryEps && u >= -kBaryEps && u + v <= 1.0 + kBaryEps;
}

// Lowest-index member of group g containing p, or -1.
WCB_D int resolve_in_group(const SceneDev& sc, int g, V3<double> p) {
    const float* bx = sc.group_box + 6 * g;
    if (p.x < bx[0] || p.y < bx[1] || p.z < bx[2] || p.x > bx[3] || p.y > bx[4] || p.z > bx[5]) return -1;
    const int beg = sc.group_member_off[g], end = sc.group_member_off[g + 1];
    for (int i = beg; i < end; ++i) {
        const int f = sc.group_members[i];
        if (point_in_face(sc, f, p)) return f;
    }
    return -1;
}

// Back projection from the receiver through precomputed images (FP64).
// planes[k] = (n, off); images[k] = image of the source after k+1 mirrors.
// Writes the hit points, returns false when a back-projected line does not
// cross its plane strictly between its ends.
// One step: moves x to its hit on plane k along the line to image k; false
// when that line does not cross the plane strictly between its ends.
WCB_D bool back_project_step(V3<double>& x, const double* planes, const double* images, int k) {
    const V3<double> n = v3(planes[4 * k], planes[4 * k + 1], planes[4 * k + 2]);
    const double off = planes[4 * k + 3];
    const V3<double> img = v3(images[3 * k], images[3 * k + 1], images[3 * k + 2]);
    const double denom = dot(img - x, n);
    if (denom == 0.0) return false;
    const double t = (off - dot(x, n)) / denom;
    if (!(t > kSegEps && t < 1.0 - kSegEps)) return false;
    x = x + (img - x) * t;
    return true;
}

WCB_D bool back_project(V3<double> R, const double* planes, const double* images, int depth, V3<double>* hits) {
    V3<double> x = R;
    for (int k = depth - 1; k >= 0; --k) {
        if (!back_project_step(x, planes, images, k)) return false;
        hits[k] = x;
    }
    return true;
}

// Ends of segment s of a back-projected chain of `depth` bounces (S or hit
// s-1, and hit s or R) with the same arithmetic as back_project and no hit
// array; false when the back projection fails.
WCB_D bool back_project_segment(V3<double> S, V3<double> R, const double* planes, const double* images, int depth,
                                int s, V3<double>* a, V3<double>* b) {
    V3<double> x = R;
    *a = S;
    *b = R;
    for (int k = depth - 1; k >= 0 && k >= s - 1; --k) {
        if (!back_project_step(x, planes, images, k)) return false;
        if (k == s) *b = x;
        if (k == s - 1) *a = x;
    }
    return true;
}

// FP32 pre-test of the last bounce: the back-projected point must fall in the
// (padded) group box.  Conservative: it only rejects candidates whose FP64
// solve fails too.  `pre` holds the chain's last plane and last image.
WCB_D bool back_project_prefilter(const SceneDev& sc, V3<float> R, const float4* pre) {
    const float4 pl = __ldg(pre);
    const float4 im = __ldg(pre + 1);
    const V3<float> n = v3(pl.x, pl.y, pl.z);
    const float off = pl.w;
    const V3<float> img = v3(im.x, im.y, im.z);
    const float denom = dot(img - R, n);
    if (fabsf(denom) < 1e-30f) return true;  // leave the decision to FP64
    const float t = (off - dot(R, n)) / denom;
    if (!(t > -1e-3f && t < 1.0f + 1e-3f)) return false;
    const V3<float> x = R + (img - R) * t;
    const float* bx = sc.group_box + 6 * __float_as_int(im.w);
    const float pad = 1e-2f + 1e-5f * (fabsf(x.x) + fabsf(x.y) + fabsf(x.z));
    return !(x.x < bx[0] - pad || x.y < bx[1] - pad || x.z < bx[2] - pad || x.x > bx[3] + pad || x.y > bx[4] + pad ||
             x.z > bx[5] + pad);
}

// Ordered wall hits along a segment, at most kMaxDepth + 1 kept.
struct HitList {
    int count;
    int face[kMaxDepth + 1];
    int group[kMaxDepth + 1];
    double t[kMaxDepth + 1];
};

template <typename G>
struct HitSink {
    HitList* list;
    int cap;
    WCB_D bool operator()(G t, int face, int group) const {
        // duplicate crossing of one plane at one parameter (shared diagonal)
        for (int i = 0; i < list->count; ++i) {
            if (list->group[i] == group && fabs(double(t) - list->t[i]) < 1e-7) return true;
        }
        if (list->count >= cap) {
            list->count = cap + 1;  // overflow marker
            return false;
        }
        int i = list->count++;
        while (i > 0 && list->t[i - 1] > double(t)) {
            list->t[i] = list->t[i - 1];
            list->face[i] = list->face[i - 1];
            list->group[i] = list->group[i - 1];
            --i;
        }
        list->t[i] = double(t);
        list->face[i] = face;
        list->group[i] = group;
        return true;
    }
};

template <typename G>
WCB_D void segment_hits(const SceneDev& sc, V3<G> p0, V3<G> p1, int cap, HitList* out, int* stack, int* err) {
    out->count = 0;
    const Ray<G> r = make_ray<G>(p0, p1 - p0, G(kSegEps), G(1) - G(kSegEps));
    G bt = G(0);
    int bf = -1, bg = -1;
    HitSink<G> sink{out, cap};
    traverse<2, G>(sc, r, ignore_none(), stack, err, &bt, &bf, &bg, sink);
}

}  // namespace wcb
