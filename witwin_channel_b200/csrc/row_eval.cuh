// Evaluation of one line-of-sight or reflection record, shared by the row
// evaluation kernel (discovered records) and the fixed-topology replay kernel
// (frozen records at new endpoints), so both publish bit-identical numbers
// for the same record at the same endpoints.
#pragma once

#include "em.cuh"
#include "paths.cuh"

namespace wcb {

// Image-method geometry of a reflection record: every bounce on the plane of
// the coplanar group of its recorded face (reference propagation/geometry.py:
// 214-264, the direct-plane EPC re-solve).  `length` is |R - last image|.
// `solved` is false when a back-projected line misses its plane between its
// ends; the hits are then NaN.
struct ReflectionGeom {
    V3<double> hits[kMaxDepth];
    double length;
    bool solved;
};

WCB_D ReflectionGeom reflection_geometry(const SceneDev& sc, const int* faces, int d, V3<double> S, V3<double> R) {
    ReflectionGeom g;
    double planes[4 * kMaxDepth], images[3 * kMaxDepth];
    V3<double> pp = S;
    for (int k = 0; k < d; ++k) {
        const int grp = sc.face_group[faces[k]];
        const double* pl = sc.group_plane + 4 * grp;
        for (int q = 0; q < 4; ++q) planes[4 * k + q] = pl[q];
        const V3<double> n = v3(pl[0], pl[1], pl[2]);
        pp = pp - n * (2.0 * (dot(pp, n) - pl[3]));
        images[3 * k] = pp.x;
        images[3 * k + 1] = pp.y;
        images[3 * k + 2] = pp.z;
    }
    g.solved = back_project(R, planes, images, d, g.hits);
    if (!g.solved) {
        for (int k = 0; k < d; ++k) g.hits[k] = v3(nan(""), nan(""), nan(""));
    }
    g.length = length(R - pp);
    return g;
}

// Unit-excitation field of a reflection record at one frequency: the source
// polarisation made transverse to the first leg, one Fresnel/Jones bounce per
// recorded face (its own normal and material), then the spreading and phase
// of the unfolded length.  `slab(face)` returns the face's material at this
// frequency.  Writes the bounce normals, the world-Cartesian field, its
// projection on rx_pol and the arrival direction.
template <class SlabAt>
WCB_D void reflection_field(const SceneDev& sc, const int* faces, int d, const ReflectionGeom& g, V3<float> Sf,
                            V3<float> Rf, V3<float> tx_pol, V3<float> rx_pol, const SlabAt& slab, double freq, double k,
                            V3<float>* normals, C3<float>* unit_field, Cx<float>* coef, V3<float>* dir) {
    const float wl = float(kC0 / freq);
    V3<float> prev = Sf;
    V3<float> incident = safe_normalize(cast3<float>(g.hits[0]) - prev, v3(0.f, 0.f, 1.f));
    C3<float> value = c3_from_real(transverse(incident, tx_pol));
    V3<float> outgoing = incident;
    for (int b = 0; b < d; ++b) {
        const V3<float> hit = cast3<float>(g.hits[b]);
        incident = safe_normalize(hit - prev, outgoing);
        const float* nf = sc.face_normal + 3 * faces[b];
        normals[b] = v3(nf[0], nf[1], nf[2]);
        reflect_bounce(value, outgoing, incident, normals[b], slab(faces[b]), freq, wl);
        prev = hit;
    }
    *dir = safe_normalize(Rf - prev, outgoing);
    const float amp = 1.0f / (2.0f * float(k) * float(fmax(g.length, kUtdEps)));
    value = c3_scale(value, phasor_neg_kd<float>(k, g.length) * amp);
    *unit_field = value;
    *coef = project_receiver(value, *dir, rx_pol);
}

// Transverse frame of one endpoint for the propagation direction `dir`
// (consumer_los_jones, native/channel/kernels/los.cu:1964-1980): u is the
// first reference vector made transverse and unit (falling back to the
// transverse part of the second, then to a fixed axis); v = dir x u, turned
// to the side of the second vector.
WCB_D void endpoint_frame(const float* ref, long long e, V3<float> dir, V3<float>* u, V3<float>* v) {
    const V3<float> first = v3(ref[6 * e], ref[6 * e + 1], ref[6 * e + 2]);
    const V3<float> second = v3(ref[6 * e + 3], ref[6 * e + 4], ref[6 * e + 5]);
    const V3<float> fallback = stable_perp_basis(dir, second);
    const V3<float> fu = safe_normalize(transverse(dir, first), fallback);
    V3<float> fv = safe_normalize(cross(dir, fu), fallback);
    if (dot(fv, second) < 0.f) fv = fv * -1.f;
    *u = fu;
    *v = fv;
}

}  // namespace wcb
