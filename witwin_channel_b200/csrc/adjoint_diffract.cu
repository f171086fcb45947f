// The diffraction records' VJP and JVP kernels (dual-number UTD), in their own
// translation unit so they compile in parallel with the other components.
#include "adjoint.cuh"

namespace wcb {
namespace adj {

// Reverse mode over the diffraction records (one thread per record).
void launch_vjp_diffraction(const AdjParams& p, cudaStream_t s) {
    if (p.order_count <= 0) return;
    k_vjp_diffraction<2><<<unsigned((p.order_count + kBlock - 1) / kBlock), kBlock, 0, s>>>(p);
}

// Forward mode over the diffraction records (one thread per record).
void launch_jvp_diffraction(const AdjParams& p, const double* tangent, double* field, double* field_tangent,
                            cudaStream_t s) {
    if (p.count <= 0) return;
    k_jvp_rows<2><<<unsigned((p.count + kBlock - 1) / kBlock), kBlock, 0, s>>>(p, tangent, field, field_tangent);
}

// The diffraction records' plain FP64 fields (one thread per record).
void launch_field64_diffraction(const AdjParams& p, double* field, cudaStream_t s) {
    if (p.count <= 0) return;
    k_field64_rows<2><<<unsigned((p.count + kBlock - 1) / kBlock), kBlock, 0, s>>>(p, field);
}

// The diffraction records' plain FP64 fields at every frequency of `fs`: the
// frequency-independent UTD geometry (stationary point, angles, bases) once
// per record, then the field at each frequency with that frequency's face
// materials (p's material pointers at frequency 0, rows of num_materials).
// field is (nf, K, 2).
__global__ void __launch_bounds__(kBlock) k_field64_diffraction_multi(AdjParams p, int nf, FreqSet fs,
                                                                      double* field) {
    using D = Dual<0>;
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= p.order_count) return;
    const long long i = p.order ? p.order[p.order_begin + j] : j;
    const RowRec row = p.rows[p.selected[i]];
    if (row.component != 2) return;
    const Plain<0> w{};
    const int t = row.tx, r = row.rx;
    const V3<D> S = v3(D(p.tx_pos[3 * t]), D(p.tx_pos[3 * t + 1]), D(p.tx_pos[3 * t + 2]));
    const V3<D> R = receiver(p, w, r);
    const V3<D> tx_pol = v3(D(p.tx_pol[3 * t]), D(p.tx_pol[3 * t + 1]), D(p.tx_pol[3 * t + 2]));
    const float* rp = p.rx_pol + (long long)r * p.rx_pol_stride;
    const V3<D> rx_pol = v3(D(rp[0]), D(rp[1]), D(rp[2]));
    const double sq = sqrt(fmax(double(p.tx_power[t]), 0.0));
    const V3<D> ez = v3(D(0.0), D(0.0), D(1.0));
    const int slot = p.edge_slot[row.edge];
    const EdgeDev& ed = p.sc.edges[slot];
    const EdgeFrame<D> fr = edge_frame_dual(p, w, slot);
    const UtdGeometry<D, D> geo = utd_geometry<D, D>(fr, S, R, tx_pol);
    const int m0 = p.sc.face_material[ed.mat_face0], m1 = p.sc.face_material[ed.mat_face1];
    const long long M = p.num_materials, K = p.count;
#pragma unroll 1
    for (int c = 0; c < nf; ++c) {
        const long long o = c * M;
        const Slab<D> s0{D(p.eps_r[o + m0]), D(p.sigma_e[o + m0]), D(p.mu_r[o + m0]), D(p.gain[o + m0]),
                         D(p.thickness[o + m0])};
        const Slab<D> s1{D(p.eps_r[o + m1]), D(p.sigma_e[o + m1]), D(p.mu_r[o + m1]), D(p.gain[o + m1]),
                         D(p.thickness[o + m1])};
        V3<D> q;
        const DiffractionResult<D> res = utd_result(geo, fr, s0, s1, D(fs.f[c]), &q);
        const V3<D> dir = safe_normalize(R - q, ez);
        const Cx<D> coef = project_receiver(res.field, dir, rx_pol);
        field[2 * (c * K + i)] = coef.re.v * sq;
        field[2 * (c * K + i) + 1] = coef.im.v * sq;
    }
}

void launch_field64_diffraction_multi(const AdjParams& p, int nf, const FreqSet& fs, double* field, cudaStream_t s) {
    if (p.order_count <= 0) return;
    k_field64_diffraction_multi<<<unsigned((p.order_count + kBlock - 1) / kBlock), kBlock, 0, s>>>(p, nf, fs, field);
}

}  // namespace adj
}  // namespace wcb
