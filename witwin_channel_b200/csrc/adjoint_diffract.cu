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

}  // namespace adj
}  // namespace wcb
