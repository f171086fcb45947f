// The diffraction records' VJP kernel (dual-number UTD), in its own
// translation unit so it compiles in parallel with the other components.
#include "adjoint.cuh"

namespace wcb {
namespace adj {

void launch_vjp_diffraction(const AdjParams& p, cudaStream_t s) {
    if (p.order_count <= 0) return;
    k_vjp_rows<kLanes, 2><<<unsigned((p.order_count + kBlock - 1) / kBlock), kBlock, 0, s>>>(p);
}

}  // namespace adj
}  // namespace wcb
