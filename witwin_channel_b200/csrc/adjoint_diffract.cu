// The diffraction records' VJP kernel (dual-number UTD), in its own
// translation unit so it compiles in parallel with the other components.
#include "adjoint.cuh"

namespace wcb {
namespace adj {

void launch_vjp_diffraction(const AdjParams& p, int grid, cudaStream_t s) {
    k_vjp_rows<kLanes, 2><<<grid, kBlock, 0, s>>>(p);
}

}  // namespace adj
}  // namespace wcb
