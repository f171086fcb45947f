// The diffraction records' VJP kernel (dual-number UTD), in its own
// translation unit so it compiles in parallel with the other components.
#include "adjoint.cuh"

namespace wcb {
namespace adj {

// One thread per (record, parameter) over the diffraction records.
void launch_vjp_diffraction(const AdjParams& p, const int* pair_base, long long total, cudaStream_t s) {
    if (p.order_count <= 0 || total <= 0) return;
    k_vjp_pairs<2><<<unsigned((total + kBlock - 1) / kBlock), kBlock, 0, s>>>(p, pair_base, total);
}

}  // namespace adj
}  // namespace wcb
