// sweep2d.cu -- single-sweep 2D kernels (not yet enabled: the autotuner
// selects the two-phase family).
#include "sweep2d.cuh"

namespace fomo {

int pick_kernel_2d(int, int, int, int, int) { return FOMO_KERNEL_TWO_PHASE; }
bool sweep2d_supported(int, int) { return false; }
cudaError_t launch_sweep_elastic(cudaStream_t, int, const Geo2&, const Coef&, float, float,
                                 const HabcDev&, const ElFields&, const ElMat&, const ElOut&, int) {
  return cudaErrorNotSupported;
}

}  // namespace fomo
