// sweep2d.cuh -- single-sweep (one fused pass per time step) 2D kernels and
// the kernel-family choice of the autotuner.
#pragma once
#include "solver2d_kernels.cuh"

namespace fomo {

// Kernel family for a problem (FOMO_KERNEL_TWO_PHASE / _SINGLE_SWEEP).
int pick_kernel_2d(int phys, int N, int nxp, int nzp, int ns);
bool sweep2d_supported(int phys, int N);
cudaError_t launch_sweep_elastic(cudaStream_t st, int N, const Geo2& g, const Coef& c, float dtx,
                                 float dtz, const HabcDev& h, const ElFields& a, const ElMat& m,
                                 const ElOut& o, int ns);

}  // namespace fomo
