// Explicit instantiations of the 2D stage kernels: shallow water, Maxwell.
#include "stage2d.cuh"

namespace mxm {
using SR2D = ShallowWater2D<double, FLUX_RUSANOV>;
using SR2F = ShallowWater2D<float, FLUX_RUSANOV>;
using SH2D = ShallowWater2D<double, FLUX_HLL>;
using SH2F = ShallowWater2D<float, FLUX_HLL>;
using M2D = Maxwell2D<double>;
using M2F = Maxwell2D<float>;
MXM_INSTANTIATE_STAGE2D(double, SR2D)
MXM_INSTANTIATE_STAGE2D(float, SR2F)
MXM_INSTANTIATE_STAGE2D(double, SH2D)
MXM_INSTANTIATE_STAGE2D(float, SH2F)
MXM_INSTANTIATE_STAGE2D(double, M2D)
MXM_INSTANTIATE_STAGE2D(float, M2F)
}  // namespace mxm
