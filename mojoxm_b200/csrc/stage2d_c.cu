// Explicit instantiations of the 2D stage kernels: ideal MHD without and
// with GLM divergence cleaning.
#include "stage2d.cuh"

namespace mxm {
using MP2D = Mhd2D<double, false>;
using MP2F = Mhd2D<float, false>;
using MG2D = Mhd2D<double, true>;
using MG2F = Mhd2D<float, true>;
MXM_INSTANTIATE_STAGE2D(double, MP2D)
MXM_INSTANTIATE_STAGE2D(float, MP2F)
MXM_INSTANTIATE_STAGE2D(double, MG2D)
MXM_INSTANTIATE_STAGE2D(float, MG2F)
}  // namespace mxm
