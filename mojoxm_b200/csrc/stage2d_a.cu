// Explicit instantiations of the 2D stage kernels: advection, Euler.
#include "stage2d.cuh"

namespace mxm {
using A2D = Advection2D<double>;
using A2F = Advection2D<float>;
using ER2D = Euler2D<double, FLUX_RUSANOV>;
using ER2F = Euler2D<float, FLUX_RUSANOV>;
using EC2D = Euler2D<double, FLUX_HLLC>;
using EC2F = Euler2D<float, FLUX_HLLC>;
using EE2D = Euler2D<double, FLUX_HLLE>;
using EE2F = Euler2D<float, FLUX_HLLE>;
MXM_INSTANTIATE_STAGE2D(double, A2D)
MXM_INSTANTIATE_STAGE2D(float, A2F)
MXM_INSTANTIATE_STAGE2D(double, ER2D)
MXM_INSTANTIATE_STAGE2D(float, ER2F)
MXM_INSTANTIATE_STAGE2D(double, EC2D)
MXM_INSTANTIATE_STAGE2D(float, EC2F)
MXM_INSTANTIATE_STAGE2D(double, EE2D)
MXM_INSTANTIATE_STAGE2D(float, EE2F)
}  // namespace mxm
