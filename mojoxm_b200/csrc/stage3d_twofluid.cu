// Explicit instantiation of the 3D stage kernel family for one physics.
#include "stage3d_launch.cuh"

namespace mxm {
using PhysD = TwoFluidD<double>;
using PhysF = TwoFluidD<float>;
MXM_INSTANTIATE_STAGE3D(double, PhysD)
MXM_INSTANTIATE_STAGE3D(float, PhysF)
}  // namespace mxm
