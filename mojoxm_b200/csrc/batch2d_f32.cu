// Batched 2D kernels, FP32 state.
#include "batch2d_kernels.cuh"

namespace mxm {
MXM_INSTANTIATE_BATCH2D(float)
}  // namespace mxm
