// Batched 2D kernels, FP64 state.
#include "batch2d_kernels.cuh"

namespace mxm {
MXM_INSTANTIATE_BATCH2D(double)
}  // namespace mxm
