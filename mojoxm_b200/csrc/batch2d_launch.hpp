// Launchers of the batched 2D kernels (instantiated in batch2d_f32.cu /
// batch2d_f64.cu) and the host-side shape arithmetic they share.
#pragma once
#include <cuda_runtime.h>

#include "../../include/mxm_dg.h"
#include "dg_common.cuh"

namespace mxm {

template <class R>
struct SolveDesc2;
template <class R>
struct Batch2DArgs;
template <class R>
struct LimBatch2DArgs;

constexpr int kBatchNT = 256;

// B-tile row stride of the 2D stage (same padding rule as Stage2DShape)
inline int bstr2d(int P, int NC, size_t rbytes) {
  const int NP = (P + 1) * (P + 2) / 2, K = 2 * NP + 3 * (P + 1);
  const int raw = K * (NC | 1), mod = rbytes == 8 ? 16 : 32;
  return raw + ((1 - raw % mod) + mod) % mod;
}

// Resident blocks per SM of the batched stage kernel for this physics and
// dynamic shared-memory size (sets the kernel's shared-memory attributes).
template <class R>
cudaError_t stage2d_batch_blocks_per_sm(const mxm_dg_physics_desc& pd, size_t smem, int* bps);
template <class R>
cudaError_t launch_stage2d_batch(const mxm_dg_physics_desc& pd, const Batch2DArgs<R>& ba, int grid, size_t smem,
                                 cudaStream_t st);
template <class R>
cudaError_t launch_lim2d_batch(int NC, const LimBatch2DArgs<R>& la, cudaStream_t st);
// Set the batched limiter's kernel attributes (before any stream capture).
template <class R>
cudaError_t prepare_lim2d_batch(int NC);

}  // namespace mxm
