// Self-test of the bounded waits that every stage kernel relies on.
//
// One block initialises an mbarrier that nothing will ever complete and
// waits on it through block_wait_bounded (the helper the stage kernels use
// for bulk copies and tensor-core commits) with a short limit.  The wait
// gives up by itself, the kernel records that and returns normally, and
// the CUDA context stays usable; no fault, trap or endless loop is involved.
#include <cuda_runtime.h>

#include "../../include/mxm_dg.h"
#include "tma.cuh"

namespace mxm {
namespace {

__global__ void wait_timeout_probe(uint64_t limit_ns, int* gave_up, unsigned long long* waited_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected; none will come
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = global_ns();
  const bool ok = block_wait_bounded(&bar, 0, limit_ns);
  if (threadIdx.x == 0) {
    gave_up[0] = ok ? 0 : 1;
    waited_ns[0] = global_ns() - t0;
  }
}

}  // namespace
}  // namespace mxm

extern "C" int mxm_dg_selftest_wait_timeout(double limit_ms, int32_t* gave_up, double* waited_ms) {
  if (!gave_up || !waited_ms || !(limit_ms >= 1.0 && limit_ms <= 2000.0)) return MXM_DG_EINVAL;
  int* d_flag = nullptr;
  unsigned long long* d_ns = nullptr;
  if (cudaMalloc(&d_flag, sizeof(int)) != cudaSuccess) return MXM_DG_ENOMEM;
  if (cudaMalloc(&d_ns, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(d_flag);
    return MXM_DG_ENOMEM;
  }
  mxm::wait_timeout_probe<<<1, 64>>>(uint64_t(limit_ms * 1e6), d_flag, d_ns);
  int flag = -1;
  unsigned long long ns = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost);
  cudaFree(d_flag);
  cudaFree(d_ns);
  if (e != cudaSuccess) return MXM_DG_ECUDA;
  *gave_up = flag;
  *waited_ms = double(ns) * 1e-6;
  return MXM_DG_OK;
}
