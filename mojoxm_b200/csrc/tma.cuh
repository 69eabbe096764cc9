// Minimal sm_90+/sm_100a bulk-copy (TMA, non-tensor) + mbarrier helpers.
// Only 1D cp.async.bulk global -> shared is used, never with cluster
// multicast, and every wait is bounded: a wait that runs past its limit
// reports failure instead of spinning forever.
#pragma once
#include <stdint.h>

namespace mxm {

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any tile load or MMA batch

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Programmatic dependent launch.  grid_dep_launch: this block lets the next
// kernel of the stream (launched with programmatic stream serialisation)
// start its blocks as SMs free up.  grid_dep_wait: block until the previous
// kernel of the stream has completed and its writes are visible; every read
// of its output (and every write the previous kernel may still read) comes
// after it.  Both return at once when the launch has no such dependency.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Order this thread's earlier generic-proxy shared accesses before later
// async-proxy (bulk copy) accesses of the same shared memory.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Bring `bytes` of global memory at src into L2 ahead of their use (no
// completion to wait for); src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test_parity(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Potentially blocking test: the thread may be suspended for a short,
// hardware-defined time while the phase is incomplete.
__device__ __forceinline__ bool mbar_try_parity(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait until the barrier phase with the given parity completes, at most
// `limit_ns` nanoseconds.  Returns false when the limit was hit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_test_parity(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (true) {
    for (int k = 0; k < 16; ++k)
      if (mbar_try_parity(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// Block-wide wait: thread 0 polls the barrier (the other threads do not
// spend issue slots on it), the result is agreed by a barrier, and the
// barrier also orders the waited-for data (bulk-copy bytes, MMA results)
// before every thread's later accesses.  Must be reached by all threads.
__device__ __forceinline__ bool block_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  bool ok = true;
  if (threadIdx.x == 0) ok = mbar_wait_bounded(bar, parity, limit_ns);
  return __syncthreads_and(ok) != 0;
}

}  // namespace mxm
