// Physics dispatch and explicit instantiation of the batched 2D kernels for
// one real type (included by batch2d_f32.cu and batch2d_f64.cu).
#pragma once
#include "batch2d.cuh"
#include "batch2d_launch.hpp"

namespace mxm {

// Build the 2D physics functor of a descriptor and call f(ph); the
// parameter layout is the one mxm_dg_physics_desc documents.
template <class R, class F>
cudaError_t with_phys2d(const mxm_dg_physics_desc& pd, F&& f) {
  const double* p = pd.p;
  switch (pd.kind) {
    case MXM_DG_PHYS_ADVECTION: {
      Advection2D<R> ph{R(p[0]), R(p[1]), R(p[3])};
      return f(ph);
    }
    case MXM_DG_PHYS_EULER: {
      auto mk = [&](auto ph) {
        ph.gamma = R(p[0]); ph.rho_min = R(p[1]); ph.p_min = R(p[2]);
        ph.gx = R(p[3]); ph.gy = R(p[4]);
        ph.inflow[0] = R(p[6]); ph.inflow[1] = R(p[7]); ph.inflow[2] = R(p[8]); ph.inflow[3] = R(p[10]);
        ph.entropy_fix = pd.entropy_fix;
        return f(ph);
      };
      switch (pd.flux_type) {
        case MXM_DG_FLUX_RUSANOV: return mk(Euler2D<R, FLUX_RUSANOV>{});
        case MXM_DG_FLUX_HLLC: return mk(Euler2D<R, FLUX_HLLC>{});
        case MXM_DG_FLUX_HLLE: return mk(Euler2D<R, FLUX_HLLE>{});
      }
      return cudaErrorInvalidValue;
    }
    case MXM_DG_PHYS_SHALLOW_WATER: {
      auto mk = [&](auto ph) {
        ph.g = R(p[0]); ph.h_min = R(p[1]);
        for (int k = 0; k < 3; ++k) ph.inflow[k] = R(p[2 + k]);
        return f(ph);
      };
      if (pd.flux_type == MXM_DG_FLUX_HLL) return mk(ShallowWater2D<R, FLUX_HLL>{});
      return mk(ShallowWater2D<R, FLUX_RUSANOV>{});
    }
    case MXM_DG_PHYS_MAXWELL: {
      Maxwell2D<R> ph;
      ph.c = R(p[0]);
      for (int k = 0; k < 3; ++k) { ph.J[k] = R(p[1 + k]); ph.M[k] = R(p[4 + k]); }
      for (int k = 0; k < 6; ++k) ph.inflow[k] = R(p[7 + k]);
      return f(ph);
    }
    case MXM_DG_PHYS_MHD:
    case MXM_DG_PHYS_MHD_PLAIN: {  // state (rho, mx, my, Bx, By, E[, psi]) from the 3D layout
      auto mk = [&](auto ph) {
        ph.gamma = R(p[0]); ph.rho_min = R(p[1]); ph.p_min = R(p[2]); ph.c_h = R(p[3]);
        const int map[7] = {5, 6, 7, 10, 11, 9, 13};
        for (int k = 0; k < 7; ++k) ph.inflow[k] = R(p[map[k]]);
        return f(ph);
      };
      if (pd.kind == MXM_DG_PHYS_MHD) return mk(Mhd2D<R, true>{});
      return mk(Mhd2D<R, false>{});
    }
  }
  return cudaErrorInvalidValue;
}

template <class R>
cudaError_t stage2d_batch_blocks_per_sm(const mxm_dg_physics_desc& pd, size_t smem, int* bps) {
  return with_phys2d<R>(pd, [&](const auto& ph) -> cudaError_t {
    using Ph = typename std::decay<decltype(ph)>::type;
    return persistent_blocks_per_sm((const void*)stage2d_batch_kernel<R, Ph, kBatchNT>, kBatchNT, smem, bps);
  });
}

template <class R>
cudaError_t launch_stage2d_batch(const mxm_dg_physics_desc& pd, const Batch2DArgs<R>& ba, int grid, size_t smem,
                                 cudaStream_t st) {
  return with_phys2d<R>(pd, [&](const auto& ph) -> cudaError_t {
    using Ph = typename std::decay<decltype(ph)>::type;
    stage2d_batch_kernel<R, Ph, kBatchNT><<<grid, kBatchNT, smem, st>>>(ba, ph);
    return cudaGetLastError();
  });
}

template <class R, int NC>
cudaError_t lim2d_batch_attr() {
  return cudaFuncSetAttribute(theta_batch_kernel<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(lim2d_smem_bytes<R, ntri(5), NC>()));
}

// Kernel attributes of the batched limiter (call before any stream capture).
template <class R>
cudaError_t prepare_lim2d_batch(int NC) {
  switch (NC) {
    case 1: return lim2d_batch_attr<R, 1>();
    case 3: return lim2d_batch_attr<R, 3>();
    case 4: return lim2d_batch_attr<R, 4>();
    case 6: return lim2d_batch_attr<R, 6>();
    case 7: return lim2d_batch_attr<R, 7>();
  }
  return cudaErrorInvalidValue;
}

template <class R, int NC>
cudaError_t lim2d_batch_nc(const LimBatch2DArgs<R>& la, cudaStream_t st) {
  constexpr size_t smem = lim2d_smem_bytes<R, ntri(5), NC>();
  avg_batch_kernel<R, NC><<<la.nitems, 256, 0, st>>>(la);
  theta_batch_kernel<R, NC><<<la.nitems, kLim2dBlock, smem, st>>>(la);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_lim2d_batch(int NC, const LimBatch2DArgs<R>& la, cudaStream_t st) {
  if (la.nitems <= 0) return cudaSuccess;
  switch (NC) {
    case 1: return lim2d_batch_nc<R, 1>(la, st);
    case 3: return lim2d_batch_nc<R, 3>(la, st);
    case 4: return lim2d_batch_nc<R, 4>(la, st);
    case 6: return lim2d_batch_nc<R, 6>(la, st);
    case 7: return lim2d_batch_nc<R, 7>(la, st);
  }
  return cudaErrorInvalidValue;
}

#define MXM_INSTANTIATE_BATCH2D(R)                                                                                  \
  template cudaError_t stage2d_batch_blocks_per_sm<R>(const mxm_dg_physics_desc&, size_t, int*);                   \
  template cudaError_t launch_stage2d_batch<R>(const mxm_dg_physics_desc&, const Batch2DArgs<R>&, int, size_t,     \
                                               cudaStream_t);                                                       \
  template cudaError_t launch_lim2d_batch<R>(int, const LimBatch2DArgs<R>&, cudaStream_t);                       \
  template cudaError_t prepare_lim2d_batch<R>(int);

}  // namespace mxm
