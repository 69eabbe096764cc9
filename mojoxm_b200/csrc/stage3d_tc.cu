// Launch + explicit instantiation of the tensor-core 3D stage kernel
// (split-BF16 or split-TF32 operands) for P = 2..5 where the shape fits
// shared memory; P = 1 uses the FP32 SIMT kernel.
#include <type_traits>

#include "stage3d_tc.cuh"

namespace mxm {

// Threads per block and resident blocks per SM of one instantiation.
// 256 threads per block; a shape that fits one block per SM (the split-TF32
// P4 tiles, split-BF16 P5) takes 512 so that the SM still holds 16 warps.
// Batched launches keep the current solve's arguments behind the tile's
// shared memory.
template <class Phys, int P, class Op, bool BATCH>
struct TcLaunch {
  using S = TcShape<P, Phys::NC, Op>;
  static constexpr int NT = S::blocks_for(S::SMEM) == 1 ? 512 : 256;
  static constexpr size_t smem = BATCH ? S::BATCH_SMEM : S::SMEM;
  static cudaError_t blocks_per_sm(int* out) {
    static int bps = -1;
    if (bps < 0) {
      cudaError_t e = persistent_blocks_per_sm((const void*)stage3d_tc_kernel<Phys, P, NT, Op, BATCH>, NT, smem, &bps);
      if (e != cudaSuccess) return e;
    }
    *out = bps;
    return cudaSuccess;
  }
  // persistent grid: every resident block, at most one per tile
  static cudaError_t grid(int nsm, int ntiles, int* out) {
    int bps = 0;
    cudaError_t e = blocks_per_sm(&bps);
    if (e != cudaSuccess) return e;
    int nblk = nsm * bps;
    if (nblk > ntiles) nblk = ntiles;
    *out = nblk < 1 ? 1 : nblk;
    return cudaSuccess;
  }
};

template <class Phys, int P, class Op, bool BATCH>
cudaError_t launch_tc_p(const Stage3DArgs<float>& a, const Tc3Batch& bat, const KuhnTab3<float>& tab, const Phys& ph,
                        const unsigned char* img, int nsm, cudaStream_t st) {
  using S = TcShape<P, Phys::NC, Op>;
  if constexpr (!S::FITS) {
    return cudaErrorInvalidValue;  // the create call refuses these shapes
  } else {
    using L = TcLaunch<Phys, P, Op, BATCH>;
    static_assert(sizeof(Stage3DArgs<float>) <= 256, "batched arguments slot");
    const int ntiles = BATCH ? bat.nitems : (a.ncell - a.cbeg + S::EC - 1) / S::EC;
    if (ntiles <= 0) return cudaSuccess;
    int nblk = 1;
    cudaError_t e = L::grid(nsm, ntiles, &nblk);
    if (e != cudaSuccess) return e;
    auto kern = stage3d_tc_kernel<Phys, P, L::NT, Op, BATCH>;
    if constexpr (BATCH) {
      kern<<<nblk, L::NT, L::smem, st>>>(a, tab, ph, img, bat);
      return cudaGetLastError();
    } else {
      return launch_dependent(kern, nblk, L::NT, L::smem, st, a, tab, ph, img, bat);
    }
  }
}

template <class Phys, class Op>
cudaError_t batch_grid_kind(int P, int nsm, int ntiles, int* out) {
  auto one = [&](auto pc) -> cudaError_t {
    constexpr int PP = decltype(pc)::value;
    if constexpr (!TcShape<PP, Phys::NC, Op>::FITS) return cudaErrorInvalidValue;
    else return TcLaunch<Phys, PP, Op, true>::grid(nsm, ntiles, out);
  };
  switch (P) {
    case 2: return one(std::integral_constant<int, 2>{});
    case 3: return one(std::integral_constant<int, 3>{});
    case 4: return one(std::integral_constant<int, 4>{});
    case 5: return one(std::integral_constant<int, 5>{});
  }
  return cudaErrorInvalidValue;
}

// Blocks a batched launch of `ntiles` tiles runs (the same rule as the launch).
template <class Phys>
cudaError_t stage3d_tc_batch_grid(int P, int kind, const Phys&, int nsm, int ntiles, int* out) {
  return kind == TC_TF32 ? batch_grid_kind<Phys, OpTF32>(P, nsm, ntiles, out)
                         : batch_grid_kind<Phys, OpBF16>(P, nsm, ntiles, out);
}

template <class Phys, class Op, bool BATCH>
cudaError_t launch_tc_kind(int P, const Stage3DArgs<float>& a, const Tc3Batch& bat, const KuhnTab3<float>& tab,
                           const Phys& ph, const unsigned char* img, int nsm, cudaStream_t st) {
  switch (P) {
    case 2: return launch_tc_p<Phys, 2, Op, BATCH>(a, bat, tab, ph, img, nsm, st);
    case 3: return launch_tc_p<Phys, 3, Op, BATCH>(a, bat, tab, ph, img, nsm, st);
    case 4: return launch_tc_p<Phys, 4, Op, BATCH>(a, bat, tab, ph, img, nsm, st);
    case 5: return launch_tc_p<Phys, 5, Op, BATCH>(a, bat, tab, ph, img, nsm, st);
  }
  return cudaErrorInvalidValue;
}

template <class Phys>
cudaError_t launch_stage3d_tc(int P, int kind, const Stage3DArgs<float>& a, const KuhnTab3<float>& tab,
                              const Phys& ph, const unsigned char* img, int nsm, cudaStream_t st) {
  const Tc3Batch none{nullptr, nullptr, nullptr, 0};
  return kind == TC_TF32 ? launch_tc_kind<Phys, OpTF32, false>(P, a, none, tab, ph, img, nsm, st)
                         : launch_tc_kind<Phys, OpBF16, false>(P, a, none, tab, ph, img, nsm, st);
}

template <class Phys>
cudaError_t launch_stage3d_tc_batch(int P, int kind, const Tc3Batch& bat, const Phys& ph, const unsigned char* img,
                                    int nsm, cudaStream_t st) {
  static const Stage3DArgs<float> a0{};
  static const KuhnTab3<float> t0{};
  return kind == TC_TF32 ? launch_tc_kind<Phys, OpTF32, true>(P, a0, bat, t0, ph, img, nsm, st)
                         : launch_tc_kind<Phys, OpBF16, true>(P, a0, bat, t0, ph, img, nsm, st);
}

int tc_tile_cubes(int P, int NC, int kind) {
  auto ec = [&](auto op) -> int {
    using O = decltype(op);
    switch (NC) {
      case 1: return P == 2 ? TcShape<2, 1, O>::EC : P == 3 ? TcShape<3, 1, O>::EC : P == 4 ? TcShape<4, 1, O>::EC : TcShape<5, 1, O>::EC;
      case 3: return P == 2 ? TcShape<2, 3, O>::EC : P == 3 ? TcShape<3, 3, O>::EC : P == 4 ? TcShape<4, 3, O>::EC : TcShape<5, 3, O>::EC;
      case 5: return P == 2 ? TcShape<2, 5, O>::EC : P == 3 ? TcShape<3, 5, O>::EC : P == 4 ? TcShape<4, 5, O>::EC : TcShape<5, 5, O>::EC;
      case 6: return P == 2 ? TcShape<2, 6, O>::EC : P == 3 ? TcShape<3, 6, O>::EC : P == 4 ? TcShape<4, 6, O>::EC : TcShape<5, 6, O>::EC;
      case 9: return P == 2 ? TcShape<2, 9, O>::EC : P == 3 ? TcShape<3, 9, O>::EC : P == 4 ? TcShape<4, 9, O>::EC : TcShape<5, 9, O>::EC;
    }
    return 0;
  };
  return kind == TC_TF32 ? ec(OpTF32{}) : ec(OpBF16{});
}

bool tc_shape_fits(int P, int NC, int kind) {
  auto fits = [&](auto op) -> bool {
    using O = decltype(op);
    switch (NC) {
      case 1: return P == 2 ? TcShape<2, 1, O>::FITS : P == 3 ? TcShape<3, 1, O>::FITS : P == 4 ? TcShape<4, 1, O>::FITS : TcShape<5, 1, O>::FITS;
      case 3: return P == 2 ? TcShape<2, 3, O>::FITS : P == 3 ? TcShape<3, 3, O>::FITS : P == 4 ? TcShape<4, 3, O>::FITS : TcShape<5, 3, O>::FITS;
      case 5: return P == 2 ? TcShape<2, 5, O>::FITS : P == 3 ? TcShape<3, 5, O>::FITS : P == 4 ? TcShape<4, 5, O>::FITS : TcShape<5, 5, O>::FITS;
      case 6: return P == 2 ? TcShape<2, 6, O>::FITS : P == 3 ? TcShape<3, 6, O>::FITS : P == 4 ? TcShape<4, 6, O>::FITS : TcShape<5, 6, O>::FITS;
      case 9: return P == 2 ? TcShape<2, 9, O>::FITS : P == 3 ? TcShape<3, 9, O>::FITS : P == 4 ? TcShape<4, 9, O>::FITS : TcShape<5, 9, O>::FITS;
    }
    return false;
  };
  if (P < 2 || P > 5) return false;
  return kind == TC_TF32 ? fits(OpTF32{}) : fits(OpBF16{});
}

using TA = AdvectionD<float>;
using TER = EulerD<float, FLUX_RUSANOV>;
using TEO = EulerD<float, FLUX_ROE>;
using TEE = EulerD<float, FLUX_HLLE>;
using TEC = EulerD<float, FLUX_HLLEC>;
using TM = MaxwellD<float>;
using TS = ShallowWaterD<float>;
using TH = MhdD<float>;
#define MXM_INST_TC(PH)                                                                                      \
  template cudaError_t launch_stage3d_tc<PH>(int, int, const Stage3DArgs<float>&, const KuhnTab3<float>&,    \
                                             const PH&, const unsigned char*, int, cudaStream_t);            \
  template cudaError_t launch_stage3d_tc_batch<PH>(int, int, const Tc3Batch&, const PH&, const unsigned char*, \
                                                   int, cudaStream_t);                                         \
  template cudaError_t stage3d_tc_batch_grid<PH>(int, int, const PH&, int, int, int*);
MXM_INST_TC(TA)
MXM_INST_TC(TER)
MXM_INST_TC(TEO)
MXM_INST_TC(TEE)
MXM_INST_TC(TEC)
MXM_INST_TC(TM)
MXM_INST_TC(TS)
MXM_INST_TC(TH)

}  // namespace mxm
