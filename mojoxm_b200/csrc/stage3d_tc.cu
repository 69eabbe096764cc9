// Launch + explicit instantiation of the tensor-core (split-BF16) 3D stage
// kernel for P = 2..5; P = 1 uses the FP32 SIMT kernel.
#include "stage3d_tc.cuh"

namespace mxm {

template <class Phys, int P>
cudaError_t launch_tc_p(const Stage3DArgs<float>& a, const KuhnTab3<float>& tab, const Phys& ph,
                        const unsigned char* img, int nsm, cudaStream_t st) {
  using S = TcShape<P, Phys::NC>;
  constexpr int NT = 256;
  auto kern = stage3d_tc_kernel<Phys, P, NT>;
  static int bps = -1;
  if (bps < 0) {
    cudaError_t e = persistent_blocks_per_sm((const void*)kern, NT, S::SMEM, &bps);
    if (e != cudaSuccess) return e;
  }
  const int ngroups = (a.ncell - a.cbeg + S::EC - 1) / S::EC;
  int nblk = nsm * bps;
  if (nblk > ngroups) nblk = ngroups;
  if (nblk < 1) nblk = 1;
  kern<<<nblk, NT, S::SMEM, st>>>(a, tab, ph, img);
  return cudaGetLastError();
}

template <class Phys>
cudaError_t launch_stage3d_tc(int P, const Stage3DArgs<float>& a, const KuhnTab3<float>& tab, const Phys& ph,
                              const unsigned char* img, int nsm, cudaStream_t st) {
  switch (P) {
    case 2: return launch_tc_p<Phys, 2>(a, tab, ph, img, nsm, st);
    case 3: return launch_tc_p<Phys, 3>(a, tab, ph, img, nsm, st);
    case 4: return launch_tc_p<Phys, 4>(a, tab, ph, img, nsm, st);
    case 5: return launch_tc_p<Phys, 5>(a, tab, ph, img, nsm, st);
  }
  return cudaErrorInvalidValue;
}

using TA = AdvectionD<float>;
using TER = EulerD<float, FLUX_RUSANOV>;
using TEO = EulerD<float, FLUX_ROE>;
using TEE = EulerD<float, FLUX_HLLE>;
using TEC = EulerD<float, FLUX_HLLEC>;
using TM = MaxwellD<float>;
using TS = ShallowWaterD<float>;
using TH = MhdD<float>;
#define MXM_INST_TC(PH)                                                                                           \
  template cudaError_t launch_stage3d_tc<PH>(int, const Stage3DArgs<float>&, const KuhnTab3<float>&, const PH&, \
                                             const unsigned char*, int, cudaStream_t);
MXM_INST_TC(TA)
MXM_INST_TC(TER)
MXM_INST_TC(TEO)
MXM_INST_TC(TEE)
MXM_INST_TC(TEC)
MXM_INST_TC(TM)
MXM_INST_TC(TS)
MXM_INST_TC(TH)

}  // namespace mxm
