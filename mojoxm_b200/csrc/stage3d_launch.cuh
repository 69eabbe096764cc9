// Launch configuration of the 3D stage kernel per (real type, P, NC).
#pragma once
#include "stage3d.cuh"

namespace mxm {

// Largest divisor of NP not above `base` whose RI x NC accumulator tile
// stays within `cap` registers' worth of values (at least 1).
constexpr int ri_capped(int base, int NP, int NC, int cap) {
  for (int r = base; r > 1; --r)
    if (NP % r == 0 && r * NC <= cap) return r;
  return 1;
}

// K-split width of the contraction: the largest power of two (at most 16)
// that keeps every work of a tile within one pass of the block and at least
// 8 K columns per lane.
constexpr int ks_pick(int works, int nt, int K) {
  int ks = 1;
  while (ks < 16 && works * ks * 2 <= nt && K / (ks * 2) >= 8) ks *= 2;
  return ks;
}

template <class R, int P, int NC>
struct Cfg3 {
  using S = Stage3DShape<P, NC, R>;
  static constexpr int NP = S::NP;
  // rows per thread: a divisor of NP (fewer for wide states)
  static constexpr int RI0 = sizeof(R) == 8 ? (P <= 3 ? 2 : (P == 4 ? 5 : 4))
                                            : (P == 1 ? 4 : (P == 2 ? 5 : (P == 3 ? 4 : (P == 4 ? 5 : 8))));
  static constexpr int RI = NC > 6 ? ri_capped(RI0, NP, NC, sizeof(R) == 8 ? 48 : 64) : RI0;
  // keep the shared operator in shared memory when it takes <= 64 KB and a
  // one-cube tile still fits beside it
  static constexpr bool ASMEM = sizeof(R) * S::K * S::NP <= 64 * 1024 &&
                                stage3d_smem(P, NC, int(sizeof(R)), 1, true) <= kMaxSmemPerBlock;
  static constexpr size_t kBudget = 110 * 1024;  // two blocks per SM
  static constexpr size_t kFixed = 16 + (sizeof(KuhnTab3<R>) + 15) / 16 * 16 + (ASMEM ? sizeof(R) * S::K * S::NP : 0);
  static constexpr size_t kPerCube = 6 * sizeof(R) * (2 * size_t(S::NP) * NC + S::BSTR);
  static constexpr int EC_RAW = kBudget > kFixed ? int((kBudget - kFixed) / kPerCube) : 1;
  static constexpr int EC = EC_RAW > 16 ? 16 : (EC_RAW < 1 ? 1 : EC_RAW);
  static constexpr int NT = 256;
  // split K only where a tile's works leave most of the block idle: with
  // 120 of 256 threads busy (FP64 P3) a 2-way split measured -4 %, with 126
  // (FP32 P4) +9 %, with 42 (FP64 P4) +69 %
  static constexpr int WORKS = 6 * EC * (S::NP / RI);
  static constexpr int KS = (sizeof(R) == 8 ? WORKS * 8 < 3 * NT : WORKS * 2 <= NT) ? ks_pick(WORKS, NT, S::K) : 1;
  static constexpr size_t kSmem = stage3d_smem_bytes<R, P, NC, EC, ASMEM>();
  static constexpr bool FITS = kSmem <= kMaxSmemPerBlock;
};

template <class R, class Phys, int P>
cudaError_t launch3_p(const Stage3DArgs<R>& a, const KuhnTab3<R>& tab, const Phys& ph, int nsm, cudaStream_t st) {
  using C = Cfg3<R, P, Phys::NC>;
  if constexpr (!C::FITS) {
    return cudaErrorInvalidConfiguration;  // refused at mxm_dg_create already
  } else {
  auto kern = stage3d_kernel<R, Phys, P, C::EC, C::RI, C::KS, C::NT, C::ASMEM>;
  static int bps = -1;
  if (bps < 0) {
    cudaError_t e = persistent_blocks_per_sm((const void*)kern, C::NT, C::kSmem, &bps);
    if (e != cudaSuccess) return e;
  }
  const int ngroups = (a.ncell - a.cbeg + C::EC - 1) / C::EC;
  int nblk = nsm * bps;
  if (nblk > ngroups) nblk = ngroups;
  if (nblk < 1) nblk = 1;
  return launch_dependent(kern, nblk, C::NT, C::kSmem, st, a, tab, ph);
  }
}

template <class R, class Phys>
cudaError_t launch_stage3d(int P, const Stage3DArgs<R>& a, const KuhnTab3<R>& tab, const Phys& ph, int nsm,
                           cudaStream_t st) {
  switch (P) {
    case 1: return launch3_p<R, Phys, 1>(a, tab, ph, nsm, st);
    case 2: return launch3_p<R, Phys, 2>(a, tab, ph, nsm, st);
    case 3: return launch3_p<R, Phys, 3>(a, tab, ph, nsm, st);
    case 4: return launch3_p<R, Phys, 4>(a, tab, ph, nsm, st);
    case 5: return launch3_p<R, Phys, 5>(a, tab, ph, nsm, st);
  }
  return cudaErrorInvalidValue;
}

template <class R, class Phys>
cudaError_t launch_wavespeed3d(int P, const Stage3DArgs<R>& a, const KuhnTab3<R>& tab, const Phys& ph,
                               unsigned long long* out, cudaStream_t st) {
  const int64_t n = int64_t(a.ncell - a.cbeg) * 6 * 4 * ntri(P);
  const int nb = int((n + 255) / 256);
  switch (P) {
    case 1: wavespeed3d_kernel<R, Phys, 1><<<nb, 256, 0, st>>>(a, tab, ph, out); break;
    case 2: wavespeed3d_kernel<R, Phys, 2><<<nb, 256, 0, st>>>(a, tab, ph, out); break;
    case 3: wavespeed3d_kernel<R, Phys, 3><<<nb, 256, 0, st>>>(a, tab, ph, out); break;
    case 4: wavespeed3d_kernel<R, Phys, 4><<<nb, 256, 0, st>>>(a, tab, ph, out); break;
    case 5: wavespeed3d_kernel<R, Phys, 5><<<nb, 256, 0, st>>>(a, tab, ph, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

#define MXM_INSTANTIATE_STAGE3D(R, PHYS)                                                                          \
  template cudaError_t launch_stage3d<R, PHYS>(int, const Stage3DArgs<R>&, const KuhnTab3<R>&, const PHYS&, int, \
                                               cudaStream_t);                                                     \
  template cudaError_t launch_wavespeed3d<R, PHYS>(int, const Stage3DArgs<R>&, const KuhnTab3<R>&, const PHYS&,  \
                                                   unsigned long long*, cudaStream_t);

}  // namespace mxm
