// Fused 2D SSPRK3 stage kernel on a Kuhn triangle mesh (sm_100a).
//
// Replaces the reference's two launches per stage -- *_face_flux_kernel_2d
// (one thread per (face, slot) writing fstar to global memory) and
// *_vol_lift_combine_rk_kernel_2d (src/local_mesh_2d_gpu_euler.mojo:33-144
// and siblings) -- with one kernel: a block owns one triangle type (2 per
// cell), stages the fused operator A_t = [D_x | D_y | -Lift_t] once, and per
// element evaluates volume fluxes and its 3 edges' numerical fluxes into a
// shared B tile, then rhs = A_t B + source and the RK combine.  Face traces
// never touch global memory; connectivity is implicit in (cell, type).
#pragma once
#include "dg_common.cuh"
#include "physics2d.cuh"

namespace mxm {

template <int P, int NC, class R>
struct Stage2DShape {
  static constexpr int NP = ntri(P), NFP = P + 1, K = 2 * NP + 3 * NFP;
  static constexpr int BSTR_RAW = K * NC;
  static constexpr int BMOD = sizeof(R) == 8 ? 16 : 32;
  static constexpr int BSTR = BSTR_RAW + ((1 - BSTR_RAW % BMOD) + BMOD) % BMOD;
};

template <class R, class Phys, int P, int RI, int EB, int NT>
__global__ void __launch_bounds__(NT) stage2d_kernel(Stage2DArgs<R> args, KuhnTab2<R> tab, Phys ph) {
  constexpr int NC = Phys::NC;
  using S = Stage2DShape<P, NC, R>;
  constexpr int NP = S::NP, NFP = S::NFP, K = S::K, BSTR = S::BSTR;
  constexpr int G = NP / RI;
  static_assert(NP % RI == 0, "row tile must divide NP");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sA = reinterpret_cast<R*>(smem_raw);  // [K][NP]
  R* sQ = sA + K * NP;                     // [EB][NP][NC]
  R* sB = sQ + EB * NP * NC;               // [EB][BSTR]
  const int tid = threadIdx.x;
  const int t = blockIdx.x & 1;
  const int nblk_t = gridDim.x >> 1;
  const int ngroups = (args.ncell + EB - 1) / EB;
  const R* gA = args.A + size_t(t) * K * NP;
  for (int idx = tid; idx < NP * K; idx += NT) sA[idx] = gA[idx];

  for (int grp = blockIdx.x >> 1; grp < ngroups; grp += nblk_t) {
    const int cell0 = grp * EB;
    const int nhere = min(EB, args.ncell - cell0);
    __syncthreads();
    for (int idx = tid; idx < EB * NP * NC; idx += NT) {
      const int el = idx / (NP * NC), r = idx - el * NP * NC;
      if (el < nhere) sQ[idx] = args.q_in[(size_t(cell0 + el) * 2 + t) * (NP * NC) + r];
    }
    __syncthreads();
    for (int idx = tid; idx < EB * NP; idx += NT) {
      const int el = idx / NP, j = idx - el * NP;
      if (el >= nhere) continue;
      R Fx[NC], Fy[NC];
      ph.flux(&sQ[(el * NP + j) * NC], Fx, Fy);
      R* b = &sB[el * BSTR];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        b[j * NC + c] = Fx[c];
        b[(NP + j) * NC + c] = Fy[c];
      }
    }
    for (int idx = tid; idx < EB * 3 * NFP; idx += NT) {
      const int el = idx / (3 * NFP), fm = idx - el * 3 * NFP;
      if (el >= nhere) continue;
      const int lf = fm / NFP, m = fm - lf * NFP;
      const int cell = cell0 + el;
      const int cj = cell / args.nx, ci = cell - cj * args.nx;
      const int ax = tab.axis[t][lf], dir = tab.dir[t][lf];
      const int cpos = ax == 0 ? ci : cj;
      const int nax = ax == 0 ? args.nx : args.ny;
      int code;
      const int mode = face_mode(ax, dir, cpos, nax, args.bc, code);
      const R* qo = &sQ[(el * NP + tab.own_node[lf][m]) * NC];
      const R nx = tab.normal[t][lf][0], ny = tab.normal[t][lf][1];
      R f[NC];
      if (mode == FACE_BC_HI) {
        ph.face(qo, qo, code, nx, ny, f);
      } else if (mode == FACE_BC_LO) {
        ph.face(qo, qo, code, -nx, -ny, f);
#pragma unroll
        for (int c = 0; c < NC; ++c) f[c] = -f[c];
      } else {
        const int ni = wrapi(ci + tab.off[t][lf][0], args.nx), nj = wrapi(cj + tab.off[t][lf][1], args.ny);
        const size_t enb = (size_t(nj) * args.nx + ni) * 2 + tab.nb_t[t][lf];
        const R* gq = args.q_in + (enb * NP + tab.nb_node[t][lf][m]) * NC;
        R qn[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) qn[c] = gq[c];
        if (mode == FACE_MIXED) ph.face(qn, qn, code, nx, ny, f);
        else if (tab.side[t][lf] == 0) ph.face(qo, qn, BC_INTERIOR, nx, ny, f);
        else ph.face(qn, qo, BC_INTERIOR, nx, ny, f);
      }
      R* b = &sB[el * BSTR + (2 * NP + fm) * NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) b[c] = f[c];
    }
    __syncthreads();
    for (int w = tid; w < EB * G; w += NT) {
      const int el = w / G, g = w - el * G;
      if (el >= nhere) continue;
      const int i0 = g * RI;
      R acc[RI][NC];
#pragma unroll
      for (int r = 0; r < RI; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[r][c] = R(0);
      const R* b = &sB[el * BSTR];
#pragma unroll 4
      for (int k = 0; k < K; ++k) {
        R av[RI], bv[NC];
#pragma unroll
        for (int r = 0; r < RI; ++r) av[r] = sA[k * NP + i0 + r];
#pragma unroll
        for (int c = 0; c < NC; ++c) bv[c] = b[k * NC + c];
#pragma unroll
        for (int r = 0; r < RI; ++r)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
      }
      const size_t e = size_t(cell0 + el) * 2 + t;
#pragma unroll
      for (int r = 0; r < RI; ++r) {
        const int i = i0 + r;
        const size_t base = (e * NP + i) * NC;
        R src[NC];
        if (Phys::kSource) ph.source(&sQ[(el * NP + i) * NC], src);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const R rhs = Phys::kSource ? acc[r][c] + src[c] : acc[r][c];
          args.q_out[base + c] =
              args.rhs_only ? rhs : args.a * args.q_a[base + c] + args.b * args.q_b[base + c] + args.cdt * rhs;
        }
      }
    }
  }
}

template <class R, int P, int NC>
struct Cfg2 {
  using S = Stage2DShape<P, NC, R>;
  static constexpr int NP = S::NP;
  static constexpr int RI = P == 1 ? 3 : (P == 2 ? 2 : (P == 3 ? 5 : (P == 4 ? 5 : 3)));  // divisors of 3,6,10,15,21
  static constexpr size_t kA = sizeof(R) * S::K * S::NP;
  static constexpr size_t kPerEl = sizeof(R) * (size_t(S::NP) * NC + S::BSTR);
  static constexpr int EB_RAW = int((96 * 1024 - kA) / kPerEl);
  static constexpr int EB = EB_RAW > 128 ? 128 : (EB_RAW < 1 ? 1 : EB_RAW);
  static constexpr int NT = 128;
  static constexpr size_t kSmem = kA + sizeof(R) * (size_t(EB) * S::NP * NC + size_t(EB) * S::BSTR);
};

template <class R, class Phys, int P>
cudaError_t launch2_p(const Stage2DArgs<R>& a, const KuhnTab2<R>& tab, const Phys& ph, int nsm, cudaStream_t st) {
  using C = Cfg2<R, P, Phys::NC>;
  auto kern = stage2d_kernel<R, Phys, P, C::RI, C::EB, C::NT>;
  static int bps = -1;
  if (bps < 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::kSmem));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, C::NT, C::kSmem);
    if (e != cudaSuccess) return e;
    if (bps < 1) bps = 1;
  }
  const int ngroups = (a.ncell + C::EB - 1) / C::EB;
  int per_type = (nsm * bps + 1) / 2;
  if (per_type > ngroups) per_type = ngroups;
  if (per_type < 1) per_type = 1;
  kern<<<2 * per_type, C::NT, C::kSmem, st>>>(a, tab, ph);
  return cudaGetLastError();
}

template <class R, class Phys>
cudaError_t launch_stage2d(int P, const Stage2DArgs<R>& a, const KuhnTab2<R>& tab, const Phys& ph, int nsm,
                           cudaStream_t st) {
  switch (P) {
    case 1: return launch2_p<R, Phys, 1>(a, tab, ph, nsm, st);
    case 2: return launch2_p<R, Phys, 2>(a, tab, ph, nsm, st);
    case 3: return launch2_p<R, Phys, 3>(a, tab, ph, nsm, st);
    case 4: return launch2_p<R, Phys, 4>(a, tab, ph, nsm, st);
    case 5: return launch2_p<R, Phys, 5>(a, tab, ph, nsm, st);
  }
  return cudaErrorInvalidValue;
}

// Nodal max of the physical signal speed (2D kernels return no face speed).
template <class R, class Phys, int NC>
__global__ void wavespeed2d_kernel(const R* q, int64_t nnodes, Phys ph, unsigned long long* out) {
  const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double best = 0.0;
  if (n < nnodes) {
    best = double(ph.speed(q + n * NC));
    if (!(best >= 0.0)) best = __longlong_as_double(0x7ff0000000000000LL);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

template <class R, class Phys>
cudaError_t launch_wavespeed2d(const R* q, int64_t nnodes, const Phys& ph, unsigned long long* out, cudaStream_t st) {
  wavespeed2d_kernel<R, Phys, Phys::NC><<<int((nnodes + 255) / 256), 256, 0, st>>>(q, nnodes, ph, out);
  return cudaGetLastError();
}

#define MXM_INSTANTIATE_STAGE2D(R, PHYS)                                                                          \
  template cudaError_t launch_stage2d<R, PHYS>(int, const Stage2DArgs<R>&, const KuhnTab2<R>&, const PHYS&, int, \
                                               cudaStream_t);                                                     \
  template cudaError_t launch_wavespeed2d<R, PHYS>(const R*, int64_t, const PHYS&, unsigned long long*, cudaStream_t);

}  // namespace mxm
