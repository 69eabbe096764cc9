// Fused 3D SSPRK3 stage kernel on a Kuhn tetrahedral mesh (sm_100a).
//
// Replaces mojoxm's rk_stage_kernel (src/solver.mojo:161-337): per element,
// pointwise physical flux, face-trace gather + numerical/boundary flux,
// volume contraction sum_j sum_k D_k[i,j] (invJ F_j)_k, lift
// sum_f sign*area*Lift*f*, source, RK combine a*q_a + b*q_b + c*dt*rhs and
// the positivity floor.
//
// B200 design:
//  * A block owns one tet type t (6 per cube) and walks groups of EB cubes,
//    so it stages ONE fused operator A_t = [D_x|D_y|D_z|-Lift_t] (physical
//    derivatives with invJ folded in, lift pre-scaled by side*area/(6V)) in
//    shared memory once, and every element's RHS is a small GEMM
//    rhs[i][c] = sum_k A_t[i][k] B[k][c] with B = [F_x; F_y; F_z; f*].
//  * Connectivity is not read from memory: neighbour element and node of
//    every face node follow from (cube, type) and a 1.7 KB table in the
//    constant bank (Kuhn meshes are translation invariant); only q moves.
//  * Element state is staged in shared memory with contiguous loads; the RK
//    combine reads q_a/q_b and writes q_out per node (NC contiguous values).
#pragma once
#include "dg_common.cuh"
#include "physics.cuh"

namespace mxm {

template <int P, int NC, class R>
struct Stage3DShape {
  static constexpr int NP = ntet(P), NFP = ntri(P), K = 3 * NP + 4 * NFP;
  // element stride of the B tile, padded so that up to 16 (FP64) / 32 (FP32)
  // elements read in the same warp land in distinct banks
  static constexpr int BSTR_RAW = K * NC;
  static constexpr int BMOD = sizeof(R) == 8 ? 16 : 32;
  static constexpr int BSTR = BSTR_RAW + ((1 - BSTR_RAW % BMOD) + BMOD) % BMOD;
};

template <class R, class Phys, int P, int RI, int EB, int NT, bool ASMEM>
__global__ void __launch_bounds__(NT) stage3d_kernel(Stage3DArgs<R> args, KuhnTab3<R> tab, Phys ph) {
  constexpr int NC = Phys::NC;
  using S = Stage3DShape<P, NC, R>;
  constexpr int NP = S::NP, NFP = S::NFP, K = S::K, BSTR = S::BSTR;
  constexpr int G = NP / RI;
  static_assert(NP % RI == 0, "row tile must divide NP");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sAbuf = reinterpret_cast<R*>(smem_raw);  // [K][NP] when staged
  R* sQ = sAbuf + (ASMEM ? K * NP : 0);          // [EB][NP][NC]
  R* sB = sQ + EB * NP * NC;               // [EB][BSTR]

  const int tid = threadIdx.x;
  const int t = blockIdx.x % 6;
  const int nblk_t = gridDim.x / 6;
  const int ngroups = (args.ncell + EB - 1) / EB;

  // Stage A_t (k-major) once per block, or read it through L1 when it
  // does not fit next to the element tiles.
  const R* gA = args.A + size_t(t) * K * NP;
  if (ASMEM)
    for (int idx = tid; idx < NP * K; idx += NT) sAbuf[idx] = gA[idx];
  const R* sA = ASMEM ? sAbuf : gA;

  const int nxy = args.nx * args.ny;
  for (int grp = blockIdx.x / 6; grp < ngroups; grp += nblk_t) {
    const int cell0 = grp * EB;
    const int ncell_here = min(EB, args.ncell - cell0);
    __syncthreads();  // previous group done with sQ / sB (and sA staged)
    // ---- stage q_in of the EB elements of type t
    for (int idx = tid; idx < EB * NP * NC; idx += NT) {
      const int el = idx / (NP * NC), r = idx - el * NP * NC;
      if (el < ncell_here) sQ[idx] = args.q_in[(size_t(cell0 + el) * 6 + t) * (NP * NC) + r];
    }
    __syncthreads();
    // ---- volume fluxes F_j -> B rows d*NP + j
    for (int idx = tid; idx < EB * NP; idx += NT) {
      const int el = idx / NP, j = idx - el * NP;
      if (el >= ncell_here) continue;
      R F[3 * NC];
      ph.flux(&sQ[(el * NP + j) * NC], F);
      R* b = &sB[el * BSTR];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int c = 0; c < NC; ++c) b[(d * NP + j) * NC + c] = F[d * NC + c];
    }
    // ---- face numerical fluxes -> B rows 3NP + lf*NFP + m
    for (int idx = tid; idx < EB * 4 * NFP; idx += NT) {
      const int el = idx / (4 * NFP), fm = idx - el * 4 * NFP;
      if (el >= ncell_here) continue;
      const int lf = fm / NFP, m = fm - lf * NFP;
      const int cell = cell0 + el;
      const int ck = cell / nxy, rem = cell - ck * nxy, cj = rem / args.nx, ci = rem - cj * args.nx;
      const int ax = tab.axis[t][lf], dir = tab.dir[t][lf];
      const int cpos = ax == 0 ? ci : (ax == 1 ? cj : ck);
      const int nax = ax == 0 ? args.nx : (ax == 1 ? args.ny : args.nz);
      int code;
      const int mode = face_mode(ax, dir, cpos, nax, args.bc, code);
      const R* qo = &sQ[(el * NP + tab.own_node[lf][m]) * NC];
      R nx = tab.normal[t][lf][0], ny = tab.normal[t][lf][1], nz = tab.normal[t][lf][2];
      R f[NC];
      if (mode == FACE_BC_HI) {
        ph.bnd_flux(qo, code, nx, ny, nz, f);
      } else if (mode == FACE_BC_LO) {
        ph.bnd_flux(qo, code, -nx, -ny, -nz, f);
#pragma unroll
        for (int c = 0; c < NC; ++c) f[c] = -f[c];  // one-sided face: element on side 0
      } else {
        const int ni = wrapi(ci + tab.off[t][lf][0], args.nx), nj = wrapi(cj + tab.off[t][lf][1], args.ny),
                  nk = wrapi(ck + tab.off[t][lf][2], args.nz);
        const size_t enb = (size_t(ni) + size_t(args.nx) * (nj + size_t(args.ny) * nk)) * 6 + tab.nb_t[t][lf];
        const R* gq = args.q_in + (enb * NP + tab.nb_node[t][lf][m]) * NC;
        R qn[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) qn[c] = gq[c];
        if (mode == FACE_MIXED) ph.bnd_flux(qn, code, nx, ny, nz, f);
        else if (tab.side[t][lf] == 0) ph.num_flux(qo, qn, nx, ny, nz, f);
        else ph.num_flux(qn, qo, nx, ny, nz, f);
      }
      R* b = &sB[el * BSTR + (3 * NP + fm) * NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) b[c] = f[c];
    }
    __syncthreads();
    // ---- contraction rhs = A_t B, source, RK combine, floor, store
    for (int w = tid; w < EB * G; w += NT) {
      const int el = w / G, g = w - el * G;
      if (el >= ncell_here) continue;
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
        for (int r = 0; r < RI; ++r) av[r] = ASMEM ? sA[k * NP + i0 + r] : __ldg(&sA[k * NP + i0 + r]);
#pragma unroll
        for (int c = 0; c < NC; ++c) bv[c] = b[k * NC + c];
#pragma unroll
        for (int r = 0; r < RI; ++r)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
      }
      const size_t e = size_t(cell0 + el) * 6 + t;
#pragma unroll
      for (int r = 0; r < RI; ++r) {
        const int i = i0 + r;
        const size_t base = (e * NP + i) * NC;
        R src[NC];
        if (Phys::kSource) ph.source(&sQ[(el * NP + i) * NC], src);
        R out[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const R rhs = Phys::kSource ? acc[r][c] + src[c] : acc[r][c];
          out[c] = args.rhs_only ? rhs : args.a * args.q_a[base + c] + args.b * args.q_b[base + c] + args.cdt * rhs;
        }
        if (Phys::kLimit && !args.rhs_only) ph.limit(out);
#pragma unroll
        for (int c = 0; c < NC; ++c) args.q_out[base + c] = out[c];
      }
    }
  }
}

// Max over every element face node of the signal speed that
// numerical_flux / boundary_flux return (the reference discards it at
// src/solver.mojo:266-268); one thread per (element, face node).  Speeds are
// non-negative, so their IEEE bit patterns order like unsigned integers and
// atomicMax on the bits gives an order-independent (deterministic) max.
template <class R, class Phys, int P>
__global__ void wavespeed3d_kernel(Stage3DArgs<R> args, KuhnTab3<R> tab, Phys ph, unsigned long long* out) {
  constexpr int NC = Phys::NC, NP = ntet(P), NFP = ntri(P);
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double best = 0.0;
  if (tid < int64_t(args.ncell) * 6 * 4 * NFP) {
    const int64_t e = tid / (4 * NFP);
    const int fm = int(tid - e * 4 * NFP), lf = fm / NFP, m = fm - lf * NFP;
    const int t = int(e % 6);
    const int cell = int(e / 6), nxy = args.nx * args.ny;
    const int ck = cell / nxy, rem = cell - ck * nxy, cj = rem / args.nx, ci = rem - cj * args.nx;
    const int ax = tab.axis[t][lf], dir = tab.dir[t][lf];
    const int cpos = ax == 0 ? ci : (ax == 1 ? cj : ck);
    const int nax = ax == 0 ? args.nx : (ax == 1 ? args.ny : args.nz);
    int code;
    const int mode = face_mode(ax, dir, cpos, nax, args.bc, code);
    const R* qo = args.q_in + (e * NP + tab.own_node[lf][m]) * NC;
    R nx = tab.normal[t][lf][0], ny = tab.normal[t][lf][1], nz = tab.normal[t][lf][2];
    R f[NC], s;
    if (mode == FACE_BC_HI) s = ph.bnd_flux(qo, code, nx, ny, nz, f);
    else if (mode == FACE_BC_LO) s = ph.bnd_flux(qo, code, -nx, -ny, -nz, f);
    else {
      const int ni = wrapi(ci + tab.off[t][lf][0], args.nx), nj = wrapi(cj + tab.off[t][lf][1], args.ny),
                nk = wrapi(ck + tab.off[t][lf][2], args.nz);
      const size_t enb = (size_t(ni) + size_t(args.nx) * (nj + size_t(args.ny) * nk)) * 6 + tab.nb_t[t][lf];
      const R* qn = args.q_in + (enb * NP + tab.nb_node[t][lf][m]) * NC;
      if (mode == FACE_MIXED) s = ph.bnd_flux(qn, code, nx, ny, nz, f);
      else if (tab.side[t][lf] == 0) s = ph.num_flux(qo, qn, nx, ny, nz, f);
      else s = ph.num_flux(qn, qo, nx, ny, nz, f);
    }
    best = double(s);
    if (!(best >= 0.0)) best = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +inf flags it
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

template <class R, int P, int NC, int EB, bool ASMEM>
constexpr size_t stage3d_smem_bytes() {
  using S = Stage3DShape<P, NC, R>;
  return sizeof(R) * ((ASMEM ? size_t(S::K) * S::NP : 0) + size_t(EB) * S::NP * NC + size_t(EB) * S::BSTR);
}

}  // namespace mxm
