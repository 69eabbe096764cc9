// Fused 2D SSPRK3 stage kernel on a Kuhn triangle mesh (sm_100a).
//
// Replaces the reference's two launches per stage -- *_face_flux_kernel_2d
// (one thread per (face, slot) writing fstar to global memory) and
// *_vol_lift_combine_rk_kernel_2d (src/local_mesh_2d_gpu_euler.mojo:33-144
// and siblings) -- with one kernel.  A block owns EC whole cells (2
// triangles each, one contiguous span of q, bulk-copied into a
// double-buffered shared tile), keeps one shared operator
// A = [D_r | D_s | -Lift_0..2] for both triangle types (invJ applied to the
// nodal flux, side*length/(2A) to f*), evaluates volume fluxes and its
// edges' numerical fluxes into a shared B tile (the diagonal's neighbour
// trace comes from the tile), then rhs = A B + source and the RK combine.
// Face traces never touch global memory; connectivity is implicit.
//
// The per-tile work is the device function stage2d_tile, shared by the
// single-solve kernel below and the batched multi-solve kernel
// (batch2d.cuh).
#pragma once
#include "dg_common.cuh"
#include "physics2d.cuh"
#include "tma.cuh"

namespace mxm {

template <int P, int NC, class R>
struct Stage2DShape {
  static constexpr int NP = ntri(P), NFP = P + 1, K = 2 * NP + 3 * NFP;
  static constexpr int NS = NC | 1;  // node stride of the B tile (odd: node-parallel accesses miss no bank)
  static constexpr int BSTR_RAW = K * NS;
  static constexpr int BMOD = sizeof(R) == 8 ? 16 : 32;
  static constexpr int BSTR = BSTR_RAW + ((1 - BSTR_RAW % BMOD) + BMOD) % BMOD;
  // rows of the contraction per thread: a divisor of NP
  static constexpr int RI = P == 1 ? 1 : (P == 2 ? 2 : (P == 3 ? 2 : (P == 4 ? 3 : 3)));
  static constexpr size_t kPerCell = 2 * sizeof(R) * (2 * size_t(NP) * NC + BSTR);  // 2 q buffers + B rows
};

constexpr uint64_t kWaitLimitNs2 = 2000000000ull;

// One node's NC state values from the shared tile; four-component nodes
// (16- or 32-byte aligned in the tile) load as vectors, which keeps
// node-parallel reads free of bank conflicts.
template <int NC, class R>
__device__ __forceinline__ void load_node(const R* p, R* v) {
  if constexpr (NC == 4 && sizeof(R) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else if constexpr (NC == 4 && sizeof(R) == 8) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  } else {
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = p[c];
  }
}

// One tile of whole cells starting at cell0 (ne_here triangles), its state
// already in shared memory at q: volume and edge fluxes into sB, then
// rhs = A B + source and the RK combine into args.q_out.  Contains one
// block barrier; every thread of the block must call it.
template <class R, class Phys, int P, int NT>
__device__ __forceinline__ void stage2d_tile(const Stage2DArgs<R>& args, const KuhnTab2<R>* tab, const Phys& ph,
                                             const R* q, R* sB, const R* sA, int cell0, int ne_here) {
  constexpr int NC = Phys::NC;
  using S = Stage2DShape<P, NC, R>;
  constexpr int NP = S::NP, NFP = S::NFP, K = S::K, BSTR = S::BSTR, NS = S::NS, RI = S::RI, G = NP / RI;
  static_assert(NP % RI == 0, "row tile must divide NP");
  const int tid = threadIdx.x;
  for (int idx = tid; idx < ne_here * NP; idx += NT) {
    const int el = idx / NP, j = idx - el * NP, t = el & 1;
    R Fx[NC], Fy[NC], qv[NC];
    load_node<NC>(&q[(el * NP + j) * NC], qv);
    ph.flux(qv, Fx, Fy);
    const R* iJ = tab->invJ[t];
    R* b = &sB[el * BSTR + j * NS];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      b[c] = iJ[0] * Fx[c] + iJ[1] * Fy[c];
      b[NP * NS + c] = iJ[2] * Fx[c] + iJ[3] * Fy[c];
    }
  }
  for (int idx = tid; idx < ne_here * 3 * NFP; idx += NT) {
    const int el = idx / (3 * NFP), fm = idx - el * 3 * NFP;
    const int lf = fm / NFP, m = fm - lf * NFP, t = el & 1, cl = el >> 1;
    const int cell = cell0 + cl;
    const int cj = cell / args.nx, ci = cell - cj * args.nx;
    const int ax = tab->axis[t][lf], dir = tab->dir[t][lf];
    int code;
    const int mode = face_mode(ax, dir, ax == 0 ? ci : cj, ax == 0 ? args.nx : args.ny, args.bc, code);
    R qo[NC];
    load_node<NC>(&q[(el * NP + tab->own_node[lf][m]) * NC], qo);
    R nx = tab->normal[t][lf][0], ny = tab->normal[t][lf][1];
    R scale = tab->fscale[t][lf];
    // one face-flux call per face node (the 2D face functions build the
    // BC ghost state themselves from the left state and the BC code)
    R qn[NC];
    if (mode == FACE_INTERIOR || mode == FACE_MIXED) {
      const int nbt = tab->nb_t[t][lf], nbn = tab->nb_node[t][lf][m];
      if (ax < 0) {
        load_node<NC>(&q[((cl * 2 + nbt) * NP + nbn) * NC], qn);
      } else {
        const int ni = wrapi(ci + tab->off[t][lf][0], args.nx), nj = wrapi(cj + tab->off[t][lf][1], args.ny);
        const R* gq = args.q_in + ((size_t(nj) * args.nx + ni) * 2 * NP + size_t(nbt) * NP + nbn) * NC;
#pragma unroll
        for (int c = 0; c < NC; ++c) qn[c] = __ldg(gq + c);
      }
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) qn[c] = qo[c];
    }
    if (mode == FACE_BC_LO) {
      nx = -nx;
      ny = -ny;
      scale = -scale;
    }
    const bool bcf = mode != FACE_INTERIOR;
    const bool own_left = tab->side[t][lf] == 0;
    // left/right states by value (selecting between pointers would force
    // the register arrays into local memory)
    R L[NC], Rr[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const R o = qo[c];
      L[c] = bcf ? qn[c] : (own_left ? o : qn[c]);
      Rr[c] = bcf ? qn[c] : (own_left ? qn[c] : o);
    }
    R f[NC];
    ph.face(L, Rr, bcf ? code : int(BC_INTERIOR), nx, ny, f);
    R* b = &sB[el * BSTR + (2 * NP + fm) * NS];
#pragma unroll
    for (int c = 0; c < NC; ++c) b[c] = scale * f[c];
  }
  __syncthreads();
  const bool a_in = args.q_a == args.q_in, b_in = args.q_b == args.q_in;
  for (int w = tid; w < ne_here * G; w += NT) {
    const int el = w / G, g = w - el * G;
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
      for (int c = 0; c < NC; ++c) bv[c] = b[k * NS + c];
#pragma unroll
      for (int r = 0; r < RI; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
    }
    const size_t e = size_t(cell0) * 2 + el;
#pragma unroll
    for (int r = 0; r < RI; ++r) {
      const int i = i0 + r;
      const size_t base = (e * NP + i) * NC;
      R ql[NC];
      load_node<NC>(&q[(el * NP + i) * NC], ql);
      R src[NC];
      if (Phys::kSource) ph.source(ql, src);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const R rhs = Phys::kSource ? acc[r][c] + src[c] : acc[r][c];
        const R va = a_in ? ql[c] : args.q_a[base + c];
        const R vb = b_in ? ql[c] : args.q_b[base + c];
        args.q_out[base + c] = args.rhs_only ? rhs : va + args.b * (vb - va) + args.cdt * rhs;
      }
    }
  }
}

template <class R, class Phys, int P, int EC, int NT>
__global__ void __launch_bounds__(NT) stage2d_kernel(Stage2DArgs<R> args, KuhnTab2<R> tabp, Phys ph) {
  constexpr int NC = Phys::NC;
  using S = Stage2DShape<P, NC, R>;
  constexpr int NP = S::NP, K = S::K, BSTR = S::BSTR;
  constexpr int EB = 2 * EC, QV = EB * NP * NC;
  constexpr bool BULK = (2 * NP * NC * sizeof(R)) % 16 == 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  KuhnTab2<R>* tab = reinterpret_cast<KuhnTab2<R>*>(smem_raw + 16);
  constexpr size_t kTabBytes = (sizeof(KuhnTab2<R>) + 15) / 16 * 16;
  R* sQ = reinterpret_cast<R*>(smem_raw + 16 + kTabBytes);  // [2][QV]
  R* sB = sQ + 2 * QV;                                      // [EB][BSTR]
  R* sA = sB + EB * BSTR;                                   // [K][NP]
  const int tid = threadIdx.x;
  const int ngroups = (args.ncell + EC - 1) / EC;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  {
    const int* src = reinterpret_cast<const int*>(&tabp);
    int* dst = reinterpret_cast<int*>(tab);
    for (int k = tid; k < int(sizeof(KuhnTab2<R>) / 4); k += NT) dst[k] = src[k];
  }
  for (int idx = tid; idx < NP * K; idx += NT) sA[idx] = args.A[idx];
  __syncthreads();
  auto issue = [&](int grp, int buf) {
    const int c0 = grp * EC, nc = min(EC, args.ncell - c0);
    const uint32_t bytes = uint32_t(nc) * 2u * NP * NC * sizeof(R);
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[buf], bytes);
    bulk_g2s(sQ + buf * QV, args.q_in + size_t(c0) * 2 * NP * NC, bytes, &bar[buf]);
    // the tile's q_a (read by the epilogue when it is not the tile's own
    // state) into L2 a tile ahead of its use
    if (!args.rhs_only && args.q_a != args.q_in) bulk_prefetch_l2(args.q_a + size_t(c0) * 2 * NP * NC, bytes);
  };
  uint32_t par = 0u;  // bit b: phase parity of tile buffer b
  int buf = 0;
  if (BULK && tid == 0 && int(blockIdx.x) < ngroups) issue(blockIdx.x, 0);

  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x, buf ^= 1) {
    const int cell0 = grp * EC;
    const int ne_here = 2 * min(EC, args.ncell - cell0);
    R* q = sQ + buf * QV;
    if (BULK) {
      if (!block_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs2)) {
        // the copy into this tile is the only one in flight: give it one
        // more bounded wait before the block (and its shared memory) ends
        if (tid == 0) {
          if (args.err) atomicOr(args.err, 1);
          mbar_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs2);
        }
        return;
      }
      par ^= 1u << buf;
      if (tid == 0 && grp + int(gridDim.x) < ngroups) issue(grp + gridDim.x, buf ^ 1);
    } else {
      const R* src = args.q_in + size_t(cell0) * 2 * NP * NC;
      for (int idx = tid; idx < ne_here * NP * NC; idx += NT) q[idx] = src[idx];
      __syncthreads();
    }
    stage2d_tile<R, Phys, P, NT>(args, tab, ph, q, sB, sA, cell0, ne_here);
  }
}

template <class R, int P, int NC>
struct Cfg2 {
  using S = Stage2DShape<P, NC, R>;
  static constexpr int NP = S::NP;
  static constexpr size_t kFixed = 16 + (sizeof(KuhnTab2<R>) + 15) / 16 * 16 + sizeof(R) * S::K * S::NP;
  static constexpr int EC_RAW = int((100 * 1024 - kFixed) / S::kPerCell);
  static constexpr int EC = EC_RAW > 64 ? 64 : (EC_RAW < 1 ? 1 : EC_RAW);
  static constexpr int NT = 256;
  static constexpr size_t kSmem = kFixed + sizeof(R) * (2 * size_t(2 * EC) * S::NP * NC + size_t(2 * EC) * S::BSTR);
};

template <class R, class Phys, int P>
cudaError_t launch2_p(const Stage2DArgs<R>& a, const KuhnTab2<R>& tab, const Phys& ph, int nsm, cudaStream_t st) {
  using C = Cfg2<R, P, Phys::NC>;
  auto kern = stage2d_kernel<R, Phys, P, C::EC, C::NT>;
  static int bps = -1;
  if (bps < 0) {
    cudaError_t e = persistent_blocks_per_sm((const void*)kern, C::NT, C::kSmem, &bps);
    if (e != cudaSuccess) return e;
  }
  const int ngroups = (a.ncell + C::EC - 1) / C::EC;
  int nblk = nsm * bps;
  if (nblk > ngroups) nblk = ngroups;
  if (nblk < 1) nblk = 1;
  kern<<<nblk, C::NT, C::kSmem, st>>>(a, tab, ph);
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
