// Fused 3D SSPRK3 stage kernel on a Kuhn tetrahedral mesh (sm_100a).
//
// Replaces mojoxm's rk_stage_kernel (src/solver.mojo:161-337): per element,
// pointwise physical flux, face-trace gather + numerical/boundary flux,
// volume contraction sum_j sum_k D_k[i,j] (invJ F_j)_k, lift
// sum_f sign*area*Lift*f*, source, RK combine a*q_a + b*q_b + c*dt*rhs and
// the positivity floor.
//
// B200 design:
//  * A block owns EC whole cubes (EB = 6*EC consecutive elements, one
//    contiguous span of q) per iteration of a persistent loop.  The span
//    arrives by a 1D bulk copy (TMA engine) into a double-buffered shared
//    tile, prefetched one iteration ahead, completion tracked by an mbarrier
//    with a bounded wait.
//  * One operator serves all six tet types: A = [D_r|D_s|D_t|-Lift_0..3]
//    (NP x K, K = 3NP + 4NFP) lives in shared memory for the block's life;
//    the per-type invJ is applied to the nodal flux and the per-face scale
//    side*area/(6V) to f*, so every element's RHS is rhs = A B with
//    B = [Fr; Fs; Ft; f*] (K x NC) in shared memory.
//  * Connectivity is never read from memory: neighbour element and node
//    follow from (cube, type) and a 1.7 KB topology table copied to shared
//    memory.  Faces between tets of the same cube read both traces from the
//    shared tile and are solved once (by the side-0 tet, which writes both
//    tets' rows); only cube-boundary faces gather from global memory, with
//    the neighbour cube and BC treatment of each cube face resolved once per
//    tile.
//  * q_a / q_b equal to q_in (SSPRK3 stages 1-3) are read from the tile, so
//    each stage moves the algorithmic minimum of state bytes.
//  * Where a tile's contraction works (element x RI-row group) would leave
//    most of the block idle (one-cube tiles at P4/P5 in FP64), KS lanes of
//    a warp share a work, each summing every KS-th K column, and a shuffle
//    butterfly (ks_fold) gives each lane complete rows for the epilogue.
#pragma once
#include <type_traits>

#include "dg_common.cuh"
#include "physics.cuh"
#include "tma.cuh"

namespace mxm {

template <int P, int NC, class R>
struct Stage3DShape {
  static constexpr int NP = ntet(P), NFP = ntri(P), K = 3 * NP + 4 * NFP;
  // element stride of the B tile, padded so that elements read in the same
  // warp land in distinct banks
  static constexpr int BSTR = stage3d_bstr(P, NC, int(sizeof(R)));
};

// Rows a lane holds after ks_fold over a group of 2M lanes: the row set
// halves (rounded up) at every level.
constexpr int ks_rows(int n, int m) { return m >= 1 ? ks_rows((n + 1) / 2, m / 2) : n; }

// K-split contraction: the 2M lanes of one aligned group each summed every
// 2M-th K column of the same RI x NC tile.  A butterfly that halves the row
// set at every level (lanes with bit m set keep the upper rows) leaves this
// lane the complete sums of rows base .. base + cnt - 1 in acc[0 .. cnt).
// Every sum adds the same partials in the same tree order on every run.
template <int M, int N, int RI, int NC, class R>
__device__ __forceinline__ void ks_fold(R (&acc)[RI][NC], unsigned gmask, int lane, int& base, int& cnt) {
  if constexpr (M >= 1) {
    constexpr int LO = (N + 1) / 2;
    const bool hi = (lane & M) != 0;
#pragma unroll
    for (int j = 0; j < LO; ++j) {
      const bool has_up = j + LO < N;
      const int ju = has_up ? j + LO : 0;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const R up = has_up ? acc[ju][c] : R(0);
        const R send = hi ? acc[j][c] : up;
        const R keep = hi ? up : acc[j][c];
        acc[j][c] = keep + __shfl_xor_sync(gmask, send, M);
      }
    }
    if (hi) {
      base += LO;
      cnt = cnt > LO ? cnt - LO : 0;
    } else {
      cnt = cnt < LO ? cnt : LO;
    }
    ks_fold<M / 2, LO, RI, NC, R>(acc, gmask, lane, base, cnt);
  }
}

template <class R, class Phys, int P, int EC, int RI, int KS, int NT, bool ASMEM>
__global__ void __launch_bounds__(NT) stage3d_kernel(Stage3DArgs<R> args, KuhnTab3<R> tabp, Phys ph) {
  constexpr int NC = Phys::NC;
  using S = Stage3DShape<P, NC, R>;
  constexpr int NP = S::NP, NFP = S::NFP, K = S::K, BSTR = S::BSTR;
  constexpr int EB = 6 * EC, G = NP / RI, QV = EB * NP * NC;
  static_assert(NP % RI == 0, "row tile must divide NP");
  static_assert(KS >= 1 && KS <= 16 && (KS & (KS - 1)) == 0 && NT % KS == 0, "K split: power of two within a warp");
  // operator rows read from shared memory as 16-byte vectors where the row
  // tile and the operator's offset in shared memory allow it
  constexpr size_t kAOff = 16 + (sizeof(KuhnTab3<R>) + 15) / 16 * 16 + sizeof(R) * (2 * size_t(QV) + size_t(EB) * BSTR);
  constexpr int AV = 16 / int(sizeof(R));
  constexpr bool AVEC = ASMEM && NP % AV == 0 && RI % AV == 0 && kAOff % 16 == 0;
  using RV = typename std::conditional<sizeof(R) == 8, double2, float4>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);                       // [2]
  KuhnTab3<R>* tab = reinterpret_cast<KuhnTab3<R>*>(smem_raw + 16);            // topology
  constexpr size_t kTabBytes = (sizeof(KuhnTab3<R>) + 15) / 16 * 16;
  R* sQ = reinterpret_cast<R*>(smem_raw + 16 + kTabBytes);                     // [2][QV]
  R* sB = sQ + 2 * QV;                                                         // [EB][BSTR]
  R* sA = sB + EB * BSTR;                                                      // [K][NP] (ASMEM)
  int* sNb = reinterpret_cast<int*>(sA + (ASMEM ? K * NP : 0));                // [EC][6] neighbour cubes
  int* sMd = sNb + EC * 6;                                                     // [EC][6] face modes
  const R* Aop = ASMEM ? sA : args.A;

  const int tid = threadIdx.x;
  grid_dep_launch();  // the next stage may set up as this one's blocks finish
  const int ngroups = (args.ncell - args.cbeg + EC - 1) / EC;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  {
    const int* src = reinterpret_cast<const int*>(&tabp);
    int* dst = reinterpret_cast<int*>(tab);
    for (int k = tid; k < int(sizeof(KuhnTab3<R>) / 4); k += NT) dst[k] = src[k];
  }
  if (ASMEM)
    for (int idx = tid; idx < NP * K; idx += NT) sA[idx] = args.A[idx];
  __syncthreads();

  auto issue = [&](int grp, int buf) {
    const int c0 = args.cbeg + grp * EC, nc = min(EC, args.ncell - c0);
    const uint32_t bytes = uint32_t(nc) * 6u * NP * NC * sizeof(R);
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[buf], bytes);
    bulk_g2s(sQ + buf * QV, args.q_in + size_t(c0) * 6 * NP * NC, bytes, &bar[buf]);
    // the tile's q_a (read by the epilogue when it is not the tile's own
    // state) into L2 a tile ahead of its use
    if (!args.rhs_only && args.q_a != args.q_in) bulk_prefetch_l2(args.q_a + size_t(c0) * 6 * NP * NC, bytes);
  };
  // bulk copy when the tile span starts and ends on 16-byte boundaries
  // (whole tiles of the usual shapes; a partial last tile may take plain loads)
  auto tile_bulk = [&](int g) -> bool {
    const size_t per_cube = size_t(6) * NP * NC * sizeof(R);
    const int cg = args.cbeg + g * EC;
    const size_t start = reinterpret_cast<uintptr_t>(args.q_in) + size_t(cg) * per_cube;
    const size_t bytes = size_t(min(EC, args.ncell - cg)) * per_cube;
    return start % 16 == 0 && bytes % 16 == 0;
  };
  uint32_t par = 0u;  // bit b: phase parity of tile buffer b
  int buf = 0;
  // the set-up above overlaps the previous stage's tail; its output (this
  // stage's q_in / q_a / q_b, and q_out may be a buffer it still reads)
  // only after it has completed
  grid_dep_wait();
  if (tid == 0 && int(blockIdx.x) < ngroups && tile_bulk(blockIdx.x)) issue(blockIdx.x, 0);

  const int nwork = tab->n_face_work;
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x, buf ^= 1) {
    const int cell0 = args.cbeg + grp * EC;
    const int nhere = min(EC, args.ncell - cell0);
    const int ne_here = 6 * nhere;
    R* q = sQ + buf * QV;
    if (tile_bulk(grp)) {
      if (!block_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs)) {
        // the copy into this tile is the only one in flight: give it one
        // more bounded wait before the block (and its shared memory) ends
        if (tid == 0) {
          if (args.err) atomicOr(args.err, 1);
          mbar_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs);
        }
        return;
      }
      par ^= 1u << buf;
      if (tid == 0 && grp + int(gridDim.x) < ngroups && tile_bulk(grp + gridDim.x)) issue(grp + gridDim.x, buf ^ 1);
    } else {
      const R* src = args.q_in + size_t(cell0) * 6 * NP * NC;
      for (int idx = tid; idx < ne_here * NP * NC; idx += NT) q[idx] = src[idx];
    }
    for (int w = tid; w < nhere * 6; w += NT) {
      const int cl = w / 6, dd = w - cl * 6;
      cube_dirs3(cell0 + cl, args.nx, args.ny, args.nz, args.bc, sNb + cl * 6, sMd + cl * 6, dd);
    }
    __syncthreads();
    // ---- volume fluxes in reference coordinates -> B rows k*NP + j
    for (int idx = tid; idx < ne_here * NP; idx += NT) {
      const int el = idx / NP, j = idx - el * NP, t = el % 6;
      R F[3 * NC];
      ph.flux(&q[(el * NP + j) * NC], F);
      const R* iJ = tab->invJ[t];
      R* b = &sB[el * BSTR + j * NC];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < NC; ++c)
          b[k * NP * NC + c] = iJ[k * 3 + 0] * F[c] + iJ[k * 3 + 1] * F[NC + c] + iJ[k * 3 + 2] * F[2 * NC + c];
    }
    // ---- face numerical fluxes, scaled by side*area/(6V) -> B rows 3NP + lf*NFP + m
    for (int idx = tid; idx < EC * nwork * NFP; idx += NT) {
      const int cl = idx % EC, rest = idx / EC, m = rest % NFP, wk = rest / NFP;
      if (cl >= nhere) continue;
      const int tl = tab->face_work[wk], t = tl >> 2, lf = tl & 3;
      const int el = cl * 6 + t, ax = tab->axis[t][lf], nbt = tab->nb_t[t][lf];
      int mode = FACE_INTERIOR, code = 0, nbcube = 0;
      if (ax >= 0) {
        const int dd = 2 * ax + (tab->dir[t][lf] > 0 ? 1 : 0);
        const int md = sMd[cl * 6 + dd];
        mode = md & 0xff;
        code = md >> 8;
        nbcube = sNb[cl * 6 + dd];
      }
      const R* qo = &q[(el * NP + tab->own_node[lf][m]) * NC];
      R nx = tab->normal[t][lf][0], ny = tab->normal[t][lf][1], nz = tab->normal[t][lf][2];
      R scale = tab->fscale[t][lf];
      // Resolve the face to (left, right, normal) and call the Riemann
      // solver once: BC faces use the ghost state (boundary_flux ==
      // numerical_flux(q_int, ghost)), interior faces keep side-0 on the left.
      R qn[NC], qg[NC];
      if (mode == FACE_INTERIOR || mode == FACE_MIXED) {
        const int nbn = tab->nb_node[t][lf][m];
        if (ax < 0) {  // face inside the cube: neighbour trace is in the tile
#pragma unroll
          for (int c = 0; c < NC; ++c) qn[c] = q[((cl * 6 + nbt) * NP + nbn) * NC + c];
        } else {
          const R* gq = args.q_in + ((size_t(nbcube) * 6 + nbt) * NP + nbn) * NC;
#pragma unroll
          for (int c = 0; c < NC; ++c) qn[c] = __ldg(gq + c);
        }
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c) qn[c] = qo[c];
      }
      if (mode == FACE_BC_LO) {  // one-sided face: the element is its side 0, outward normal -n
        nx = -nx;
        ny = -ny;
        nz = -nz;
        scale = -scale;
      }
      const bool bcf = mode != FACE_INTERIOR;
      if (bcf) ph.ghost(qn, code, nx, ny, nz, qg);  // BC_HI/BC_LO: qn = own trace; MIXED: neighbour's
      const bool own_left = bcf ? (mode != FACE_MIXED) : (tab->side[t][lf] == 0);
      // left/right states by value (selecting between pointers would force
      // the register arrays into local memory)
      R L[NC], Rr[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const R o = qo[c];
        L[c] = bcf ? qn[c] : (own_left ? o : qn[c]);
        Rr[c] = bcf ? qg[c] : (own_left ? qn[c] : o);
      }
      R f[NC];
      ph.num_flux(L, Rr, nx, ny, nz, f);
      R* b = &sB[el * BSTR + (3 * NP + lf * NFP + m) * NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) b[c] = scale * f[c];
      if (ax < 0) {  // the other tet of this inner face: same flux, its own scale
        const int lf2 = tab->nb_lf[t][lf];
        const R s2 = tab->fscale[nbt][lf2];
        R* b2 = &sB[(cl * 6 + nbt) * BSTR + (3 * NP + lf2 * NFP + tab->nb_m[t][lf][m]) * NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) b2[c] = s2 * f[c];
      }
    }
    __syncthreads();
    // ---- contraction rhs = A B, source, RK combine, floor, store.  A work
    // is an RI x NC tile of one element; KS consecutive lanes share it, each
    // summing every KS-th K column, and ks_fold hands each lane its rows.
    const bool a_in = args.q_a == args.q_in, b_in = args.q_b == args.q_in;
    constexpr int RO = ks_rows(RI, KS / 2);
    for (int w = tid; w < ne_here * G * KS; w += NT) {
      const int wk = w / KS, s = w - wk * KS;
      const int el = wk / G, g = wk - el * G;
      const int i0 = g * RI;
      R acc[RI][NC];
#pragma unroll
      for (int r = 0; r < RI; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[r][c] = R(0);
      const R* b = &sB[el * BSTR];
#pragma unroll 4
      for (int k = s; k < K; k += KS) {
        R av[RI], bv[NC];
        if constexpr (AVEC) {
#pragma unroll
          for (int r = 0; r < RI; r += AV) {
            const RV v = *reinterpret_cast<const RV*>(&Aop[k * NP + i0 + r]);
            if constexpr (sizeof(R) == 8) {
              av[r] = R(v.x);
              av[r + 1] = R(v.y);
            } else {
              const float4 f = *reinterpret_cast<const float4*>(&v);
              av[r] = R(f.x);
              av[r + 1] = R(f.y);
              av[r + 2] = R(f.z);
              av[r + 3] = R(f.w);
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < RI; ++r) av[r] = ASMEM ? Aop[k * NP + i0 + r] : __ldg(&Aop[k * NP + i0 + r]);
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) bv[c] = b[k * NC + c];
#pragma unroll
        for (int r = 0; r < RI; ++r)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
      }
      int rbase = 0, rcnt = RI;
      if constexpr (KS > 1) {
        const int lane = tid & 31;
        const unsigned gmask = ((1u << KS) - 1u) << (lane & ~(KS - 1));
        ks_fold<KS / 2, RI, RI, NC, R>(acc, gmask, lane, rbase, rcnt);
      }
      const size_t e = size_t(cell0) * 6 + el;
#pragma unroll
      for (int r = 0; r < RO; ++r) {
        if (r >= rcnt) break;
        const int i = i0 + rbase + r;
        const size_t base = (e * NP + i) * NC;
        const R* ql = &q[(el * NP + i) * NC];
        R src[NC];
        if (Phys::kSource) ph.source(ql, src);
        R out[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const R rhs = Phys::kSource ? acc[r][c] + src[c] : acc[r][c];
          if (args.rhs_only) {
            out[c] = rhs;
          } else {
            const R va = a_in ? ql[c] : args.q_a[base + c];
            const R vb = b_in ? ql[c] : args.q_b[base + c];
            out[c] = va + args.b * (vb - va) + args.cdt * rhs;
          }
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
  if (tid < int64_t(args.ncell - args.cbeg) * 6 * 4 * NFP) {
    const int64_t el = tid / (4 * NFP), e = int64_t(args.cbeg) * 6 + el;
    const int fm = int(tid - el * 4 * NFP), lf = fm / NFP, m = fm - lf * NFP;
    const int t = int(e % 6);
    const int cell = int(e / 6), nxy = args.nx * args.ny;
    const int ck = cell / nxy, rem = cell - ck * nxy, cj = rem / args.nx, ci = rem - cj * args.nx;
    const int ax = tab.axis[t][lf], dir = tab.dir[t][lf];
    int code;
    const int mode = face_mode(ax, dir, ax == 0 ? ci : (ax == 1 ? cj : ck),
                               ax == 0 ? args.nx : (ax == 1 ? args.ny : args.nz), args.bc, code);
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

template <class R, int P, int NC, int EC, bool ASMEM>
constexpr size_t stage3d_smem_bytes() {
  return stage3d_smem(P, NC, int(sizeof(R)), EC, ASMEM);
}

}  // namespace mxm
