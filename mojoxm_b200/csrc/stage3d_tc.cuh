// Mixed-precision 3D stage kernel: FP32 state, fluxes and Riemann solves,
// the volume + lift contraction on the 5th-generation tensor cores
// (tcgen05.mma, split-BF16 operands, FP32 accumulation in tensor memory).
//
// Same dataflow as stage3d_kernel (whole cubes per tile, bulk-copied
// double-buffered state, implicit connectivity), with the contraction in
// the transposed form
//     RHS^T[(c,el), i] = sum_k  B^T[(c,el), k] * A[i, k]
// so one 128-row MMA tile covers the (component, element) pairs of a tile
// against the shared operator A (N = NP rounded up to 16, K = 3NP + 4NFP
// rounded up to the MMA K step).  Operands are split x = hi + lo in
// bfloat16 (kind::f16) or TF32 (kind::tf32) and the product is
// hi*hi + hi*lo + lo*hi (three MMAs into one FP32 accumulator).
//
// Accuracy: before splitting, every element subtracts its own constant flux
// Fbar = F(q at node 0) from its volume fluxes and Fbar.n from its face
// fluxes.  The weak-form operator maps a constant flux to zero
// (sum_j D_k[i,j] = lift of the constant normal flux), so the RHS is
// unchanged in exact arithmetic while the operands -- and with them the
// cancellation error of the O(|F|/h) terms -- shrink to the flux variation
// across the element.
//
// Layout: the (c,el) x K operand is MN-major for split-BF16 (8 consecutive
// rows of one k in 16 bytes) and K-major for split-TF32 (4 consecutive k of
// one row in 16 bytes).  Work is mapped element-fastest: 8 consecutive threads take 8
// consecutive elements at the same node, so a warp's operand stores land in
// one or two 128-byte core matrices.  Faces are walked through a per-cube
// work list (every cube-boundary face, and each face inside the cube once,
// by its side-0 tet, which writes both tets' rows); the neighbour cube and
// boundary treatment of the six cube faces are resolved once per tile.  One
// thread issues the MMAs; completion is tracked by tcgen05.commit on an
// mbarrier with a bounded wait; warps 0-3 read the accumulator with
// tcgen05.ld into a padded [row][i] staging tile for the FP32 epilogue
// (source, RK combine, positivity floor).
#pragma once
#include "dg_common.cuh"
#include "physics.cuh"
#include "tc.cuh"

namespace mxm {

__host__ __device__ constexpr int rup16(int x) { return (x + 15) / 16 * 16; }
__host__ __device__ constexpr int rupk(int x, int k) { return (x + k - 1) / k * k; }
__host__ __device__ constexpr int tmem_cols_for(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 256)); }

// The K dimension is split into the volume columns (3 NP, padded to KV) and
// the face columns (4 NFP, padded to KF), each padded to the operand kind's
// MMA K step; both halves reuse one operand buffer of KB = max(KV, KF)
// columns, and the operator image stores the face columns from KV on
// (tc_operator_image's `kvol`).
template <int P, int NC, class Op = OpBF16>
struct TcShape {
  static constexpr int NP = ntet(P), NFP = ntri(P), K = 3 * NP + 4 * NFP;
  static constexpr int KV = rupk(3 * NP, Op::KSTEP), KF = rupk(4 * NFP, Op::KSTEP), KA = KV + KF;
  static constexpr int KB = KV > KF ? KV : KF;
  static constexpr int NN = rup16(NP), M = 128;
  static constexpr int EBP = (M / NC) / 8 * 8;      // element slots per component (multiple of 8)
  static constexpr int EC = EBP / 6, EB = 6 * EC;   // whole cubes in a tile
  static constexpr int NPO = NP | 1;                // odd row stride of the accumulator staging tile
  static constexpr int NCOLS = tmem_cols_for(NN);
  static constexpr size_t A_BYTES = size_t(NN) * KA * Op::ELEM;  // one of hi / lo
  static constexpr size_t B_BYTES = size_t(M) * KB * Op::ELEM;
  static constexpr size_t Q_BYTES = size_t(EB) * NP * NC * 4;
  static constexpr size_t O_BYTES = size_t(M) * NPO * 4;   // aliases the operand buffer (free by then)
  static constexpr size_t FB_BYTES = size_t(EB) * 3 * NC * 4;
  static constexpr size_t FN_BYTES = size_t(EB) * 4 * NC * 4;  // Fbar . n per (element, face)
  static constexpr size_t CD_BYTES = size_t(EC) * 12 * 4;  // per cube: 6 neighbour cubes + 6 face modes
  // per face-work entry: normal, scale, the inner neighbour's scale, packed
  // indices; per (entry, face node): own / neighbour node, neighbour's slot
  static constexpr size_t FR_BYTES = 24 * 8 * 4, FM_BYTES = size_t(24) * NFP * 4;
  static constexpr size_t HDR = 128;
  static constexpr size_t TAB = (sizeof(KuhnTab3<float>) + 127) / 128 * 128;
  static constexpr size_t FIXED0 = HDR + TAB + 2 * A_BYTES + 2 * B_BYTES + FB_BYTES + FN_BYTES + CD_BYTES;
  static constexpr size_t FIXED1 = FIXED0 + 16 + FR_BYTES + FM_BYTES;
  // State tile buffers: two (prefetch the next tile during this one) unless
  // a single buffer lets more blocks share an SM (228 KB of shared memory
  // per SM, 1 KB reserved per block on sm_100a; at most 4 blocks of 256
  // threads at the kernel's ~64 registers per thread).
  static constexpr size_t blocks_for(size_t s) {
    return size_t(228 * 1024) / (s + 1024) < 4 ? size_t(228 * 1024) / (s + 1024) : 4;
  }
  static constexpr int qb_for(size_t fixed) {
    return blocks_for(fixed + Q_BYTES) > blocks_for(fixed + 2 * Q_BYTES) ? 1 : 2;
  }
  // the face records only where they cost neither a block per SM nor the
  // second state buffer
  static constexpr bool FREC = qb_for(FIXED1) >= qb_for(FIXED0) &&
                               blocks_for(FIXED1 + qb_for(FIXED1) * Q_BYTES) >= blocks_for(FIXED0 + qb_for(FIXED0) * Q_BYTES);
  static constexpr size_t FIXED = FREC ? FIXED1 : FIXED0;
  static constexpr int QB = qb_for(FIXED);
  static constexpr size_t OFF_A = HDR + TAB;
  static constexpr size_t OFF_B = OFF_A + 2 * A_BYTES;
  static constexpr size_t OFF_Q = OFF_B + 2 * B_BYTES;
  static constexpr size_t OFF_F = OFF_Q + QB * Q_BYTES;
  static constexpr size_t OFF_N = OFF_F + FB_BYTES;
  static constexpr size_t OFF_C = OFF_N + FN_BYTES;
  static constexpr size_t OFF_R = (OFF_C + CD_BYTES + 15) / 16 * 16;
  static constexpr size_t OFF_M = OFF_R + FR_BYTES;
  static constexpr size_t SMEM = FREC ? OFF_M + FM_BYTES : OFF_C + CD_BYTES;
  static constexpr bool BULK = (6 * NP * NC * 4) % 16 == 0;
  static_assert(O_BYTES <= 2 * B_BYTES, "staging tile must fit the operand buffer");
  static constexpr bool FITS = SMEM + 1024 <= size_t(227 * 1024);
  // batched launches: the current solve's stage arguments behind the tile
  static constexpr size_t OFF_ARGS = (SMEM + 15) / 16 * 16, BATCH_SMEM = OFF_ARGS + 256;
};

// Blocks per SM the register allocation must allow: what fits in shared
// memory, at most three for register-light fluxes and two for the Roe /
// HLLE / HLLEC solvers (capping those at three blocks' registers spills).
template <class Phys, int P, class Op>
__host__ __device__ constexpr int tc_min_blocks() {
  return int(TcShape<P, Phys::NC, Op>::blocks_for(TcShape<P, Phys::NC, Op>::SMEM)) < (Phys::kLightFlux ? 3 : 2)
             ? int(TcShape<P, Phys::NC, Op>::blocks_for(TcShape<P, Phys::NC, Op>::SMEM))
             : (Phys::kLightFlux ? 3 : 2);
}

// BATCH: the tiles of many solves of one physics, order and operand kind
// (Tc3Batch: per-tile {solve, first cell, cells}, grouped by solve; per
// solve its stage arguments and metric table).  Each block takes a
// contiguous range of tiles; when the solve changes, the block reloads the
// solve's arguments (into shared memory, `args` then refers there), table
// and face records.  A solve's tiles get exactly the arithmetic of the
// single-solve launch, so batched results are bit-identical to it.
// Single-solve launches pass `args0` / `tabp` and leave `bat` empty.
template <class Phys, int P, int NT, class Op, bool BATCH>
__global__ void __launch_bounds__(NT, tc_min_blocks<Phys, P, Op>()) stage3d_tc_kernel(
    Stage3DArgs<float> args0, const __grid_constant__ KuhnTab3<float> tabp, Phys ph,
    const unsigned char* __restrict__ a_image, const __grid_constant__ Tc3Batch bat) {
  constexpr int NC = Phys::NC;
  using S = TcShape<P, NC, Op>;
  constexpr int NP = S::NP, NFP = S::NFP, KV = S::KV, KF = S::KF, NN = S::NN, M = S::M, NPO = S::NPO;
  constexpr int EC = S::EC, EB = S::EB, EBP = S::EBP, QV = EB * NP * NC;
  // LBO of the K-major operator image and of the flux tile (MN-major for
  // split-BF16, K-major for split-TF32); the start-address step of one MMA
  // K step in each
  constexpr uint32_t LBO_A = NN * 16, LBO_B = umma_a_lbo<Op>(M), SBO = 128;
  constexpr uint32_t KSTEP_A = (Op::KSTEP / Op::CM) * LBO_A, KSTEP_B = umma_a_kstep<Op>(M);
  // byte step between the rows of consecutive components (EBP rows apart)
  constexpr uint32_t CSTRIDE = (EBP / (Op::A_MN ? Op::CM : 8)) * 128;
  constexpr uint32_t IDESC = umma_idesc_f32acc<Op>(M, NN);
  static_assert(NN % 16 == 0 && NN <= 256 && KV % Op::KSTEP == 0 && KF % Op::KSTEP == 0 && EC >= 1 &&
                    EBP * NC <= M && EBP % Op::CM == 0,
                "UMMA shape");
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // [0..1] q tiles, [2] mma, [3] A image
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 32);
  KuhnTab3<float>* tab = reinterpret_cast<KuhnTab3<float>*>(smem + S::HDR);
  unsigned char* sAhi = smem + S::OFF_A;
  unsigned char* sAlo = sAhi + S::A_BYTES;
  unsigned char* sBhi = smem + S::OFF_B;
  unsigned char* sBlo = sBhi + S::B_BYTES;
  float* sQ = reinterpret_cast<float*>(smem + S::OFF_Q);
  float* sO = reinterpret_cast<float*>(sBhi);              // [M rows (c, el)][NPO], after the MMAs
  float* sF = reinterpret_cast<float*>(smem + S::OFF_F);   // [EB][3][NC] element flux Fbar
  float* sFn = reinterpret_cast<float*>(smem + S::OFF_N);  // [EB][4][NC] Fbar . n of each face
  int* sNb = reinterpret_cast<int*>(smem + S::OFF_C);      // [EC][6] neighbour cube per direction
  int* sMd = sNb + EC * 6;                                 // [EC][6] face mode | code << 8
  float* sFR = reinterpret_cast<float*>(smem + S::OFF_R);  // [work][8] face records
  int* sFM = reinterpret_cast<int*>(smem + S::OFF_M);      // [work][NFP] face-node indices

  // the stage arguments: the kernel parameter, or the current solve's copy
  // in shared memory (batched launches)
  Stage3DArgs<float>* sArgs = reinterpret_cast<Stage3DArgs<float>*>(smem + S::OFF_ARGS);
  const Stage3DArgs<float>& args = BATCH ? *sArgs : args0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  grid_dep_launch();  // the next stage may set up as this one's blocks finish
  const int ngroups = BATCH ? bat.nitems : (args0.ncell - args0.cbeg + EC - 1) / EC;
  // tiles of this block: every gridDim.x-th from blockIdx.x (one solve), or
  // a contiguous range (batched)
  const int t_first = BATCH ? int(int64_t(blockIdx.x) * ngroups / gridDim.x) : int(blockIdx.x);
  const int t_end = BATCH ? int(int64_t(blockIdx.x + 1) * ngroups / gridDim.x) : ngroups;
  auto next_tile = [&](int g) -> int {
    if constexpr (BATCH) return g + 1 < t_end ? g + 1 : ngroups;
    else return g + int(gridDim.x);
  };
  auto tile_member = [&](int g) -> int {
    if constexpr (BATCH) return bat.items[g].x;
    else return 0;
  };
  auto tile_cell0 = [&](int g) -> int {
    if constexpr (BATCH) return bat.items[g].y;
    else return args0.cbeg + g * EC;
  };
  auto tile_cells = [&](int g) -> int {
    if constexpr (BATCH) return bat.items[g].z;
    else return min(EC, args0.ncell - args0.cbeg - g * EC);
  };
  auto tile_qin = [&](int g) -> const float* {
    if constexpr (BATCH) return bat.margs[bat.items[g].x].q_in;
    else return args0.q_in;
  };
  if (tid == 0) {
    for (int k = 0; k < 4; ++k) mbar_init(&bar[k], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, S::NCOLS);
    tmem_relinquish();
  }
  // the solve's metric table into shared memory and its face records,
  // decoded from the table: bits
  // t | lf << 3 | nb_t << 5 | nb_lf << 8 | (axis + 1) << 10 | (dir > 0) << 12 | (side == 0) << 13
  auto load_table = [&](const KuhnTab3<float>& tsrc) {
  {
    const int* src = reinterpret_cast<const int*>(&tsrc);
    int* dst = reinterpret_cast<int*>(tab);
    for (int k = tid; k < int(sizeof(KuhnTab3<float>) / 4); k += NT) dst[k] = src[k];
  }
  if constexpr (S::FREC) {
  for (int w = tid; w < tsrc.n_face_work; w += NT) {
    const int tl = tsrc.face_work[w], t = tl >> 2, lf = tl & 3;
    const int ax = tsrc.axis[t][lf], nbt = tsrc.nb_t[t][lf], lf2 = tsrc.nb_lf[t][lf];
    float* r = sFR + w * 8;
    r[0] = tsrc.normal[t][lf][0];
    r[1] = tsrc.normal[t][lf][1];
    r[2] = tsrc.normal[t][lf][2];
    r[3] = tsrc.fscale[t][lf];
    r[4] = ax < 0 ? tsrc.fscale[nbt][lf2] : 0.f;
    r[5] = __int_as_float(t | (lf << 3) | ((nbt & 7) << 5) | ((lf2 & 3) << 8) | ((ax + 1) << 10) |
                          ((tsrc.dir[t][lf] > 0 ? 1 : 0) << 12) | ((tsrc.side[t][lf] == 0 ? 1 : 0) << 13));
  }
  for (int idx = tid; idx < tsrc.n_face_work * NFP; idx += NT) {
    const int w = idx / NFP, m = idx - w * NFP;
    const int tl = tsrc.face_work[w], t = tl >> 2, lf = tl & 3;
    sFM[idx] = int(tsrc.own_node[lf][m]) | (int(tsrc.nb_node[t][lf][m]) << 8) | (int(tsrc.nb_m[t][lf][m]) << 16);
  }
  }
  };
  if constexpr (!BATCH) load_table(tabp);
  // zero the flux tiles once: padding rows / k columns stay zero for good
  for (int k = tid; k < int(2 * S::B_BYTES / 16); k += NT) reinterpret_cast<uint4*>(sBhi)[k] = make_uint4(0, 0, 0, 0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {  // operator image (hi | lo), already in the K-major UMMA layout
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[3], uint32_t(2 * S::A_BYTES));
    bulk_g2s(sAhi, a_image, uint32_t(2 * S::A_BYTES), &bar[3]);
  }
  // the tile's state into shared memory; the tile's q_a (read by the
  // epilogue when it is not the tile's own state) into L2 at the same time
  auto issue = [&](int grp, int buf) {
    const int c0 = tile_cell0(grp), nc = tile_cells(grp);
    const uint32_t bytes = uint32_t(nc) * 6u * NP * NC * 4u;
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[buf], bytes);
    const float* qin = tile_qin(grp);
    bulk_g2s(sQ + buf * QV, qin + size_t(c0) * 6 * NP * NC, bytes, &bar[buf]);
    const Stage3DArgs<float>& ta = BATCH ? bat.margs[bat.items[grp].x] : args0;
    if (!ta.rhs_only && ta.q_a != qin) bulk_prefetch_l2(ta.q_a + size_t(c0) * 6 * NP * NC, bytes);
  };
  // store the NC operand values v[c] of row (c, el), column k as bf16 hi / lo
  auto put = [&](int el, int k, const float* v) {
    const uint32_t off = umma_a_off<Op>(el, k, M);
#pragma unroll
    for (int c = 0; c < NC; ++c) Op::put1(sBhi + off + c * CSTRIDE, sBlo + off + c * CSTRIDE, v[c]);
  };
  // bit b: phase parity / copy in flight of tile buffer b (scalars, so they
  // stay in registers)
  uint32_t par = 0u, pend = 0u, mma_parity = 0u;
  bool mma_pending = false;
  // One half of K: make the operand writes visible to the tensor-core
  // (async) proxy, let one thread issue nks K-steps (hi*hi + hi*lo + lo*hi)
  // against operator K-steps [ka0, ka0 + nks) (mma_issue), and wait
  // (bounded) until they completed (mma_wait); ka0 == 0 starts the
  // accumulator.  All threads call both.
  auto mma_issue = [&](int ka0, int nks) {
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t ah = smem_u32(sAhi), al = smem_u32(sAlo), bh = smem_u32(sBhi), bl = smem_u32(sBlo);
#pragma unroll 1
      for (int ks = 0; ks < nks; ++ks) {
        const uint32_t oa = uint32_t(ka0 + ks) * KSTEP_A, ob = uint32_t(ks) * KSTEP_B;
        const uint64_t dAh = umma_desc(ah + oa, LBO_A, SBO), dAl = umma_desc(al + oa, LBO_A, SBO);
        const uint64_t dBh = umma_desc(bh + ob, LBO_B, SBO), dBl = umma_desc(bl + ob, LBO_B, SBO);
        Op::mma(tmem, dBh, dAh, IDESC, (ka0 + ks) > 0 ? 1u : 0u);
        Op::mma(tmem, dBh, dAl, IDESC, 1u);
        Op::mma(tmem, dBl, dAh, IDESC, 1u);
      }
      tc_commit(&bar[2]);
    }
    mma_pending = true;
  };
  auto mma_wait = [&]() -> bool {
    if (!block_wait_bounded(&bar[2], mma_parity, kWaitLimitNs)) return false;
    mma_parity ^= 1u;
    mma_pending = false;
    tc_fence_after();
    return true;
  };
  // A tile's state span goes by bulk copy when its start and length are
  // multiples of 16 bytes (always for whole tiles of the usual shapes; the
  // last, partial tile of an odd-sized span takes plain loads).
  auto tile_bulk = [&](int g) -> bool {
    const size_t per_cube = size_t(6) * NP * NC * 4;
    const size_t start = reinterpret_cast<uintptr_t>(tile_qin(g)) + size_t(tile_cell0(g)) * per_cube;
    const size_t bytes = size_t(tile_cells(g)) * per_cube;
    return start % 16 == 0 && bytes % 16 == 0;
  };
  int buf = 0;
  bool failed = !block_wait_bounded(&bar[3], 0, kWaitLimitNs);
  // the set-up above overlaps the previous stage's tail; its output (this
  // stage's q_in / q_a / q_b, and q_out may be a buffer it still reads)
  // only after it has completed
  grid_dep_wait();
  if (t_first < t_end && !failed && tile_bulk(t_first)) {
    if (tid == 0) issue(t_first, 0);
    pend |= 1u;
  }
  const int nwork = BATCH ? (bat.nitems > 0 ? bat.tabs[bat.items[0].x].n_face_work : 0) : tab->n_face_work;
  int cur_member = -1;  // batched: the solve whose arguments and table are loaded
  // ---- per-element constant flux Fbar = F(q at node 0) and the cube-face
  // treatment of tile g (state tile qt): one thread per (element, face); each
  // evaluates the element's flux at node 0 (4x redundant, but the phase's
  // latency is one flux, not four face products); the lf = 0 thread stores
  // Fbar.  The cube-face treatment runs at the same time on threads from
  // NT/2 on.
  auto fbar_phase = [&](int g, const float* qt) {
    const int ncg = tile_cells(g), cg0 = tile_cell0(g);
    for (int w = tid; w < ncg * 24; w += NT) {
      const int el = w >> 2, lf = w & 3, t = el % 6;
      float F[3 * NC];
      ph.flux(&qt[el * NP * NC], F);
      if (lf == 0) {
#pragma unroll
        for (int k = 0; k < 3 * NC; ++k) sF[el * 3 * NC + k] = F[k];
      }
      const float nx = tab->normal[t][lf][0], ny = tab->normal[t][lf][1], nz = tab->normal[t][lf][2];
#pragma unroll
      for (int c = 0; c < NC; ++c) sFn[w * NC + c] = F[c] * nx + F[NC + c] * ny + F[2 * NC + c] * nz;
    }
    for (int w = tid - NT / 2; w >= 0 && w < ncg * 6; w += NT / 2) {
      const int cl = w / 6, dd = w - cl * 6;
      cube_dirs3(cg0 + cl, args.nx, args.ny, args.nz, args.bc, sNb + cl * 6, sMd + cl * 6, dd);
    }
  };
  // With two state buffers the next tile's copy lands while this tile is
  // computed; its Fbar phase then runs while this tile's face MMAs do
  // (fb_ready: sF, sFn, sNb, sMd and the tile wait are done for grp).
  bool fb_ready = false;

  for (int grp = t_first; grp < t_end && !failed; grp = next_tile(grp), buf ^= (S::QB - 1)) {
    if constexpr (BATCH) {  // a new solve: its arguments, table and face records
      const int m = tile_member(grp);
      if (m != cur_member) {
        __syncthreads();  // every thread is done with the previous solve's tile
        {
          const int* src = reinterpret_cast<const int*>(&bat.margs[m]);
          int* dst = reinterpret_cast<int*>(sArgs);
          for (int k = tid; k < int(sizeof(Stage3DArgs<float>) / 4); k += NT) dst[k] = src[k];
        }
        load_table(bat.tabs[m]);
        __syncthreads();
        cur_member = m;
      }
    }
    const int cell0 = tile_cell0(grp);
    const int nc_here = tile_cells(grp);
    const int ne_here = 6 * nc_here;
    float* q = sQ + buf * QV;
    if (fb_ready) {
      __syncthreads();  // every thread is done with the previous tile (its buffer, sO)
      if (S::QB == 2 && next_tile(grp) < ngroups && tile_bulk(next_tile(grp))) {
        if (tid == 0) issue(next_tile(grp), buf ^ 1);
        pend |= 1u << (buf ^ 1);
      }
    } else if (tile_bulk(grp)) {
      if (S::QB == 1 && grp != t_first) {  // single buffer: load this tile now
        __syncthreads();                            // every thread is done with the previous tile
        if (tid == 0) issue(grp, 0);
        pend |= 1u;
      }
      if (!block_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs)) {
        failed = true;
        break;
      }
      par ^= 1u << buf;
      pend &= ~(1u << buf);
      if (S::QB == 2 && next_tile(grp) < ngroups && tile_bulk(next_tile(grp))) {
        if (tid == 0) issue(next_tile(grp), buf ^ 1);
        pend |= 1u << (buf ^ 1);
      }
    } else {
      // plain loads; with one buffer, every thread must be done with the
      // previous tile first
      if (S::QB == 1) __syncthreads();
      const float* src = args.q_in + size_t(cell0) * 6 * NP * NC;
      for (int idx = tid; idx < ne_here * NP * NC; idx += NT) q[idx] = src[idx];
      __syncthreads();
    }
    if (!fb_ready) {
      fbar_phase(grp, q);
      __syncthreads();
    }
    // ---- volume fluxes (F - Fbar) in reference coordinates -> k = d*NP + j
    // Up to five components, each thread takes two neighbouring elements
    // (rows el, el + 1) at one node: their operand values share a 4-byte
    // word of the MN-major tile, so each hi / lo pair is one packed
    // conversion and one 32-bit store.  Six components (36 flux values per
    // pair) take one element per thread.
    if constexpr (NC > 5) {
      for (int idx = tid; idx < EBP * NP; idx += NT) {
        const int el8 = idx & 7, rest = idx >> 3, j = rest % NP, el = (rest / NP) * 8 + el8;
        if (el >= ne_here) continue;
        const int t = el % 6;
        float F[3 * NC];
        ph.flux(&q[(el * NP + j) * NC], F);
        const float* Fb = &sF[el * 3 * NC];
#pragma unroll
        for (int k = 0; k < 3 * NC; ++k) F[k] -= Fb[k];
        const float* iJ = tab->invJ[t];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          float v[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c)
            v[c] = iJ[d * 3 + 0] * F[c] + iJ[d * 3 + 1] * F[NC + c] + iJ[d * 3 + 2] * F[2 * NC + c];
          put(el, d * NP + j, v);
        }
      }
    } else
    for (int idx = tid; idx < (EBP / 2) * NP; idx += NT) {
      const int e4 = idx & 3, rest = idx >> 2, j = rest % NP, el = (rest / NP) * 8 + 2 * e4;
      if (el >= ne_here) continue;  // ne_here is even: el + 1 is in the tile too
      const int t0 = el % 6, t1 = t0 + 1;  // el even: t0 in {0, 2, 4}
      float Fa[3 * NC], Fb[3 * NC];
      ph.flux(&q[(el * NP + j) * NC], Fa);
      ph.flux(&q[((el + 1) * NP + j) * NC], Fb);
      const float* Fba = &sF[el * 3 * NC];
#pragma unroll
      for (int k = 0; k < 3 * NC; ++k) {
        Fa[k] -= Fba[k];
        Fb[k] -= Fba[3 * NC + k];
      }
      const float* iJa = tab->invJ[t0];
      const float* iJb = tab->invJ[t1];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const uint32_t off = umma_a_off<Op>(el, d * NP + j, M);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float va = iJa[d * 3 + 0] * Fa[c] + iJa[d * 3 + 1] * Fa[NC + c] + iJa[d * 3 + 2] * Fa[2 * NC + c];
          const float vb = iJb[d * 3 + 0] * Fb[c] + iJb[d * 3 + 1] * Fb[NC + c] + iJb[d * 3 + 2] * Fb[2 * NC + c];
          if constexpr (Op::A_MN) {
            Op::put2(sBhi + off + c * CSTRIDE, sBlo + off + c * CSTRIDE, va, vb);
          } else {  // K-major: row el + 1 lies 16 bytes on, in the same core matrix (el even)
            Op::put1(sBhi + off + c * CSTRIDE, sBlo + off + c * CSTRIDE, va);
            Op::put1(sBhi + off + 16 + c * CSTRIDE, sBlo + off + 16 + c * CSTRIDE, vb);
          }
        }
      }
    }
    // ---- face fluxes: (f - Fbar.n) * side*area/(6V) -> operand column lf*NFP + m
    //      (operator column KV + lf*NFP + m), into the same operand buffer.
    // face_item evaluates work item idx into up to two operand entries
    // (element, column, NC values); it returns how many (0: nothing to do).
    auto face_item = [&](int idx, int& e1, int& k1, float* v1, int& e2, int& k2, float* v2) -> int {
      const int cl = idx % EC, rest = idx / EC, m = rest % NFP, wk = rest / NFP;
      if (cl >= nc_here) return 0;
      int t, lf, nbt, ax, own_n, bits = 0, nm = 0;
      bool own_left;
      float nx, ny, nz, scale, s2r = 0.f;
      if constexpr (S::FREC) {
        const float4 fr = *reinterpret_cast<const float4*>(sFR + wk * 8);
        const float2 fr2 = *reinterpret_cast<const float2*>(sFR + wk * 8 + 4);
        bits = __float_as_int(fr2.y);
        nm = sFM[wk * NFP + m];
        t = bits & 7, lf = (bits >> 3) & 3, nbt = (bits >> 5) & 7, ax = ((bits >> 10) & 3) - 1;
        own_left = (bits >> 13) & 1;
        own_n = nm & 255;
        nx = fr.x, ny = fr.y, nz = fr.z, scale = fr.w, s2r = fr2.x;
      } else {
        const int tl = tab->face_work[wk];
        t = tl >> 2, lf = tl & 3;
        ax = tab->axis[t][lf];
        own_left = tab->side[t][lf] == 0;
        nbt = tab->nb_t[t][lf];
        own_n = tab->own_node[lf][m];
        nx = tab->normal[t][lf][0], ny = tab->normal[t][lf][1], nz = tab->normal[t][lf][2];
        scale = tab->fscale[t][lf];
      }
      const int el = cl * 6 + t;
      int mode = FACE_INTERIOR, code = 0, nbcube = 0;
      if (ax >= 0) {
        const int dd = 2 * ax + (S::FREC ? ((bits >> 12) & 1) : (tab->dir[t][lf] > 0 ? 1 : 0));
        const int md = sMd[cl * 6 + dd];
        mode = md & 0xff;
        code = md >> 8;
        nbcube = sNb[cl * 6 + dd];
      }
      const float* qo = &q[(el * NP + own_n) * NC];
      float qn[NC], qg[NC];
      if (mode == FACE_INTERIOR || mode == FACE_MIXED) {
        const int nbn = S::FREC ? (nm >> 8) & 255 : int(tab->nb_node[t][lf][m]);
        if (ax < 0) {
#pragma unroll
          for (int c = 0; c < NC; ++c) qn[c] = q[((cl * 6 + nbt) * NP + nbn) * NC + c];
        } else {
          const float* gq = args.q_in + ((size_t(nbcube) * 6 + nbt) * NP + nbn) * NC;
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
        nz = -nz;
        scale = -scale;
      }
      const bool bcf = mode != FACE_INTERIOR;
      if (bcf) ph.ghost(qn, code, nx, ny, nz, qg);
      // left/right states by value (selecting between pointers would force
      // the register arrays into local memory)
      float L[NC], Rr[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float o = qo[c];
        L[c] = bcf ? qn[c] : (own_left ? o : qn[c]);
        Rr[c] = bcf ? qg[c] : (own_left ? qn[c] : o);
      }
      float f[NC];
      ph.num_flux(L, Rr, nx, ny, nz, f);
      // Fbar . n was taken with the table normal; a one-sided low face flips it
      const float* Fn = &sFn[(el * 4 + lf) * NC];
      const float sg = mode == FACE_BC_LO ? -1.f : 1.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) v1[c] = scale * (f[c] - sg * Fn[c]);
      e1 = el;
      k1 = lf * NFP + m;
      if (ax >= 0) return 1;
      // the other tet of this inner face: same flux and normal, its own scale and Fbar
      const int el2 = cl * 6 + nbt, lf2 = S::FREC ? (bits >> 8) & 3 : int(tab->nb_lf[t][lf]);
      const float s2 = S::FREC ? s2r : tab->fscale[nbt][lf2];
      const float* Fn2 = &sFn[(el2 * 4 + lf2) * NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) v2[c] = s2 * (f[c] - Fn2[c]);
      e2 = el2;
      k2 = lf2 * NFP + (S::FREC ? (nm >> 16) : int(tab->nb_m[t][lf][m]));
      return 2;
    };
    const int nface_items = EC * nwork * NFP;
    // volume half of K: operand columns [0, KV) against operator columns
    // [0, KV).  While those MMAs run, each thread evaluates its first face
    // item into registers; the operand columns are overwritten only after
    // the MMAs completed.
    mma_issue(0, KV / Op::KSTEP);
    int e1 = 0, k1 = 0, e2 = 0, k2 = 0;
    float v1[NC], v2[NC];
    const int nfirst = tid < nface_items ? face_item(tid, e1, k1, v1, e2, k2, v2) : 0;
    if (!mma_wait()) {
      failed = true;
      break;
    }
    if (nfirst >= 1) put(e1, k1, v1);
    if (nfirst == 2) put(e2, k2, v2);
    for (int idx = tid + NT; idx < nface_items; idx += NT) {
      const int n = face_item(idx, e1, k1, v1, e2, k2, v2);
      if (n >= 1) put(e1, k1, v1);
      if (n == 2) put(e2, k2, v2);
    }
    // face half of K: operand columns [0, KF) against operator columns [KV, KV + KF)
    mma_issue(KV / Op::KSTEP, KF / Op::KSTEP);
    // while the face MMAs run: the next tile's wait and Fbar phase (its
    // copy was issued a whole tile earlier) ...
    fb_ready = false;
    if (S::QB == 2) {
      // (a tile of another solve waits for the solve's table instead)
      const int nxt = next_tile(grp);
      if (nxt < ngroups && tile_bulk(nxt) && tile_member(nxt) == tile_member(grp)) {
        if (!block_wait_bounded(&bar[buf ^ 1], (par >> (buf ^ 1)) & 1u, kWaitLimitNs)) {
          failed = true;
          break;
        }
        par ^= 1u << (buf ^ 1);
        pend &= ~(1u << (buf ^ 1));
        fbar_phase(nxt, sQ + (buf ^ 1) * QV);
        fb_ready = true;
      }
    }
    // ... and q_a of this thread's first epilogue node (global memory when
    // q_a is not the tile's own state)
    const bool a_in = args.q_a == args.q_in, b_in = args.q_b == args.q_in;
    const bool pre_a = !args.rhs_only && !a_in && tid < ne_here * NP;
    float pa[NC];
    if (pre_a) {
      const size_t base = (size_t(cell0) * 6 * NP + tid) * NC;
#pragma unroll
      for (int c = 0; c < NC; ++c) pa[c] = args.q_a[base + c];
    }
    if (!mma_wait()) {
      failed = true;
      break;
    }
    {  // warp w reads TMEM lanes [32 (w % 4), +32) (rows (c, el)), columns
       // [16 (w / 4), +16) of every 16 (NT / 128) (16 at a time: bounded
       // registers)
      const int row = (warp & 3) * 32 + lane;
#pragma unroll
      for (int c0 = (warp >> 2) * 16; c0 < NN; c0 += 16 * (NT / 128)) {
        float v[16];
        tmem_ld16(tmem + (uint32_t((warp & 3) * 32) << 16) + c0, v);
        tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (c0 + i < NP) sO[row * NPO + c0 + i] = v[i];
      }
    }
    tc_fence_before();
    __syncthreads();
    // ---- epilogue per node: source, RK combine, floor, store
    for (int idx = tid; idx < ne_here * NP; idx += NT) {
      const int el = idx / NP, i = idx - el * NP;
      const size_t base = (size_t(cell0) * 6 * NP + idx) * NC;
      const float* ql = &q[idx * NC];
      float src[NC], out[NC];
      if (Phys::kSource) ph.source(ql, src);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float r = sO[(c * EBP + el) * NPO + i];
        const float rhs = Phys::kSource ? r + src[c] : r;
        if (args.rhs_only) {
          out[c] = rhs;
        } else {
          const float va = a_in ? ql[c] : (pre_a && idx == tid ? pa[c] : args.q_a[base + c]);
          const float vb = b_in ? ql[c] : args.q_b[base + c];
          out[c] = va + args.b * (vb - va) + args.cdt * rhs;
        }
      }
      if (Phys::kLimit && !args.rhs_only) ph.limit(out);
#pragma unroll
      for (int c = 0; c < NC; ++c) args.q_out[base + c] = out[c];
    }
  }
  if (failed) {
    // (batched: every solve's arguments carry the batch's error word; the
    // shared copy may not be loaded yet when the operator image wait gave up)
    int* errp = BATCH ? (bat.nitems > 0 ? bat.margs[bat.items[0].x].err : nullptr) : args0.err;
    if (tid == 0 && errp) atomicOr(errp, 2);
    // let copies and the MMA batch still in flight land before the shared
    // tiles and the accumulator are released (each wait bounded)
    if (tid == 0) {
      for (int b = 0; b < 2; ++b)
        if ((pend >> b) & 1u) mbar_wait_bounded(&bar[b], (par >> b) & 1u, kWaitLimitNs);
      if (mma_pending) mbar_wait_bounded(&bar[2], mma_parity, kWaitLimitNs);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, S::NCOLS);
}

}  // namespace mxm
