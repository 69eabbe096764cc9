// Batched 2D DG: many independent solves of uneven mesh size and order P in
// one persistent stage launch.
//
// Work is a list of items (solve, first cell, cells, P), one tile of whole
// cells each; the tile size per P comes from the autotuner.  Blocks take
// items from a global counter (dynamic scheduling, so big-P tiles do not
// leave blocks idle at the end), prefetch the next item's state span with a
// bulk copy into the other half of a double-buffered shared tile, and run the
// same per-tile code as the single-solve kernel (stage2d_tile) instantiated
// for P = 1..5 behind a switch.  The five shared operators live in shared
// memory for the launch.  Each solve carries its own topology/metric table,
// state buffers, time step and boundary codes (SolveDesc2).
//
// The SSPRK3 routing is the reference's (src/ssprk3.mojo:56-78): stage 0
// q -> q1 (1, 0, 1), stage 1 q1 -> q2 (3/4, 1/4, 1/4), stage 2 q2 -> q
// (1/3, 2/3, 2/3).  The limiter passes (cell means, theta + apply, as in
// src/local_mesh_2d_gpu_limiter.mojo:74-210 and
// src/local_mesh_2d_gpu.mojo:180-198) run over the limited solves' element
// chunks, one block per chunk.
#pragma once
#include "limiter.cuh"
#include "stage2d.cuh"

namespace mxm {

template <class R>
struct SolveDesc2 {
  KuhnTab2<R> tab;
  R* q[3];
  R* avg;
  const R* w;
  R cdt[3];  // c dt of the three SSPRK3 stages, rounded once from FP64
  R eps2;
  int P, nx, ny, ncell;
  int bc[4];
  int limiter;
  int pad;
};

template <class R>
struct Batch2DArgs {
  const SolveDesc2<R>* solves;
  const int4* items;  // {solve, first cell, cells, P}
  int nitems;
  int* counter;       // work counter, zero before the launch
  int stage;          // SSPRK3 stage 0..2
  const R* A[6];      // shared operator [K][NP] per P (index P)
  int aoff[6];        // element offset of each P's operator in the shared copy
  int a_len;          // values of all operators, a multiple of 4
  int qv;             // values per tile buffer, a multiple of 4
  int* err;
};

template <int P, int NC, class R>
__host__ __device__ constexpr bool bulk2d_ok() {
  return (2 * ntri(P) * NC * sizeof(R)) % 16 == 0;
}

template <class R, int NC>
__device__ __forceinline__ bool bulk2d(int P) {
  switch (P) {
    case 1: return bulk2d_ok<1, NC, R>();
    case 2: return bulk2d_ok<2, NC, R>();
    case 3: return bulk2d_ok<3, NC, R>();
    case 4: return bulk2d_ok<4, NC, R>();
    default: return bulk2d_ok<5, NC, R>();
  }
}

template <class R>
__device__ __forceinline__ void ssprk3_route(int stage, R* const* q, const R*& qi, const R*& qa, const R*& qb,
                                             R*& qo, R& b) {
  if (stage == 0) {
    qi = q[0]; qa = q[0]; qb = q[0]; qo = q[1];
    b = R(0);
  } else if (stage == 1) {
    qi = q[1]; qa = q[0]; qb = q[1]; qo = q[2];
    b = R(0.25);
  } else {
    qi = q[2]; qa = q[0]; qb = q[2]; qo = q[0];
    b = R(2.0 / 3.0);
  }
}

template <class R, class Phys, int NT>
__global__ void __launch_bounds__(NT) stage2d_batch_kernel(Batch2DArgs<R> ba, Phys ph) {
  constexpr int NC = Phys::NC;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);          // [2]
  int* sIt = reinterpret_cast<int*>(smem_raw + 16);               // [2] item of each tile buffer
  constexpr size_t kTabBytes = (sizeof(KuhnTab2<R>) + 15) / 16 * 16;
  KuhnTab2<R>* tabs = reinterpret_cast<KuhnTab2<R>*>(smem_raw + 32);  // [2]
  R* sA = reinterpret_cast<R*>(smem_raw + 32 + 2 * kTabBytes);  // operators of P = 1..5
  R* sQ = sA + ba.a_len;                                          // [2][qv], 16-byte aligned
  R* sB = sQ + 2 * size_t(ba.qv);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  for (int P = 1; P <= 5; ++P) {
    const int n = (2 * ntri(P) + 3 * (P + 1)) * ntri(P);
    if (ba.A[P])
      for (int idx = tid; idx < n; idx += NT) sA[ba.aoff[P] + idx] = ba.A[P][idx];
  }
  auto issue = [&](int it, int b) {
    const int4 item = ba.items[it];
    const int np = ntri(item.w);
    const uint32_t bytes = uint32_t(item.z) * 2u * np * NC * sizeof(R);
    const R* src = ba.solves[item.x].q[ba.stage] + size_t(item.y) * 2 * np * NC;  // stage s reads q_s
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[b], bytes);
    bulk_g2s(sQ + size_t(b) * ba.qv, src, bytes, &bar[b]);
    // stages 1 and 2 combine with q (the step's start state): that span of
    // the item into L2 an item ahead of its epilogue
    if (ba.stage > 0) bulk_prefetch_l2(ba.solves[item.x].q[0] + size_t(item.y) * 2 * np * NC, bytes);
  };
  if (tid == 0) {
    const int it = atomicAdd(ba.counter, 1);
    sIt[0] = it;
    if (it < ba.nitems && bulk2d<R, NC>(ba.items[it].w)) issue(it, 0);
  }
  __syncthreads();
  uint32_t par = 0u;  // bit b: phase parity of tile buffer b
  int buf = 0;
  while (true) {
    const int it = sIt[buf];
    if (it >= ba.nitems) break;
    const int4 item = ba.items[it];
    const SolveDesc2<R>* sd = &ba.solves[item.x];
    const int P = item.w, np = ntri(P);
    {  // this solve's table into the buffer's table slot
      const int* src = reinterpret_cast<const int*>(&sd->tab);
      int* dst = reinterpret_cast<int*>(&tabs[buf]);
      for (int k = tid; k < int(sizeof(KuhnTab2<R>) / 4); k += NT) dst[k] = src[k];
    }
    R* q = sQ + size_t(buf) * ba.qv;
    const bool bulk = bulk2d<R, NC>(P);
    if (bulk) {
      if (!block_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs2)) {
        if (tid == 0) {
          if (ba.err) atomicOr(ba.err, 1);
          mbar_wait_bounded(&bar[buf], (par >> buf) & 1u, kWaitLimitNs2);
        }
        return;
      }
      par ^= 1u << buf;
    } else {
      const R* src = sd->q[ba.stage] + size_t(item.y) * 2 * np * NC;
      for (int idx = tid; idx < item.z * 2 * np * NC; idx += NT) q[idx] = src[idx];
      __syncthreads();
    }
    if (tid == 0) {  // next item into the other buffer (its previous tile is finished)
      const int nx = atomicAdd(ba.counter, 1);
      sIt[buf ^ 1] = nx;
      if (nx < ba.nitems && bulk2d<R, NC>(ba.items[nx].w)) issue(nx, buf ^ 1);
    }
    Stage2DArgs<R> args;
    R b;
    ssprk3_route(ba.stage, sd->q, args.q_in, args.q_a, args.q_b, args.q_out, b);
    args.A = nullptr;
    args.b = b;
    args.cdt = sd->cdt[ba.stage];
    args.nx = sd->nx;
    args.ny = sd->ny;
    args.ncell = sd->ncell;
    for (int k = 0; k < 4; ++k) args.bc[k] = sd->bc[k];
    args.rhs_only = 0;
    args.err = ba.err;
    const int ne_here = 2 * item.z;
    switch (P) {
      case 1: stage2d_tile<R, Phys, 1, NT>(args, &tabs[buf], ph, q, sB, sA + ba.aoff[1], item.y, ne_here); break;
      case 2: stage2d_tile<R, Phys, 2, NT>(args, &tabs[buf], ph, q, sB, sA + ba.aoff[2], item.y, ne_here); break;
      case 3: stage2d_tile<R, Phys, 3, NT>(args, &tabs[buf], ph, q, sB, sA + ba.aoff[3], item.y, ne_here); break;
      case 4: stage2d_tile<R, Phys, 4, NT>(args, &tabs[buf], ph, q, sB, sA + ba.aoff[4], item.y, ne_here); break;
      default: stage2d_tile<R, Phys, 5, NT>(args, &tabs[buf], ph, q, sB, sA + ba.aoff[5], item.y, ne_here); break;
    }
    buf ^= 1;
  }
}

// ---- batched limiter passes over element chunks of the limited solves
template <class R>
struct LimBatch2DArgs {
  const SolveDesc2<R>* solves;
  const int4* items;  // {solve, first element, elements, P}
  int nitems;
  int which;          // state buffer to limit (0..2)
};

template <class R, int NP, int NC>
__device__ __forceinline__ void avg_chunk(const SolveDesc2<R>* sd, int which, int e0, int ne) {
  const R* qb = sd->q[which];
  R* ext = sd->avg + int64_t(2) * sd->ncell * NC;  // component 0's nodal extrema
  for (int idx = threadIdx.x; idx < ne * NC; idx += blockDim.x) {
    const int64_t e = e0 + idx / NC;
    const int c = idx % NC;
    const R* q = qb + e * NP * NC + c;
    R s = R(0), lo = q[0], hi = q[0];
#pragma unroll
    for (int n = 0; n < NP; ++n) {
      const R v = q[n * NC];
      s = fma(__ldg(&sd->w[n]), v, s);
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    }
    sd->avg[e * NC + c] = s;
    if (c == 0) {
      ext[e * 2] = lo;
      ext[e * 2 + 1] = hi;
    }
  }
}

template <class R, int NC>
__global__ void avg_batch_kernel(LimBatch2DArgs<R> la) {
  const int4 item = la.items[blockIdx.x];
  const SolveDesc2<R>* sd = &la.solves[item.x];
  switch (item.w) {
    case 1: avg_chunk<R, ntri(1), NC>(sd, la.which, item.y, item.z); break;
    case 2: avg_chunk<R, ntri(2), NC>(sd, la.which, item.y, item.z); break;
    case 3: avg_chunk<R, ntri(3), NC>(sd, la.which, item.y, item.z); break;
    case 4: avg_chunk<R, ntri(4), NC>(sd, la.which, item.y, item.z); break;
    default: avg_chunk<R, ntri(5), NC>(sd, la.which, item.y, item.z); break;
  }
}

// Theta + apply of one chunk (blocks of kLim2dBlock threads, chunks of at
// most kLim2dBlock elements): the single-solve limiter's staged block
// function on this solve's buffers and table.  Dynamic shared memory sized
// for P = 5.
template <class R, int NC>
__global__ void __launch_bounds__(kLim2dBlock) theta_batch_kernel(LimBatch2DArgs<R> la) {
  extern __shared__ __align__(16) unsigned char lim_smem[];
  const int4 item = la.items[blockIdx.x];
  const SolveDesc2<R>* sd = &la.solves[item.x];
  R* q = sd->q[la.which];
  const R* ext = sd->avg + int64_t(2) * sd->ncell * NC;
  switch (item.w) {
    case 1: theta2d_block<R, ntri(1), NC>(q, sd->avg, ext, item.y, item.z, sd->tab, sd->nx, sd->ny, sd->bc, sd->eps2, lim_smem); break;
    case 2: theta2d_block<R, ntri(2), NC>(q, sd->avg, ext, item.y, item.z, sd->tab, sd->nx, sd->ny, sd->bc, sd->eps2, lim_smem); break;
    case 3: theta2d_block<R, ntri(3), NC>(q, sd->avg, ext, item.y, item.z, sd->tab, sd->nx, sd->ny, sd->bc, sd->eps2, lim_smem); break;
    case 4: theta2d_block<R, ntri(4), NC>(q, sd->avg, ext, item.y, item.z, sd->tab, sd->nx, sd->ny, sd->bc, sd->eps2, lim_smem); break;
    default: theta2d_block<R, ntri(5), NC>(q, sd->avg, ext, item.y, item.z, sd->tab, sd->nx, sd->ny, sd->bc, sd->eps2, lim_smem); break;
  }
}

}  // namespace mxm
