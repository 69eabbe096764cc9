// Barth-Jespersen / Venkatakrishnan cell limiter and FP64 diagnostics.
//
// Reference: compute_cell_averages_kernel, bj_limiter_compute_theta_kernel,
// bj_limiter_apply_kernel (src/solver.mojo:384-530) for 3D -- theta over
// every node and component, neighbour set = self + 4 face neighbours with BC
// faces resolving to self; and cell_mean_kernel_2d +
// bj_limit_{compute_theta,apply}_kernel_2d (src/local_mesh_2d_gpu.mojo:180-198,
// src/local_mesh_2d_gpu_limiter.mojo:74-153) for 2D -- theta from component 0
// only, BC self-neighbours skipped, applied to every component.
//
// B200 form: pass 1 computes cell means with one thread per (element,
// component) over coalesced loads, and beside each mean of a component that
// enters theta the least and the largest of its nodal values; pass 2 gets
// theta from those extrema and the neighbours' means without reading the
// nodal state, and reads and rewrites the values of the elements with
// theta < 1 only (3D: a warp per element; 2D: a block per chunk of
// elements, theta2d_block).
//
// Why the extrema suffice: the ratio alpha(d) = (D^2 + 2 D d + eps^2) /
// (D^2 + 2 d^2 + D d + eps^2) of a node with deviation magnitude d from the
// mean (D the neighbours' bound on that side) is 1 at d = 0, rises to a
// single maximum and then falls (the numerator of its derivative, D^3 + D
// eps^2 - 4 D d^2 - 4 D^2 d - 4 d eps^2, is positive at d = 0 and
// decreasing in d).  So over the nodes of one side it is >= 1 before its
// crossing of 1 and decreasing after it, and min(1, min over the side's
// nodes) is min(1, alpha at the side's largest deviation); d = u - mean is
// monotone in u (also in floating point), so that node is the one with the
// largest (or, below the mean, the least) value.  theta is then the
// reference's minimum over every node, up to the rounding of alpha at
// near-equal deviations.
//
// Extrema layout: ext = avg + ne * NC, ext[(e * NCT + c) * 2 + {0, 1}] =
// {least, largest} nodal value of component c of element e, for the NCT
// components that enter theta (every component in 3D, component 0 in 2D).
#pragma once
#include "dg_common.cuh"

namespace mxm {

template <class R, int NP, int NC>
__global__ void cell_avg_kernel(LimArgs<R> a) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= a.ne * NC) return;
  const int64_t e = tid / NC;
  const int c = int(tid - e * NC);
  const R* q = a.q + e * NP * NC + c;
  R s = R(0);
#pragma unroll
  for (int n = 0; n < NP; ++n) s = fma(__ldg(&a.w[n]), q[n * NC], s);
  a.avg[tid] = s;
}

template <class R, int NP, int NC, int NCT>
__global__ void cell_avg_kernel(LimArgs<R> a) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= a.ne * NC) return;
  const int64_t e = tid / NC;
  const int c = int(tid - e * NC);
  const R* q = a.q + e * NP * NC + c;
  R s = R(0), lo = q[0], hi = q[0];
#pragma unroll
  for (int n = 0; n < NP; ++n) {
    const R v = q[n * NC];
    s = fma(__ldg(&a.w[n]), v, s);
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  a.avg[tid] = s;
  if (c < NCT) {
    R* x = a.avg + a.ne * NC + (e * NCT + c) * 2;
    x[0] = lo;
    x[1] = hi;
  }
}

// min(1, alpha at the largest deviation above and below the mean): theta
// of one component from its mean `own`, the neighbours' bounds lo / hi and
// the element's least / largest nodal value.  Deviations of magnitude
// <= 1e-30 do not constrain, as in the reference.
template <class R>
__device__ __forceinline__ R theta_from_extrema(R own, R lo, R hi, R umin, R umax, R eps2) {
  const R tiny = R(1.0e-30);
  R th = R(1);
  R pD = hi - own;
  if (pD < R(0)) pD = R(0);
  R nD = own - lo;
  if (nD < R(0)) nD = R(0);
  const R dp = umax - own;
  if (dp > tiny) {
    const R D2 = pD * pD, d2 = dp * dp, Dd = pD * dp;
    const R al = (D2 + R(2) * Dd + eps2) / (D2 + R(2) * d2 + Dd + eps2);
    if (al < th) th = al;
  }
  const R dn = own - umin;
  if (dn > tiny) {
    const R D2 = nD * nD, d2 = dn * dn, Dd = nD * dn;
    const R al = (D2 + R(2) * Dd + eps2) / (D2 + R(2) * d2 + Dd + eps2);
    if (al < th) th = al;
  }
  return th;
}

// Theta + apply of element e (< a.e1) by one warp; every lane of the warp
// calls it with the same e.
template <class R, int DIM, int NP, int NC>
__device__ __forceinline__ void theta_apply_elem(const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2,
                                                 int64_t e) {
  constexpr int NTYPE = DIM == 3 ? 6 : 2, NFACE = DIM + 1, VALS = NP * NC;
  constexpr int NCT = DIM == 3 ? NC : 1;  // components entering theta
  const int lane = threadIdx.x & 31;
  const int t = int(e % NTYPE);
  const int64_t cell = e / NTYPE;
  int cpos[3];
  if (DIM == 3) {
    const int64_t nxy = int64_t(a.nx) * a.ny;
    cpos[2] = int(cell / nxy);
    const int64_t rem = cell - int64_t(cpos[2]) * nxy;
    cpos[1] = int(rem / a.nx);
    cpos[0] = int(rem - int64_t(cpos[1]) * a.nx);
  } else {
    cpos[1] = int(cell / a.nx);
    cpos[0] = int(cell - int64_t(cpos[1]) * a.nx);
    cpos[2] = 0;
  }
  const int ncells[3] = {a.nx, a.ny, a.nz};
  // neighbour elements: lanes 0..NFACE-1 each resolve one face
  int64_t nb = e;
  if (lane < NFACE) {
    const int lf = lane;
    const int ax = DIM == 3 ? t3.axis[t][lf] : t2.axis[t][lf];
    const int dir = DIM == 3 ? t3.dir[t][lf] : t2.dir[t][lf];
    int code;
    const int mode = face_mode(ax, dir, ax >= 0 ? cpos[ax] : 0, ax >= 0 ? ncells[ax] : 1, a.bc, code);
    if (mode == FACE_INTERIOR || mode == FACE_MIXED) {
      if (DIM == 3) {
        const int ni = wrapi(cpos[0] + t3.off[t][lf][0], a.nx), nj = wrapi(cpos[1] + t3.off[t][lf][1], a.ny),
                  nk = wrapi(cpos[2] + t3.off[t][lf][2], a.nz);
        nb = (int64_t(ni) + int64_t(a.nx) * (nj + int64_t(a.ny) * nk)) * 6 + t3.nb_t[t][lf];
      } else {
        const int ni = wrapi(cpos[0] + t2.off[t][lf][0], a.nx), nj = wrapi(cpos[1] + t2.off[t][lf][1], a.ny);
        nb = (int64_t(nj) * a.nx + ni) * 2 + t2.nb_t[t][lf];
      }
    }
  }
  int64_t nbs[NFACE];
#pragma unroll
  for (int lf = 0; lf < NFACE; ++lf) nbs[lf] = __shfl_sync(0xffffffffu, nb, lf);
  // lane c < NCT: theta of component c
  R th = R(1);
  if (lane < NCT) {
    const int c = lane;
    const R own = a.avg[e * NC + c];
    R lo = own, hi = own;
#pragma unroll
    for (int lf = 0; lf < NFACE; ++lf) {
      if (DIM == 2 && nbs[lf] == e) continue;  // 2D: BC faces do not constrain
      const R v = a.avg[nbs[lf] * NC + c];
      if (v < lo) lo = v;
      if (v > hi) hi = v;
    }
    const R* x = a.avg + a.ne * NC + (e * NCT + c) * 2;
    th = theta_from_extrema(own, lo, hi, x[0], x[1], a.eps2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R v = __shfl_xor_sync(0xffffffffu, th, o);
    th = v < th ? v : th;
  }
  if (!(th < R(1))) return;
  R* qe = a.q + e * VALS;
  for (int idx = lane; idx < VALS; idx += 32) {
    const int c = idx % NC;
    const R bm = a.avg[e * NC + c];
    qe[idx] = bm + th * (qe[idx] - bm);
  }
}

// One warp per element; EPB elements per block of 32*EPB threads.
template <class R, int DIM, int NP, int NC, int EPB>
__global__ void __launch_bounds__(32 * EPB) theta_apply_kernel(LimArgs<R> a, KuhnTab3<R> t3, KuhnTab2<R> t2) {
  const int64_t e = a.e0 + int64_t(blockIdx.x) * EPB + (threadIdx.x >> 5);
  if (e < a.e1) theta_apply_elem<R, DIM, NP, NC>(a, t3, t2, e);
}

// ---- batched 3D limiter: the cell-mean and theta passes of many limited
// solves (any order) in one launch each, over chunks of elements.
template <class R>
struct LimDesc3 {
  LimArgs<R> a;  // q unused: the buffer is qs[which]
  R* qs[3];
  KuhnTab3<R> tab;
  int P;
};
template <class R>
struct LimBatch3 {
  const LimDesc3<R>* solves;
  const int4* items;  // {solve, first element, elements, 0}
  int nitems, which;
};
constexpr int kLim3Chunk = 128, kLim3Epb = 8;

template <class R, int NP, int NC>
__device__ __forceinline__ void avg3d_chunk(const LimDesc3<R>& d, R* q, int64_t e0, int ne) {
  R* ext = d.a.avg + d.a.ne * NC;
  for (int idx = threadIdx.x; idx < ne * NC; idx += blockDim.x) {
    const int64_t e = e0 + idx / NC;
    const int c = idx % NC;
    const R* qe = q + e * NP * NC + c;
    R s = R(0), lo = qe[0], hi = qe[0];
#pragma unroll
    for (int n = 0; n < NP; ++n) {
      const R v = qe[n * NC];
      s = fma(__ldg(&d.a.w[n]), v, s);
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    }
    d.a.avg[e * NC + c] = s;
    ext[(e * NC + c) * 2] = lo;
    ext[(e * NC + c) * 2 + 1] = hi;
  }
}

template <class R, int NC>
__global__ void avg3d_batch_kernel(LimBatch3<R> lb) {
  const int4 it = lb.items[blockIdx.x];
  const LimDesc3<R>& d = lb.solves[it.x];
  R* q = d.qs[lb.which];
  switch (d.P) {
    case 1: avg3d_chunk<R, ntet(1), NC>(d, q, it.y, it.z); break;
    case 2: avg3d_chunk<R, ntet(2), NC>(d, q, it.y, it.z); break;
    case 3: avg3d_chunk<R, ntet(3), NC>(d, q, it.y, it.z); break;
    case 4: avg3d_chunk<R, ntet(4), NC>(d, q, it.y, it.z); break;
    default: avg3d_chunk<R, ntet(5), NC>(d, q, it.y, it.z); break;
  }
}

// The elements of a chunk, one warp each in turn.
template <class R, int NP, int NC>
__device__ __forceinline__ void theta3d_chunk(const LimDesc3<R>& d, R* q, int64_t e0, int ne) {
  LimArgs<R> a = d.a;
  a.q = q;
  a.e1 = e0 + ne;
  for (int g = threadIdx.x >> 5; g < ne; g += kLim3Epb) theta_apply_elem<R, 3, NP, NC>(a, d.tab, KuhnTab2<R>{}, e0 + g);
}

template <class R, int NC>
__global__ void __launch_bounds__(32 * kLim3Epb) theta3d_batch_kernel(LimBatch3<R> lb) {
  const int4 it = lb.items[blockIdx.x];
  const LimDesc3<R>& d = lb.solves[it.x];
  R* q = d.qs[lb.which];
  switch (d.P) {
    case 1: theta3d_chunk<R, ntet(1), NC>(d, q, it.y, it.z); break;
    case 2: theta3d_chunk<R, ntet(2), NC>(d, q, it.y, it.z); break;
    case 3: theta3d_chunk<R, ntet(3), NC>(d, q, it.y, it.z); break;
    case 4: theta3d_chunk<R, ntet(4), NC>(d, q, it.y, it.z); break;
    default: theta3d_chunk<R, ntet(5), NC>(d, q, it.y, it.z); break;
  }
}

// A block of kLim2dBlock threads limits up to kLim2dBlock consecutive
// elements: (1) one thread per element resolves its cell mean and the
// neighbours' bounds (component 0; BC faces skipped) and gets theta from
// the element's nodal extrema of component 0 (theta_from_extrema); (2) one
// thread per value rewrites the values of the elements with theta < 1, over
// consecutive values of the chunk.  The arithmetic is the reference's 2D
// limiter (src/local_mesh_2d_gpu_limiter.mojo:74-153): theta from component
// 0, faces whose neighbour resolves to the element itself (BC faces) do not
// constrain, theta scales every component's deviation from its cell mean.
// `ext` holds the extrema (one theta component).  Dynamic shared memory
// lim2d_smem_bytes<R, NP, NC>().
constexpr int kLim2dBlock = 128;
template <class R, int NP, int NC>
constexpr size_t lim2d_smem_bytes() {
  return size_t(kLim2dBlock) * sizeof(R);
}

template <class R, int NP, int NC>
__device__ __forceinline__ void theta2d_block(R* q, const R* avg, const R* ext, int64_t e0, int ne,
                                              const KuhnTab2<R>& tab, int nx, int ny, const int* bc, R eps2,
                                              unsigned char* smem) {
  constexpr int VALS = NP * NC;
  R* s_th = reinterpret_cast<R*>(smem);
  const int tid = threadIdx.x;
  bool lim = false;
  if (tid < ne) {
    const int64_t e = e0 + tid;
    const int t = int(e & 1);
    const int64_t cell = e >> 1;
    const int cj = int(cell / nx), ci = int(cell - int64_t(cj) * nx);
    const R own = avg[e * NC];
    R lo = own, hi = own;
#pragma unroll
    for (int lf = 0; lf < 3; ++lf) {
      const int ax = tab.axis[t][lf], dir = tab.dir[t][lf];
      int code;
      const int mode = face_mode(ax, dir, ax == 0 ? ci : cj, ax == 0 ? nx : ny, bc, code);
      if (mode != FACE_INTERIOR && mode != FACE_MIXED) continue;
      const int ni = wrapi(ci + tab.off[t][lf][0], nx), nj = wrapi(cj + tab.off[t][lf][1], ny);
      const int64_t nb = (int64_t(nj) * nx + ni) * 2 + tab.nb_t[t][lf];
      if (nb == e) continue;
      const R v = avg[nb * NC];
      if (v < lo) lo = v;
      if (v > hi) hi = v;
    }
    const R th = theta_from_extrema(own, lo, hi, ext[e * 2], ext[e * 2 + 1], eps2);
    s_th[tid] = th;
    lim = th < R(1);
  }
  if (!__syncthreads_or(lim)) return;  // no element of the chunk is limited
  R* base = q + e0 * VALS;
#pragma unroll 4
  for (int idx = tid; idx < ne * VALS; idx += blockDim.x) {
    const int el = idx / VALS;
    const R th = s_th[el];
    if (!(th < R(1))) continue;
    const int c = (idx - el * VALS) % NC;
    const R bm = avg[(e0 + el) * NC + c];
    base[idx] = bm + th * (base[idx] - bm);
  }
}

template <class R, int NP, int NC>
__global__ void __launch_bounds__(kLim2dBlock) theta2d_kernel(LimArgs<R> a, KuhnTab2<R> t2) {
  extern __shared__ __align__(16) unsigned char lim_smem[];
  const int64_t e0 = int64_t(blockIdx.x) * kLim2dBlock;
  const int ne = int(a.ne - e0 < kLim2dBlock ? a.ne - e0 : kLim2dBlock);
  theta2d_block<R, NP, NC>(a.q, a.avg, a.avg + a.ne * NC, e0, ne, t2, a.nx, a.ny, a.bc, a.eps2, lim_smem);
}

// ---- FP64 reductions: per-block partial sums, then a fixed-order final sum.
template <class R, int NP, int NC>
__global__ void reduce_partial_kernel(const R* q, const R* w, int64_t ne, int c, int kind, double* partial) {
  __shared__ double red[32];
  double acc = kind == 2 ? 0.0 : 0.0;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    const R* qe = q + e * NP * NC + c;
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < NP; ++n) {
      const double v = double(qe[n * NC]);
      if (kind == 0) s += double(__ldg(&w[n])) * v;
      else if (kind == 1) s += double(__ldg(&w[n])) * v * v;
      else if (kind == 3) s += v;
      else if (kind == 4) s += v * v;
      else s = fmax(s, fabs(v));
    }
    if (kind == 2) acc = fmax(acc, s);
    else acc += s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, acc, o);
    acc = kind == 2 ? fmax(acc, v) : acc + v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < int(blockDim.x >> 5); ++k) s = kind == 2 ? fmax(s, red[k]) : s + red[k];
    partial[blockIdx.x] = s;
  }
}

__global__ void reduce_final_kernel(const double* partial, int n, int kind, double scale, double* out);

}  // namespace mxm
