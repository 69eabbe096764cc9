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
// component) over coalesced loads; pass 2 (3D) stages a group of elements'
// nodal values in shared memory with contiguous loads, reduces theta per
// element with warp shuffles, and writes the limited values back
// contiguously only for elements with theta < 1; pass 2 (2D) runs
// node-parallel over a chunk of elements (theta2d_block).
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

// Theta + apply of elements eb .. eb + EPB - 1 (those below a.e1), one
// warp per element, in a block of 32*EPB threads; `sqf` is the block's
// staging space of EPB * NP * NC values.  Every thread must call it (it
// synchronises the block once).
template <class R, int DIM, int NP, int NC, int EPB>
__device__ __forceinline__ void theta_apply_group(const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2,
                                                  int64_t eb, R* sqf) {
  constexpr int NTYPE = DIM == 3 ? 6 : 2, NFACE = DIM + 1, VALS = NP * NC;
  R (*sq)[VALS] = reinterpret_cast<R (*)[VALS]>(sqf);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = eb + warp;
  const bool valid = e < a.e1;
  // contiguous block load of the EPB elements
  const int64_t base = eb * VALS;
  const int64_t nvals = (a.e1 - eb) * VALS;
  for (int idx = threadIdx.x; idx < EPB * VALS; idx += 32 * EPB)
    if (idx < nvals) (&sq[0][0])[idx] = a.q[base + idx];
  __syncthreads();
  if (!valid) return;
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
  // neighbour cell means: lanes 0..NFACE-1 each resolve one face
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
  constexpr int NCT = DIM == 3 ? NC : 1;  // components entering theta
  R own[NCT], lo[NCT], hi[NCT];
#pragma unroll
  for (int c = 0; c < NCT; ++c) own[c] = lo[c] = hi[c] = a.avg[e * NC + c];
#pragma unroll
  for (int lf = 0; lf < NFACE; ++lf) {
    const int64_t n = __shfl_sync(0xffffffffu, nb, lf);
    if (DIM == 2 && n == e) continue;  // 2D: BC faces do not constrain
#pragma unroll
    for (int c = 0; c < NCT; ++c) {
      const R v = a.avg[n * NC + c];
      if (v < lo[c]) lo[c] = v;
      if (v > hi[c]) hi[c] = v;
    }
  }
  R th = R(1);
  const R tiny = R(1.0e-30);
  for (int idx = lane; idx < NP * NCT; idx += 32) {
    const int n = idx / NCT, c = idx - n * NCT;
    const R dl = sq[warp][n * NC + c] - own[c];
    const R da = dl >= R(0) ? dl : -dl;
    if (da <= tiny) continue;
    R pD = hi[c] - own[c];
    if (pD < R(0)) pD = R(0);
    R nD = own[c] - lo[c];
    if (nD < R(0)) nD = R(0);
    const R D = dl > R(0) ? pD : nD;
    const R D2 = D * D, d2 = da * da, Dd = D * da;
    const R al = (D2 + R(2) * Dd + a.eps2) / (D2 + R(2) * d2 + Dd + a.eps2);
    if (al < th) th = al;
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
    qe[idx] = bm + th * (sq[warp][idx] - bm);
  }
}

// One warp per element; EPB elements per block of 32*EPB threads.
template <class R, int DIM, int NP, int NC, int EPB>
__global__ void __launch_bounds__(32 * EPB) theta_apply_kernel(LimArgs<R> a, KuhnTab3<R> t3, KuhnTab2<R> t2) {
  __shared__ R sq[EPB * NP * NC];
  theta_apply_group<R, DIM, NP, NC, EPB>(a, t3, t2, a.e0 + int64_t(blockIdx.x) * EPB, sq);
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
  for (int idx = threadIdx.x; idx < ne * NC; idx += blockDim.x) {
    const int64_t e = e0 + idx / NC;
    const int c = idx % NC;
    const R* qe = q + e * NP * NC + c;
    R s = R(0);
#pragma unroll
    for (int n = 0; n < NP; ++n) s = fma(__ldg(&d.a.w[n]), qe[n * NC], s);
    d.a.avg[e * NC + c] = s;
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

template <class R, int NP, int NC>
__device__ __forceinline__ void theta3d_chunk(const LimDesc3<R>& d, R* q, int64_t e0, int ne, R* sq) {
  LimArgs<R> a = d.a;
  a.q = q;
  a.e1 = e0 + ne;
  for (int g = 0; g < ne; g += kLim3Epb) {
    theta_apply_group<R, 3, NP, NC, kLim3Epb>(a, d.tab, KuhnTab2<R>{}, e0 + g, sq);
    __syncthreads();  // the staging space is reused by the next group
  }
}

template <class R, int NC>
__global__ void __launch_bounds__(32 * kLim3Epb) theta3d_batch_kernel(LimBatch3<R> lb) {
  __shared__ R sq[kLim3Epb * ntet(5) * NC];
  const int4 it = lb.items[blockIdx.x];
  const LimDesc3<R>& d = lb.solves[it.x];
  R* q = d.qs[lb.which];
  switch (d.P) {
    case 1: theta3d_chunk<R, ntet(1), NC>(d, q, it.y, it.z, sq); break;
    case 2: theta3d_chunk<R, ntet(2), NC>(d, q, it.y, it.z, sq); break;
    case 3: theta3d_chunk<R, ntet(3), NC>(d, q, it.y, it.z, sq); break;
    case 4: theta3d_chunk<R, ntet(4), NC>(d, q, it.y, it.z, sq); break;
    default: theta3d_chunk<R, ntet(5), NC>(d, q, it.y, it.z, sq); break;
  }
}

// A block of kLim2dBlock threads limits up to kLim2dBlock consecutive
// elements, node-parallel: (1) one thread per element resolves its cell
// mean and the neighbours' bounds (component 0; BC faces skipped); (2) one
// thread per (element, node) evaluates the Barth-Jespersen / Venkatakrishnan
// ratio of its node and folds it into the element's theta with a shared
// atomic minimum on the value's bits (non-negative IEEE values order like
// their unsigned bit patterns, and a minimum is exact in any order, so theta
// equals the reference's sequential minimum bit for bit); (3) one thread per
// value rewrites the values of elements with theta < 1.  Loads and stores
// run over consecutive values of the chunk.  The arithmetic is the
// reference's 2D limiter (src/local_mesh_2d_gpu_limiter.mojo:74-153): theta
// from component 0, faces whose neighbour resolves to the element itself
// (BC faces) do not constrain, theta scales every component's deviation from
// its cell mean.  Dynamic shared memory lim2d_smem_bytes<R, NP, NC>().
constexpr int kLim2dBlock = 128;
template <class R, int NP, int NC>
constexpr size_t lim2d_smem_bytes() {
  return size_t(kLim2dBlock) * (3 * sizeof(R) + sizeof(unsigned long long));
}

template <class R>
struct ThetaBits;  // theta as an unsigned integer of the same width
template <>
struct ThetaBits<float> {
  using U = unsigned int;
  __device__ static U to(float v) { return __float_as_uint(v); }
  __device__ static float from(U u) { return __uint_as_float(u); }
};
template <>
struct ThetaBits<double> {
  using U = unsigned long long;
  __device__ static U to(double v) { return (unsigned long long)__double_as_longlong(v); }
  __device__ static double from(U u) { return __longlong_as_double((long long)u); }
};

template <class R, int NP, int NC>
__device__ __forceinline__ void theta2d_block(R* q, const R* avg, int64_t e0, int ne, const KuhnTab2<R>& tab, int nx,
                                              int ny, const int* bc, R eps2, unsigned char* smem) {
  constexpr int VALS = NP * NC;
  using TB = ThetaBits<R>;
  using U = typename TB::U;
  U* s_th = reinterpret_cast<U*>(smem);  // 8-byte aligned first
  R* s_own = reinterpret_cast<R*>(smem + size_t(kLim2dBlock) * sizeof(unsigned long long));
  R* s_lo = s_own + kLim2dBlock;
  R* s_hi = s_lo + kLim2dBlock;
  const int tid = threadIdx.x;
  if (tid < ne) {  // the element's cell mean and its interior neighbours' bounds
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
    s_own[tid] = own;
    s_lo[tid] = lo;
    s_hi[tid] = hi;
    s_th[tid] = TB::to(R(1));
  }
  __syncthreads();
  R* base = q + e0 * VALS;
  const R tiny = R(1.0e-30);
#pragma unroll 4
  for (int idx = tid; idx < ne * NP; idx += blockDim.x) {
    const int el = idx / NP;
    const R own = s_own[el];
    const R dl = base[size_t(idx) * NC] - own;  // component 0 of node idx - el NP of element el
    const R da = dl >= R(0) ? dl : -dl;
    if (da <= tiny) continue;
    R pD = s_hi[el] - own;
    if (pD < R(0)) pD = R(0);
    R nD = own - s_lo[el];
    if (nD < R(0)) nD = R(0);
    const R D = dl > R(0) ? pD : nD;
    const R D2 = D * D, d2 = da * da, Dd = D * da;
    const R al = (D2 + R(2) * Dd + eps2) / (D2 + R(2) * d2 + Dd + eps2);
    if (al < R(1)) atomicMin(&s_th[el], TB::to(al));
  }
  __syncthreads();
#pragma unroll 4
  for (int idx = tid; idx < ne * VALS; idx += blockDim.x) {
    const int el = idx / VALS;
    const R th = TB::from(s_th[el]);
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
  theta2d_block<R, NP, NC>(a.q, a.avg, e0, ne, t2, a.nx, a.ny, a.bc, a.eps2, lim_smem);
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
