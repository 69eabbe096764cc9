// Instantiation and dispatch of the limiter and FP64 reduction kernels.
#include "limiter.cuh"

namespace mxm {

__global__ void reduce_final_kernel(const double* partial, int n, int kind, double scale, double* out) {
  // one warp, fixed order: deterministic
  __shared__ double red[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += 32) s = kind == 2 ? fmax(s, partial[k]) : s + partial[k];
  red[threadIdx.x] = s;
  __syncwarp();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < 32; ++k) t = kind == 2 ? fmax(t, red[k]) : t + red[k];
    *out = t * scale;
  }
}

template <class R, int DIM, int NP, int NC>
cudaError_t lim_np(const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2, cudaStream_t st) {
  const int64_t n1 = a.ne * NC;
  cell_avg_kernel<R, NP, NC, DIM == 3 ? NC : 1><<<int((n1 + 255) / 256), 256, 0, st>>>(a);
  if (DIM == 2) {
    constexpr size_t smem = lim2d_smem_bytes<R, NP, NC>();
    static bool attr = false;
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(theta2d_kernel<R, NP, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(smem));
      if (e != cudaSuccess) return e;
      attr = true;
    }
    theta2d_kernel<R, NP, NC><<<int((a.ne + kLim2dBlock - 1) / kLim2dBlock), kLim2dBlock, smem, st>>>(a, t2);
  } else {
    constexpr int EPB = 8;  // warps (elements) per block
    if (a.e1 > a.e0)
      theta_apply_kernel<R, DIM, NP, NC, EPB><<<int((a.e1 - a.e0 + EPB - 1) / EPB), 32 * EPB, 0, st>>>(a, t3, t2);
  }
  return cudaGetLastError();
}

template <class R, int DIM, int NC>
cudaError_t lim_nc(int P, const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2, cudaStream_t st) {
  switch (P) {
    case 1: return lim_np<R, DIM, DIM == 3 ? ntet(1) : ntri(1), NC>(a, t3, t2, st);
    case 2: return lim_np<R, DIM, DIM == 3 ? ntet(2) : ntri(2), NC>(a, t3, t2, st);
    case 3: return lim_np<R, DIM, DIM == 3 ? ntet(3) : ntri(3), NC>(a, t3, t2, st);
    case 4: return lim_np<R, DIM, DIM == 3 ? ntet(4) : ntri(4), NC>(a, t3, t2, st);
    case 5: return lim_np<R, DIM, DIM == 3 ? ntet(5) : ntri(5), NC>(a, t3, t2, st);
  }
  return cudaErrorInvalidValue;
}

template <class R>
cudaError_t launch_limiter(int dim, int P, int NC, const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2,
                           cudaStream_t st) {
  if (dim == 3) {
    switch (NC) {
      case 1: return lim_nc<R, 3, 1>(P, a, t3, t2, st);
      case 3: return lim_nc<R, 3, 3>(P, a, t3, t2, st);
      case 5: return lim_nc<R, 3, 5>(P, a, t3, t2, st);
      case 6: return lim_nc<R, 3, 6>(P, a, t3, t2, st);
      case 9: return lim_nc<R, 3, 9>(P, a, t3, t2, st);
      case 17: return lim_nc<R, 3, 17>(P, a, t3, t2, st);
    }
  } else {
    switch (NC) {
      case 1: return lim_nc<R, 2, 1>(P, a, t3, t2, st);
      case 3: return lim_nc<R, 2, 3>(P, a, t3, t2, st);
      case 4: return lim_nc<R, 2, 4>(P, a, t3, t2, st);
      case 6: return lim_nc<R, 2, 6>(P, a, t3, t2, st);
      case 7: return lim_nc<R, 2, 7>(P, a, t3, t2, st);
    }
  }
  return cudaErrorInvalidValue;
}

template <class R, int NP, int NC>
cudaError_t red_np(const R* q, const R* w, int64_t ne, int c, int kind, double scale, double* partial, int npartial,
                   double* out, cudaStream_t st) {
  int nb = int((ne + 255) / 256);
  if (nb > npartial) nb = npartial;
  if (nb < 1) nb = 1;
  reduce_partial_kernel<R, NP, NC><<<nb, 256, 0, st>>>(q, w, ne, c, kind, partial);
  reduce_final_kernel<<<1, 32, 0, st>>>(partial, nb, kind, scale, out);
  return cudaGetLastError();
}

template <class R, int NP>
cudaError_t red_nc(int NC, const R* q, const R* w, int64_t ne, int c, int kind, double scale, double* partial,
                   int npartial, double* out, cudaStream_t st) {
  switch (NC) {
    case 1: return red_np<R, NP, 1>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 3: return red_np<R, NP, 3>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 4: return red_np<R, NP, 4>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 5: return red_np<R, NP, 5>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 6: return red_np<R, NP, 6>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 7: return red_np<R, NP, 7>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 9: return red_np<R, NP, 9>(q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 17: return red_np<R, NP, 17>(q, w, ne, c, kind, scale, partial, npartial, out, st);
  }
  return cudaErrorInvalidValue;
}

template <class R>
cudaError_t launch_reduce(int P, int dim, int NC, const R* q, const R* w, int64_t ne, int c, int kind, double scale,
                          double* partial, int npartial, double* out, cudaStream_t st) {
  const int NP = dim == 3 ? ntet(P) : ntri(P);
  switch (NP) {
    case 3: return red_nc<R, 3>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 4: return red_nc<R, 4>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 6: return red_nc<R, 6>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 10: return red_nc<R, 10>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 15: return red_nc<R, 15>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 20: return red_nc<R, 20>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 21: return red_nc<R, 21>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 35: return red_nc<R, 35>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
    case 56: return red_nc<R, 56>(NC, q, w, ne, c, kind, scale, partial, npartial, out, st);
  }
  return cudaErrorInvalidValue;
}

// Scratch of the allocation-free reduction: kStaticPartials first-pass
// partial sums followed by one result slot, in the module's own static
// device memory.  The first pass writes every partial it launches a block
// for and the second pass writes the result slot, so nothing here has to
// start at zero.  The array is shared by every caller on a device: two
// reductions in flight at once on one device race on it.
static __device__ __align__(256) double g_static_reduce_scratch[kStaticPartials + 32];

cudaError_t static_reduce_scratch(double** ptr) {
  return cudaGetSymbolAddress((void**)ptr, g_static_reduce_scratch);
}

template cudaError_t launch_limiter<double>(int, int, int, const LimArgs<double>&, const KuhnTab3<double>&,
                                            const KuhnTab2<double>&, cudaStream_t);
template cudaError_t launch_limiter<float>(int, int, int, const LimArgs<float>&, const KuhnTab3<float>&,
                                           const KuhnTab2<float>&, cudaStream_t);
template cudaError_t launch_reduce<double>(int, int, int, const double*, const double*, int64_t, int, int, double,
                                           double*, int, double*, cudaStream_t);
template cudaError_t launch_reduce<float>(int, int, int, const float*, const float*, int64_t, int, int, double, double*,
                                          int, double*, cudaStream_t);

}  // namespace mxm
