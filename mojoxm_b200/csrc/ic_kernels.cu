// Initial conditions written on the device, one thread per node, from node
// coordinates computed in FP64 from (cell, element type, barycentric node
// exponents).  This is the role of the reference's IC kernels, which write
// d_q from elem_node_xyz (examples/euler_vortex.mojo:87-129,
// benchmarks/bench_euler_smooth_wave_3d_p3.mojo:68-93,
// examples/euler_sod_2d_gpu.mojo:83-103,
// benchmarks/bench_shallow_water_dam_break_2d.mojo:41-58,
// benchmarks/bench_maxwell_cavity_3d.mojo:76).
#include <cuda_runtime.h>

#include "../../include/mxm_dg.h"
#include "ic.hpp"

namespace mxm {

namespace {

constexpr double kPi = 3.14159265358979323846;

template <class R>
__global__ void ic_kernel(IcArgs a, R* q) {
  const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (n >= a.ne * a.NP) return;
  const int64_t e = n / a.NP;
  const int i = int(n - e * a.NP);
  const int ntypes = a.dim == 3 ? 6 : 2;
  const int t = int(e % ntypes);
  const int64_t cell = e / ntypes;
  int ci, cj, ck = 0;
  if (a.dim == 3) {
    const int64_t nxy = int64_t(a.nx) * a.ny;
    const int kl = int(cell / nxy);
    ck = kl + a.kz0;
    const int64_t rem = cell - int64_t(kl) * nxy;
    cj = int(rem / a.nx);
    ci = int(rem - int64_t(cj) * a.nx);
  } else {
    cj = int(cell / a.nx);
    ci = int(cell - int64_t(cj) * a.nx);
  }
  const int nv = a.dim + 1;
  double x[3] = {0.0, 0.0, 0.0};
  for (int v = 0; v < nv; ++v) {
    const double b = double(a.bary[i][v]) / a.P;
    for (int d = 0; d < a.dim; ++d) x[d] += b * a.vert[t][v][d];
  }
  x[0] = (ci + x[0]) * a.h[0];
  x[1] = (cj + x[1]) * a.h[1];
  x[2] = a.dim == 3 ? (ck + x[2]) * a.h[2] : 0.0;
  const double* p = a.prm;
  const double g = a.gamma, g1 = g - 1.0;
  double s[kMaxIcNC] = {};
  const bool e3 = a.dim == 3;  // Euler: 3D (rho, m, E) or 2D (rho, mx, my, E)
  auto euler = [&](double rho, double u, double v, double w, double pr) {
    if (e3) {
      s[0] = rho; s[1] = rho * u; s[2] = rho * v; s[3] = rho * w;
      s[4] = pr / g1 + 0.5 * rho * (u * u + v * v + w * w);
    } else {
      s[0] = rho; s[1] = rho * u; s[2] = rho * v;
      s[3] = pr / g1 + 0.5 * rho * (u * u + v * v);
    }
  };
  switch (a.kind) {
    case MXM_DG_IC_CONSTANT:
      for (int c = 0; c < a.NC; ++c) s[c] = p[c];
      break;
    case MXM_DG_IC_SINE_WAVE: {  // rho0 + amp sin(2 pi k.x), uniform u, p
      const double ph = 2.0 * kPi * (p[6] * x[0] + p[7] * x[1] + p[8] * x[2]);
      euler(p[0] + p[1] * sin(ph), p[2], p[3], p[4], p[5]);
      break;
    }
    case MXM_DG_IC_VORTEX: {  // isentropic vortex of strength beta centred at (x0, y0)
      double dx = x[0] - p[1], dy = x[1] - p[2];
      if (p[6] != 0.0) {  // nearest periodic image
        dx -= a.L[0] * floor(dx / a.L[0] + 0.5);
        dy -= a.L[1] * floor(dy / a.L[1] + 0.5);
      }
      const double r2 = dx * dx + dy * dy, f = p[0] / (2.0 * kPi);
      const double ex = exp(0.5 * (1.0 - r2));
      const double T = 1.0 - g1 * f * f / (2.0 * g) * exp(1.0 - r2);
      const double rho = pow(T, 1.0 / g1);
      euler(rho, p[3] - f * dy * ex, p[4] + f * dx * ex, p[5], pow(rho, g));
      break;
    }
    case MXM_DG_IC_SOD: {  // tanh-smoothed tube along x
      const double w = 0.5 * (1.0 + tanh((x[0] - p[4]) / p[5]));
      euler(p[0] + (p[2] - p[0]) * w, 0.0, 0.0, 0.0, p[1] + (p[3] - p[1]) * w);
      break;
    }
    case MXM_DG_IC_DAM_BREAK: {  // shallow water: h from hL to hR across x0, at rest
      const double w = 0.5 * (1.0 + tanh((x[0] - p[2]) / p[3]));
      s[0] = p[0] + (p[1] - p[0]) * w;
      break;
    }
    case MXM_DG_IC_CAVITY: {  // Maxwell: E_z = amp sin(mx pi x / Lx) sin(my pi y / Ly), B = 0
      s[2] = p[2] * sin(p[0] * kPi * x[0] / a.L[0]) * sin(p[1] * kPi * x[1] / a.L[1]);
      break;
    }
    case MXM_DG_IC_PLANE_WAVE: {  // Maxwell: E_z = amp sin(2 pi k x / Lx), B_y = -E_z / c
      const double ez = p[0] * sin(2.0 * kPi * p[1] * x[0] / a.L[0]);
      s[2] = ez;
      s[4] = -ez / a.c;
      break;
    }
    case MXM_DG_IC_ALFVEN: {  // MHD: right-going Alfven wave along x (bench_mhd_alfven_3d_p3.mojo:68-102)
      const double sn = sin(2.0 * kPi * p[4] * x[0] / a.L[0]);
      const double rho = p[0], bx = p[1], v = p[3] * sn, by = -p[3] * sqrt(rho) * sn;
      const double E = p[2] / g1 + 0.5 * rho * v * v + 0.5 * (bx * bx + by * by);
      s[0] = rho; s[2] = rho * v;
      if (e3) {  // (rho, m, E, B, psi)
        s[4] = E; s[5] = bx; s[6] = by;
      } else {   // (rho, mx, my, Bx, By, E[, psi])
        s[3] = bx; s[4] = by; s[5] = E;
      }
      break;
    }
  }
  R* out = q + n * a.NC;
  for (int c = 0; c < a.NC; ++c) out[c] = R(s[c]);
}

}  // namespace

template <class R>
__global__ void scale_component_kernel(R* q, int64_t nnodes, int NC, int c, R f) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nnodes) q[i * NC + c] = q[i * NC + c] * f;
}

cudaError_t launch_scale_component(void* q, size_t rbytes, int64_t nnodes, int NC, int c, double f,
                                   cudaStream_t st) {
  const int nb = int((nnodes + 255) / 256);
  if (nb == 0) return cudaSuccess;
  if (rbytes == 8) scale_component_kernel<double><<<nb, 256, 0, st>>>((double*)q, nnodes, NC, c, f);
  else scale_component_kernel<float><<<nb, 256, 0, st>>>((float*)q, nnodes, NC, c, float(f));
  return cudaGetLastError();
}

cudaError_t launch_ic(const IcArgs& a, void* q, size_t rbytes, cudaStream_t st) {
  const int64_t n = a.ne * a.NP;
  const int nb = int((n + 255) / 256);
  if (rbytes == 8) ic_kernel<double><<<nb, 256, 0, st>>>(a, (double*)q);
  else ic_kernel<float><<<nb, 256, 0, st>>>(a, (float*)q);
  return cudaGetLastError();
}

}  // namespace mxm
