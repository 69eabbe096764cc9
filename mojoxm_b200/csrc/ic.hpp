// Device initial-condition fill (ic_kernels.cu): arguments and launcher.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mxm {

constexpr int kMaxIcNC = 17;  // components of the widest physics (two-fluid)

struct IcArgs {
  int64_t ne;
  int dim, P, NP, NC, nx, ny, nz, kind;
  int kz0;                  // global z index of local layer 0 (slab parts)
  double h[3], L[3];
  double prm[32];
  double gamma, c;          // Euler gamma, Maxwell wave speed (from the physics)
  int8_t vert[6][4][3];     // cube-/cell-corner coordinates of each element type's vertices
  uint8_t bary[56][4];      // barycentric exponents of each node (sum P)
};

cudaError_t launch_ic(const IcArgs& a, void* q, size_t rbytes, cudaStream_t st);
// q[node * NC + c] *= f for every node (FP32 states multiply by float(f))
cudaError_t launch_scale_component(void* q, size_t rbytes, int64_t nnodes, int NC, int c, double f,
                                   cudaStream_t st);

}  // namespace mxm
