// Shared device-side definitions of the B200 DG kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mxm {

__host__ __device__ constexpr int ntet(int P) { return (P + 1) * (P + 2) * (P + 3) / 6; }
__host__ __device__ constexpr int ntri(int P) { return (P + 1) * (P + 2) / 2; }
constexpr int kMaxNFP3 = 21;  // P = 5 tet face
constexpr int kMaxNFP2 = 6;   // P = 5 triangle edge

enum : int { BC_INTERIOR = 0, BC_WALL = 1, BC_OUTFLOW = 2, BC_INFLOW = 3 };
enum : int { FLUX_RUSANOV = 0, FLUX_ROE = 1, FLUX_HLLE = 2, FLUX_HLLEC = 3, FLUX_HLLC = 4, FLUX_HLL = 5 };

// Kuhn topology of one tet type's faces, passed by value as a kernel
// parameter (lives in the constant bank; ~1.7 KB).
template <class R>
struct KuhnTab3 {
  R normal[6][4][3];  // unit normal, side 0 -> side 1
  R invJ[6][9];       // d(r,s,t)/d(x,y,z) per tet type, [k][d]
  R fscale[6][4];     // side_sign * face area / (6 V)
  int8_t nb_t[6][4];
  int8_t off[6][4][3];
  int8_t side[6][4];
  int8_t axis[6][4];
  int8_t dir[6][4];
  uint8_t own_node[4][kMaxNFP3];
  uint8_t nb_node[6][4][kMaxNFP3];
  uint8_t nb_lf[6][4];             // neighbour's local face
  uint8_t nb_m[6][4][kMaxNFP3];    // neighbour's face-local index of face node m
};

template <class R>
struct KuhnTab2 {
  R normal[2][3][2];
  R invJ[2][4];    // d(r,s)/d(x,y) per triangle type, [k][d]
  R fscale[2][3];  // side_sign * edge length / (2 A)
  int8_t nb_t[2][3];
  int8_t off[2][3][2];
  int8_t side[2][3];
  int8_t axis[2][3];
  int8_t dir[2][3];
  uint8_t own_node[3][kMaxNFP2];
  uint8_t nb_node[2][3][kMaxNFP2];
};

// Face treatment for an element's face, resolved from the cell position and
// the six BC codes exactly as mojoxm's BC overlay resolves it
// (src/local_mesh.mojo:946-1187): the +axis cube face of the last cell
// layer becomes a boundary face when bc_hi != 0; the -axis face of the first
// layer gets its own one-sided boundary face when bc_lo != 0; with bc_lo ==
// 0 but bc_hi != 0 the first layer still reads the shared face, whose flux
// is the boundary flux of the last layer's state.
enum : int { FACE_INTERIOR = 0, FACE_BC_HI = 1, FACE_BC_LO = 2, FACE_MIXED = 3 };

__device__ __forceinline__ int face_mode(int axis, int dir, int cpos, int ncell_axis, const int* bc, int& code) {
  code = 0;
  if (axis < 0) return FACE_INTERIOR;
  // constant indices keep a by-value bc[] in the parameter bank (no local copy)
  const int lo = axis == 0 ? bc[0] : (axis == 1 ? bc[2] : bc[4]);
  const int hi = axis == 0 ? bc[1] : (axis == 1 ? bc[3] : bc[5]);
  if (dir > 0) {
    if (cpos == ncell_axis - 1 && hi != 0) {
      code = hi;
      return FACE_BC_HI;
    }
    return FACE_INTERIOR;
  }
  if (cpos == 0) {
    if (lo != 0) {
      code = lo;
      return FACE_BC_LO;
    }
    if (hi != 0) {
      code = hi;
      return FACE_MIXED;
    }
  }
  return FACE_INTERIOR;
}

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Per-tile face descriptor, resolved once per (element, local face) at the
// start of a tile so the face-node loops do no integer division:
//   x = mode | code << 8,  y = neighbour element (global index), z = neighbour
//   element inside the tile (-1 when outside)
struct FaceInfo {
  int x, y, z;
};

// Fill info[el*4 + lf] for the ne_here elements of a tile of whole cubes
// starting at cell0 (3D Kuhn meshes).
template <class Tab, class Args>
__device__ __forceinline__ void setup_faces3(const Tab* tab, const Args& args, int cell0, int ne_here, FaceInfo* info,
                                             int tid, int nt) {
  const int nxy = args.nx * args.ny;
  for (int idx = tid; idx < ne_here * 4; idx += nt) {
    const int el = idx >> 2, lf = idx & 3, t = el % 6, cl = el / 6;
    const int cell = cell0 + cl;
    const int ck = cell / nxy, rem = cell - ck * nxy, cj = rem / args.nx, ci = rem - cj * args.nx;
    const int ax = tab->axis[t][lf];
    int code;
    const int mode = face_mode(ax, tab->dir[t][lf], ax == 0 ? ci : (ax == 1 ? cj : ck),
                               ax == 0 ? args.nx : (ax == 1 ? args.ny : args.nz), args.bc, code);
    const int nbt = tab->nb_t[t][lf];
    const int ni = wrapi(ci + tab->off[t][lf][0], args.nx), nj = wrapi(cj + tab->off[t][lf][1], args.ny),
              nk = wrapi(ck + tab->off[t][lf][2], args.nz);
    FaceInfo f;
    f.x = mode | (code << 8);
    f.y = (ni + args.nx * (nj + args.ny * nk)) * 6 + nbt;
    f.z = ax < 0 ? cl * 6 + nbt : -1;
    info[idx] = f;
  }
}

// Kernel argument blocks (by value).
template <class R>
struct Stage3DArgs {
  const R* q_in;
  const R* q_a;
  const R* q_b;
  R* q_out;
  const R* A;  // [K][NP] shared operator [D_r|D_s|D_t|-Lift_0..3], k-major
  R a, b, cdt;
  int nx, ny, nz;
  int ncell;
  int bc[6];
  int rhs_only;
  int* err;  // device error word (bounded waits that gave up set bit 0)
};

template <class R>
struct Stage2DArgs {
  const R* q_in;
  const R* q_a;
  const R* q_b;
  R* q_out;
  const R* A;  // [K][NP] shared operator [D_r|D_s|-Lift_0..2], k-major
  R a, b, cdt;
  int nx, ny;
  int ncell;
  int bc[4];
  int rhs_only;
  int* err;
};

template <class R>
struct LimArgs {
  R* q;
  R* avg;          // [Ne][NC]
  const R* w;      // [NP] node weights
  int64_t ne;
  int nx, ny, nz;  // cells (nz = 1 in 2D)
  int bc[6];
  R eps2;
};

// Host launchers; each is explicitly instantiated next to its kernels.
template <class R, class Phys>
cudaError_t launch_stage3d(int P, const Stage3DArgs<R>& a, const KuhnTab3<R>& tab, const Phys& ph, int nsm,
                           cudaStream_t st);
template <class R, class Phys>
cudaError_t launch_wavespeed3d(int P, const Stage3DArgs<R>& a, const KuhnTab3<R>& tab, const Phys& ph,
                               unsigned long long* out, cudaStream_t st);
// Tensor-core (split-BF16 tcgen05) 3D stage for FP32 state, P = 2..4;
// `img` is the operator image built by tc_operator_image().
template <class Phys>
cudaError_t launch_stage3d_tc(int P, const Stage3DArgs<float>& a, const KuhnTab3<float>& tab, const Phys& ph,
                              const unsigned char* img, int nsm, cudaStream_t st);
template <class R, class Phys>
cudaError_t launch_stage2d(int P, const Stage2DArgs<R>& a, const KuhnTab2<R>& tab, const Phys& ph, int nsm,
                           cudaStream_t st);
template <class R, class Phys>
cudaError_t launch_wavespeed2d(const R* q, int64_t nnodes, const Phys& ph, unsigned long long* out, cudaStream_t st);
template <class R>
cudaError_t launch_limiter(int dim, int P, int NC, const LimArgs<R>& a, const KuhnTab3<R>& t3, const KuhnTab2<R>& t2,
                           cudaStream_t st);
template <class R>
cudaError_t launch_reduce(int P, int dim, int NC, const R* q, const R* w, int64_t ne, int c, int kind, double scale,
                          double* partial, int npartial, double* out, cudaStream_t st);
// Static (module-resident) scratch of the allocation-free reduction: the
// address of kStaticPartials partial slots followed by the result slot, on
// the calling thread's current device.
constexpr int kStaticPartials = 4096;
cudaError_t static_reduce_scratch(double** ptr);

}  // namespace mxm
