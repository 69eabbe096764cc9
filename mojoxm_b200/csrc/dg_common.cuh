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
  // faces a cube evaluates once: every cube-boundary face (axis >= 0) and
  // the side-0 copy of every face inside the cube; entry = t * 4 + lf
  uint8_t face_work[24];
  int32_t n_face_work;
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

// Dynamic shared memory one block may use on sm_100a.
constexpr size_t kMaxSmemPerBlock = 227 * 1024;

// Element stride of the 3D SIMT stage's B tile (K columns x NC values,
// padded so that elements read by one warp fall in distinct banks).
__host__ __device__ constexpr int stage3d_bstr(int P, int NC, int rb) {
  const int K = 3 * ntet(P) + 4 * ntri(P), raw = K * NC, mod = rb == 8 ? 16 : 32;
  return raw + ((1 - raw % mod) + mod) % mod;
}
// Shared memory of the 3D SIMT stage with EC cubes per tile: barriers, the
// Kuhn table, two state tiles, the B tile, the operator (asmem) and the
// per-cube neighbour table.
__host__ __device__ constexpr size_t stage3d_smem(int P, int NC, int rb, int EC, bool asmem) {
  const size_t tab = rb == 8 ? (sizeof(KuhnTab3<double>) + 15) / 16 * 16 : (sizeof(KuhnTab3<float>) + 15) / 16 * 16;
  const size_t NP = size_t(ntet(P)), K = size_t(3 * ntet(P) + 4 * ntri(P));
  return 16 + tab + size_t(rb) * (2 * size_t(6 * EC) * NP * NC + size_t(6 * EC) * stage3d_bstr(P, NC, rb) +
                                  (asmem ? K * NP : 0)) +
         size_t(EC) * 12 * sizeof(int);
}
// Least shared memory the 3D SIMT stage needs (one cube per tile, operator
// read from global memory).
inline size_t stage3d_smem_need(int P, int NC, size_t rb) { return stage3d_smem(P, NC, int(rb), 1, false); }

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

// Neighbour cube and face treatment of the six cube faces of one cube,
// resolved once per tile so the face-node loops do no integer division.
// Direction index dd = 2 * axis + (dir > 0).  nb[dd] = neighbour cube
// (periodic wrap), md[dd] = face mode | BC code << 8.
__device__ __forceinline__ void cube_dirs3(int cell, int nx, int ny, int nz, const int* bc, int* nb, int* md, int dd) {
  const int nxy = nx * ny;
  const int ck = cell / nxy, rem = cell - ck * nxy, cj = rem / nx, ci = rem - cj * nx;
  const int ax = dd >> 1, dir = (dd & 1) ? 1 : -1;
  int code;
  const int mode = face_mode(ax, dir, ax == 0 ? ci : (ax == 1 ? cj : ck), ax == 0 ? nx : (ax == 1 ? ny : nz), bc, code);
  const int ni = ax == 0 ? wrapi(ci + dir, nx) : ci, nj = ax == 1 ? wrapi(cj + dir, ny) : cj,
            nk = ax == 2 ? wrapi(ck + dir, nz) : ck;
  nb[dd] = ni + nx * (nj + ny * nk);
  md[dd] = mode | (code << 8);
}

// Resident blocks per SM of a persistent kernel with `nt` threads and `smem`
// bytes of dynamic shared memory: the shared-memory carveout is set to its
// maximum first, then the count is the least of the shared-memory, thread
// and register limits (what the occupancy calculator reports, computed here
// from the device attributes so the carveout choice cannot lower it).
// Launch with programmatic stream serialisation: the kernel's blocks may
// start while the previous kernel of the stream finishes; the kernel itself
// waits (grid_dep_wait) before it touches that kernel's data.
template <class... KArgs, class... Args>
cudaError_t launch_dependent(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                             Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(unsigned(grid));
  cfg.blockDim = dim3(unsigned(block));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<Args&&>(args)...);
}

inline cudaError_t persistent_blocks_per_sm(const void* kern, int nt, size_t smem, int* bps) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  int dev = 0, smem_sm = 0, resv = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess) return e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, kern)) != cudaSuccess) return e;
  const size_t per_block = smem + size_t(fa.sharedSizeBytes) + size_t(resv);
  int by_smem = int(size_t(smem_sm) / per_block);
  int by_threads = 2048 / nt;
  const int regs_warp = ((fa.numRegs > 0 ? fa.numRegs : 1) * 32 + 255) / 256 * 256;
  int by_regs = 65536 / (regs_warp * ((nt + 31) / 32));
  int n = by_smem < by_threads ? by_smem : by_threads;
  n = n < by_regs ? n : by_regs;
  *bps = n < 1 ? 1 : n;
  return cudaSuccess;
}

// Kernel argument blocks (by value).
template <class R>
struct Stage3DArgs {
  const R* q_in;
  const R* q_a;
  const R* q_b;
  R* q_out;
  const R* A;  // [K][NP] shared operator [D_r|D_s|D_t|-Lift_0..3], k-major
  // q_out = q_a + b (q_b - q_a) + cdt rhs: the weights of q_a and q_b sum to
  // one exactly in any precision (in FP32, a = 1/3 and b = 2/3 rounded
  // separately sum to 1 + 3e-8, which scales the state by that much every
  // step); cdt = c dt is rounded once from FP64.
  R b, cdt;
  int nx, ny, nz;
  // cells cbeg .. ncell-1 are computed (all cells, or the owned layers of a
  // z-slab whose ghost layers are filled by the halo exchange)
  int cbeg, ncell;
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
  // q_out = q_a + b (q_b - q_a) + cdt rhs: the weights of q_a and q_b sum to
  // one exactly in any precision (in FP32, a = 1/3 and b = 2/3 rounded
  // separately sum to 1 + 3e-8, which scales the state by that much every
  // step); cdt = c dt is rounded once from FP64.
  R b, cdt;
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
  int64_t ne;      // cell means over elements 0 .. ne-1
  int64_t e0, e1;  // theta and its application over elements e0 .. e1-1 (3D)
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
// Batched tensor-core 3D stage: the tiles of many solves of one physics,
// order and operand kind in one launch.  items[t] = {solve, first cell,
// cells, 0}, the tiles of one solve consecutive; margs[solve] are the
// solve's arguments of the stage launched (q_in / q_a / q_b / q_out, b,
// c dt, mesh, boundaries), tabs[solve] its metric table.
struct Tc3Batch {
  const Stage3DArgs<float>* margs;
  const KuhnTab3<float>* tabs;
  const int4* items;
  int nitems;
};
template <class Phys>
cudaError_t launch_stage3d_tc_batch(int P, int kind, const Tc3Batch& bat, const Phys& ph, const unsigned char* img,
                                    int nsm, cudaStream_t st);
// Blocks that launch_stage3d_tc_batch runs for `ntiles` tiles.
template <class Phys>
cudaError_t stage3d_tc_batch_grid(int P, int kind, const Phys& ph, int nsm, int ntiles, int* out);

// Tensor-core 3D stage for FP32 state, P = 2..5: split-BF16 (kind
// TC_BF16, tcgen05 kind::f16) or split-TF32 (TC_TF32, kind::tf32) operands;
// `img` is the operator image built by tc_operator_image() for that kind.
constexpr int TC_BF16 = 0, TC_TF32 = 1;
template <class Phys>
cudaError_t launch_stage3d_tc(int P, int kind, const Stage3DArgs<float>& a, const KuhnTab3<float>& tab,
                              const Phys& ph, const unsigned char* img, int nsm, cudaStream_t st);
// Whether the tensor-core stage of (P, components, kind) fits one block's
// shared memory.
bool tc_shape_fits(int P, int NC, int kind);
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
