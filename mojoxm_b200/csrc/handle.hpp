// Host-side state of one solve (the C ABI's opaque handle) and the error
// types of the library's host code; shared by capi.cu and batch.cu.
#pragma once
#include <cuda_runtime.h>

#include <exception>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mxm_dg.h"
#include "dg_common.cuh"
#include "refops.hpp"

namespace mxm {

struct CudaError : std::exception {
  cudaError_t e;
  std::string msg;
  CudaError(cudaError_t e_, const char* where) : e(e_), msg(std::string(where) + ": " + cudaGetErrorString(e_)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};
struct ArgError : std::exception {
  std::string msg;
  explicit ArgError(std::string m) : msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};
#define CK(x)                                              \
  do {                                                     \
    cudaError_t _e = (x);                                  \
    if (_e != cudaSuccess) throw ::mxm::CudaError(_e, #x); \
  } while (0)

struct Handle {
  int dim = 3, P = 1, prec = MXM_DG_PREC_F64, NP = 0, NFP = 0, NC = 0, ntypes = 6, K = 0;
  mxm_dg_physics_desc phys{};
  int nx = 1, ny = 1, nz = 1;
  double lx = 1, ly = 1, lz = 1;
  int bc[6] = {0, 0, 0, 0, 0, 0};
  int64_t ncell = 0, ne = 0;
  // z-slab decomposition (mxm_dg_create_slab): the local z layers are
  // [ghost lo] owned layers [ghost hi]; cells cbeg .. cend-1 are owned and
  // computed, the ghost layers are filled by the halo exchange.  A plain
  // handle is one part with no ghosts (cbeg = 0, cend = ncell).
  int nparts = 1, part = 0, glo = 0, ghi = 0, nb_lo = -1, nb_hi = -1;
  int nzg = 1, kz0 = 0;  // global z cells; global z index of local layer 0
  int64_t cbeg = 0, cend = 0;
  struct NcclLink* nccl = nullptr;  // halo transport of a multi-process slab
  cudaStream_t comm = nullptr;       // a slab part's exchange stream
  // host pipeline of mxm_dg_advance_host_async: copy streams, the result's
  // device staging buffer and the events that order them
  // host-buffer pipeline: two staging buffers per direction, used by
  // alternate calls (slot = pipe_calls & 1)
  cudaStream_t h2d = nullptr, d2h = nullptr;
  void *in_stage[2] = {nullptr, nullptr}, *out_stage[2] = {nullptr, nullptr};
  cudaEvent_t e_in_free[2] = {nullptr, nullptr}, e_in[2] = {nullptr, nullptr};
  cudaEvent_t e_res[2] = {nullptr, nullptr}, e_out_free[2] = {nullptr, nullptr};
  int64_t pipe_calls = 0;
  cudaEvent_t ev_in = nullptr, ev_x = nullptr;  // input written / ghosts landed
  size_t rbytes = 8;
  int device = 0, nsm = 148;
  cudaStream_t stream = nullptr;
  void* q[3] = {nullptr, nullptr, nullptr};
  void* A = nullptr;
  void* w = nullptr;
  void* avg = nullptr;
  float* xyz = nullptr;
  double* partial = nullptr;
  double* dscalar = nullptr;
  unsigned long long* uscalar = nullptr;
  int* derr = nullptr;  // device error word written by bounded waits
  bool use_tc = false;  // MIXED / MIXED_TF32 precision: tensor-core contraction
  int tc_kind = 0;      // TC_BF16 or TC_TF32 operands
  void* tcimg = nullptr;  // operator image (bf16 hi | lo) in the UMMA layout
  int npartial = 1024;
  bool lim_on = false;
  double lim_eps = 0.1;
  RefOps ref;
  Kuhn3D k3;
  Kuhn2D k2;
  std::vector<double> Ahost;
  KuhnTab3<double> t3d{};
  KuhnTab3<float> t3f{};
  KuhnTab2<double> t2d{};
  KuhnTab2<float> t2f{};
  std::string err;
  size_t qcount() const { return size_t(ne) * NP * NC; }
  int64_t own_e0() const { return cbeg * ntypes; }
  int64_t own_ne() const { return (cend - cbeg) * ntypes; }
  double hz() const { return lz / nzg; }  // cell size along z (global)
  size_t qbytes() const { return qcount() * rbytes; }
};

// error text of calls that have no handle yet (create, batch create)
extern std::mutex g_err_mu;
extern std::string g_create_err;

// Solver operations shared by the C ABI, the batch and the server (capi.cu);
// they throw CudaError / ArgError.
// One part of a z-slab decomposition: global z cells [cz0, cz1) owned, ghost
// layers below/above (glo, ghi) and the local BC codes of the z faces.
struct SlabPlan {
  int cz0, cz1, glo, ghi, bc_lo, bc_hi, nb_lo, nb_hi;
};
SlabPlan slab_plan(int nz, int bc_lo, int bc_hi, int nparts, int part);
// One point-to-point operation of a part's ghost exchange: send (recv = 0)
// the local z layer `layer` to part `peer`, or receive (recv = 1) into it.
struct SlabXOp {
  int recv, peer, layer;
};
// The exchange of a part with ghost layers (glo, ghi), neighbours (nb_lo,
// nb_hi) and local_nz local layers, in the order the NCCL transport issues
// it; returns the count (at most 4).
int slab_exchange_ops(int glo, int ghi, int nb_lo, int nb_hi, int local_nz, SlabXOp out[4]);

Handle* create(const mxm_dg_mesh_desc* m, const mxm_dg_physics_desc* ph, int P, int prec,
               const SlabPlan* slab = nullptr, int nparts = 1, int part = 0);
void destroy(Handle* h);
void step_n(Handle* h, double dt, int n);
// stage kernel of Shu-Osher stage s without exchange or limiter, and the
// buffers it reads and writes
void stage_only(Handle* h, int s, double dt, int64_t c0 = -1, int64_t c1 = -1);
void slab_ranges(const Handle* h, int64_t in[2], int64_t lo[2], int64_t hi[2]);
int stage_in(int s);
int stage_out(int s);
void limit_buf(Handle* h, void* qv);
// Batched 3D tensor-core stages: stage s's arguments of a handle (its error
// word replaced by `err`), the launch of a batch of tiles of handles of h0's
// physics, order and operand kind, and the cubes per tile of that shape.
Stage3DArgs<float> tc_stage_args(const Handle* h, int s, double dt, int* err);
cudaError_t launch_tc_group(const Handle* h0, const Tc3Batch& bat, cudaStream_t st);
cudaError_t tc_group_grid(const Handle* h0, int ntiles, int* out);
int tc_tile_cubes(int P, int NC, int kind);
// NCCL halo transport (slab.cu): exchange the ghost layers of state buffer
// `which` on the handle's stream; release the link
void nccl_exchange(Handle* h, int which, cudaStream_t st);
void nccl_release(Handle* h);
void fill_ic(Handle* h, int which, int kind, const double* params, int nparams);
// 2D GLM-MHD psi damping after each step: whether h has it, and its factor
bool glm_damped(const Handle* h);
double psi_decay(const Handle* h, double dt);

}  // namespace mxm
