// Domain decomposition of one 3D mesh into z-slabs with a one-layer halo.
//
// Replaces the reference's np > 1 path: build_partition / choose_proc_grid
// (src/partition.mojo:106-228) and HaloExchange (src/halo_exchange.mojo:
// 187-395), which give every rank a box of cubes with a one-cube ghost ring
// and exchange the six face rings once per RK stage through pack kernels,
// MPI and unpack kernels.
//
// B200 form: the parts are slabs of whole z layers.  Cells are numbered
// i + Nx (j + Ny k), so a z layer of cubes is one contiguous span of the
// state (Nx Ny 6 NP NC values) and a ghost layer is filled by ONE copy from
// the neighbour's boundary layer -- no pack or unpack kernels, no index
// lists.  Through NVSwitch every GPU reaches every peer at full bandwidth,
// so the surface-minimising process grid of the reference buys nothing here,
// while contiguous layers keep the exchange a plain DMA.  The stage and
// limiter kernels are the single-domain ones run over the owned cell range
// (the ghost layers are read, never computed); the local z boundary faces
// next to a ghost layer are interior faces, so the owned elements see
// exactly the neighbours and arithmetic of the undecomposed mesh and the
// decomposed solve is bit-identical to it.
//
// Transports: (1) an in-process group of handles (one host thread, any
// devices; copies with cudaMemcpyPeerAsync, ordered by events), and (2) NCCL
// point-to-point over NVLink between processes, one per GPU (NCCL is loaded
// at run time, only when a part connects).
#include <dlfcn.h>
#include <nccl.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "handle.hpp"

namespace mxm {

SlabPlan slab_plan(int nz, int bc_lo, int bc_hi, int nparts, int part) {
  if (nparts < 1 || part < 0 || part >= nparts) throw ArgError("part must lie in 0..nparts-1");
  if (nz < nparts) throw ArgError("every part needs at least one z layer of cells (nz >= nparts)");
  if ((bc_lo == 0) != (bc_hi == 0))
    throw ArgError("a z-slab decomposition needs both z boundaries periodic or both bounded");
  SlabPlan p{};
  p.cz0 = int(int64_t(part) * nz / nparts);
  p.cz1 = int(int64_t(part + 1) * nz / nparts);
  const bool periodic = bc_lo == 0;
  p.glo = nparts > 1 && (part > 0 || periodic);
  p.ghi = nparts > 1 && (part < nparts - 1 || periodic);
  // a face next to a ghost layer is interior; the ghost layers themselves
  // are never computed, so the wrap between them is never read
  p.bc_lo = p.glo ? 0 : bc_lo;
  p.bc_hi = p.ghi ? 0 : bc_hi;
  p.nb_lo = p.glo ? (part + nparts - 1) % nparts : -1;
  p.nb_hi = p.ghi ? (part + 1) % nparts : -1;
  return p;
}

// Every part issues its sends in the order (up: top owned layer to the hi
// neighbour, down: bottom owned layer to the lo neighbour) and its receives
// in the order (from lo: the up message, from hi: the down message), so the
// messages of a pair of parts that neighbour each other on both sides (two
// periodic parts) match in NCCL's per-pair issue order.
int slab_exchange_ops(int glo, int ghi, int nb_lo, int nb_hi, int local_nz, SlabXOp out[4]) {
  int n = 0;
  if (ghi) out[n++] = SlabXOp{0, nb_hi, local_nz - 2};  // top owned layer
  if (glo) out[n++] = SlabXOp{0, nb_lo, glo};           // bottom owned layer (local layer 1)
  if (glo) out[n++] = SlabXOp{1, nb_lo, 0};             // ghost layer below
  if (ghi) out[n++] = SlabXOp{1, nb_hi, local_nz - 1};  // ghost layer above
  return n;
}

namespace {

size_t layer_vals(const Handle* h) { return size_t(h->nx) * h->ny * 6 * h->NP * h->NC; }
// local z-layer indices of the owned boundary layers and the ghost layers
int owned_lo_layer(const Handle* h) { return h->glo; }
int owned_hi_layer(const Handle* h) { return h->nz - h->ghi - 1; }
int ghost_lo_layer(const Handle* h) { return h->glo ? 0 : -1; }
int ghost_hi_layer(const Handle* h) { return h->ghi ? h->nz - 1 : -1; }
char* layer_ptr(const Handle* h, int which, int layer) {
  return static_cast<char*>(h->q[which]) + size_t(layer) * layer_vals(h) * h->rbytes;
}

// ---- NCCL, resolved at run time --------------------------------------------
struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

std::mutex g_nccl_mu;

const NcclApi& nccl_api() {
  static NcclApi api;
  static bool loaded = false;
  std::lock_guard<std::mutex> g(g_nccl_mu);
  if (loaded) return api;
  // an NCCL already in the process (e.g. the one a framework loaded) is reused
  void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) throw ArgError(std::string("NCCL is not loadable: ") + dlerror());
  auto sym = [&](const char* n) {
    void* f = dlsym(lib, n);
    if (!f) throw ArgError(std::string("NCCL lacks ") + n);
    return f;
  };
  api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
  api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(sym("ncclCommInitRank"));
  api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
  api.group_start = reinterpret_cast<decltype(api.group_start)>(sym("ncclGroupStart"));
  api.group_end = reinterpret_cast<decltype(api.group_end)>(sym("ncclGroupEnd"));
  api.send = reinterpret_cast<decltype(api.send)>(sym("ncclSend"));
  api.recv = reinterpret_cast<decltype(api.recv)>(sym("ncclRecv"));
  api.error_string = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
  loaded = true;
  return api;
}

void nck(ncclResult_t r, const char* where) {
  if (r != ncclSuccess) throw ArgError(std::string(where) + ": " + nccl_api().error_string(r));
}

}  // namespace

struct NcclLink {
  ncclComm_t comm = nullptr;
};

// The part's sends and receives in slab_exchange_ops' order, as one NCCL group.
void nccl_exchange(Handle* h, int which, cudaStream_t st) {
  const NcclApi& api = nccl_api();
  const size_t bytes = layer_vals(h) * h->rbytes;
  SlabXOp ops[4];
  const int n = slab_exchange_ops(h->glo, h->ghi, h->nb_lo, h->nb_hi, h->nz, ops);
  nck(api.group_start(), "ncclGroupStart");
  for (int k = 0; k < n; ++k) {
    char* p = layer_ptr(h, which, ops[k].layer);
    if (ops[k].recv) nck(api.recv(p, bytes, ncclUint8, ops[k].peer, h->nccl->comm, st), "ncclRecv");
    else nck(api.send(p, bytes, ncclUint8, ops[k].peer, h->nccl->comm, st), "ncclSend");
  }
  nck(api.group_end(), "ncclGroupEnd");
}

void nccl_release(Handle* h) {
  if (h->nccl && h->nccl->comm) nccl_api().comm_destroy(h->nccl->comm);
  delete h->nccl;
  h->nccl = nullptr;
}

// ---- in-process group ------------------------------------------------------
struct Group {
  std::vector<Handle*> parts;
  std::vector<cudaEvent_t> ev;
  std::string err;

  // every part's stream waits for its neighbours' work enqueued so far
  void barrier() {
    for (size_t r = 0; r < parts.size(); ++r) {
      CK(cudaSetDevice(parts[r]->device));
      CK(cudaEventRecord(ev[r], parts[r]->stream));
    }
    for (size_t r = 0; r < parts.size(); ++r) {
      Handle* h = parts[r];
      CK(cudaSetDevice(h->device));
      for (int n : {h->nb_lo, h->nb_hi})
        if (n >= 0 && n != int(r)) CK(cudaStreamWaitEvent(h->stream, ev[n], 0));
    }
  }
  // ghost layers of buffer `which` from the neighbours' boundary layers: the
  // first barrier orders the copies after the neighbours' writes, the second
  // keeps a part from rewriting layers its neighbours are still copying
  void exchange(int which) {
    barrier();
    for (int r = 0; r < int(parts.size()); ++r) {
      CK(cudaSetDevice(parts[r]->device));
      pull(r, which, parts[r]->stream);
    }
    barrier();
  }
  // copy the neighbours' boundary layers of `which` into part r's ghost layers on stream st
  void pull(int r, int which, cudaStream_t st) {
    Handle* h = parts[r];
    const size_t bytes = layer_vals(h) * h->rbytes;
    if (h->glo) {
      const Handle* lo = parts[h->nb_lo];
      CK(cudaMemcpyPeerAsync(layer_ptr(h, which, ghost_lo_layer(h)), h->device,
                             layer_ptr(lo, which, owned_hi_layer(lo)), lo->device, bytes, st));
    }
    if (h->ghi) {
      const Handle* hi = parts[h->nb_hi];
      CK(cudaMemcpyPeerAsync(layer_ptr(h, which, ghost_hi_layer(h)), h->device,
                             layer_ptr(hi, which, owned_lo_layer(hi)), hi->device, bytes, st));
    }
  }
  // One stage with the exchange of its input overlapped: each part's
  // exchange stream waits for its own and its neighbours' last writes, pulls
  // its ghost layers while the main stream computes the interior cells; the
  // boundary layers wait for the part's own copies and for the neighbours'
  // copies out of this part (which must finish before it writes again).
  void stage_overlapped(int s, double dt) {
    const int n = int(parts.size());
    for (int r = 0; r < n; ++r) {
      CK(cudaSetDevice(parts[r]->device));
      CK(cudaEventRecord(parts[r]->ev_in ? parts[r]->ev_in : ev[r], parts[r]->stream));
    }
    auto ev_in = [&](int r) { return parts[r]->ev_in ? parts[r]->ev_in : ev[r]; };
    for (int r = 0; r < n; ++r) {
      Handle* h = parts[r];
      if (!h->comm) continue;  // no ghost layers
      CK(cudaSetDevice(h->device));
      CK(cudaStreamWaitEvent(h->comm, ev_in(r), 0));
      for (int nb : {h->nb_lo, h->nb_hi})
        if (nb >= 0 && nb != r) CK(cudaStreamWaitEvent(h->comm, ev_in(nb), 0));
      pull(r, stage_in(s), h->comm);
      CK(cudaEventRecord(h->ev_x, h->comm));
    }
    int64_t in[2], lo[2], hi[2];
    for (int r = 0; r < n; ++r) {
      Handle* h = parts[r];
      CK(cudaSetDevice(h->device));
      slab_ranges(h, in, lo, hi);
      if (in[1] > in[0]) stage_only(h, s, dt, in[0], in[1]);
    }
    for (int r = 0; r < n; ++r) {
      Handle* h = parts[r];
      CK(cudaSetDevice(h->device));
      if (h->comm) CK(cudaStreamWaitEvent(h->stream, h->ev_x, 0));
      for (int nb : {h->nb_lo, h->nb_hi})
        if (nb >= 0 && nb != r && parts[nb]->comm) CK(cudaStreamWaitEvent(h->stream, parts[nb]->ev_x, 0));
      slab_ranges(h, in, lo, hi);
      if (lo[1] > lo[0]) stage_only(h, s, dt, lo[0], lo[1]);
      if (hi[1] > hi[0]) stage_only(h, s, dt, hi[0], hi[1]);
    }
  }
  void step_n(double dt, int nsteps) {
    for (int k = 0; k < nsteps; ++k)
      for (int s = 0; s < 3; ++s) {
        stage_overlapped(s, dt);
        if (parts[0]->lim_on) {
          exchange(stage_out(s));
          for (Handle* h : parts) {
            CK(cudaSetDevice(h->device));
            limit_buf(h, h->q[stage_out(s)]);
          }
        }
      }
  }
};

}  // namespace mxm

using mxm::Group;
using mxm::Handle;

#define SLAB_BEGIN                \
  Handle* h = (Handle*)handle;    \
  if (!h) return MXM_DG_EINVAL;   \
  try {                           \
    cudaSetDevice(h->device);
#define SLAB_END                                                              \
  return MXM_DG_OK;                                                           \
  }                                                                           \
  catch (mxm::CudaError & ex) {                                               \
    h->err = ex.what();                                                       \
    return ex.e == cudaErrorMemoryAllocation ? MXM_DG_ENOMEM : MXM_DG_ECUDA;  \
  }                                                                           \
  catch (std::exception & ex) {                                               \
    h->err = ex.what();                                                       \
    return MXM_DG_EINVAL;                                                     \
  }

static int create_error(const std::exception& ex, int rc) {
  std::lock_guard<std::mutex> g(mxm::g_err_mu);
  mxm::g_create_err = ex.what();
  return rc;
}

extern "C" {

int mxm_dg_slab_plan(int nz, int bc_lo, int bc_hi, int nparts, int part, int32_t* out8) {
  if (!out8) return MXM_DG_EINVAL;
  try {
    const mxm::SlabPlan p = mxm::slab_plan(nz, bc_lo, bc_hi, nparts, part);
    const int32_t v[8] = {p.cz0, p.cz1, p.glo, p.ghi, p.bc_lo, p.bc_hi, p.nb_lo, p.nb_hi};
    std::memcpy(out8, v, sizeof(v));
    return MXM_DG_OK;
  } catch (std::exception& ex) {
    return create_error(ex, MXM_DG_EINVAL);
  }
}

int mxm_dg_slab_exchange_ops(int nz, int bc_lo, int bc_hi, int nparts, int part, int32_t* out12, int* nops) {
  if (!out12 || !nops) return MXM_DG_EINVAL;
  try {
    const mxm::SlabPlan p = mxm::slab_plan(nz, bc_lo, bc_hi, nparts, part);
    mxm::SlabXOp ops[4];
    const int n = mxm::slab_exchange_ops(p.glo, p.ghi, p.nb_lo, p.nb_hi, p.cz1 - p.cz0 + p.glo + p.ghi, ops);
    for (int k = 0; k < n; ++k) {
      out12[3 * k] = ops[k].recv;
      out12[3 * k + 1] = ops[k].peer;
      out12[3 * k + 2] = ops[k].layer;
    }
    *nops = n;
    return MXM_DG_OK;
  } catch (std::exception& ex) {
    return create_error(ex, MXM_DG_EINVAL);
  }
}

int mxm_dg_create_slab(const mxm_dg_mesh_desc* mesh, const mxm_dg_physics_desc* phys, int P, int precision,
                       int nparts, int part, void** out) {
  if (!out) return MXM_DG_EINVAL;
  *out = nullptr;
  try {
    if (!mesh || mesh->dim != 3) throw mxm::ArgError("slab decomposition is for 3D meshes");
    const mxm::SlabPlan p = mxm::slab_plan(mesh->nz, mesh->bc[4], mesh->bc[5], nparts, part);
    *out = mxm::create(mesh, phys, P, precision, &p, nparts, part);
    return MXM_DG_OK;
  } catch (mxm::CudaError& ex) {
    return create_error(ex, ex.e == cudaErrorMemoryAllocation ? MXM_DG_ENOMEM : MXM_DG_ECUDA);
  } catch (std::exception& ex) {
    return create_error(ex, MXM_DG_EINVAL);
  }
}

int mxm_dg_slab_info(void* handle, int64_t* out8) {
  SLAB_BEGIN
  if (!out8) throw mxm::ArgError("out8 must be non-null");
  const int64_t v[8] = {h->nparts, h->part, h->kz0 + h->glo, h->kz0 + h->glo + (h->nz - h->glo - h->ghi),
                        h->glo, h->ghi, h->own_e0(), h->own_ne()};
  std::memcpy(out8, v, sizeof(v));
  SLAB_END
}

int mxm_dg_slab_layout(void* handle, int64_t* out5) {
  SLAB_BEGIN
  if (!out5) throw mxm::ArgError("out5 must be non-null");
  const int64_t L = int64_t(mxm::layer_vals(h));
  out5[0] = L;
  out5[1] = int64_t(mxm::owned_lo_layer(h)) * L;
  out5[2] = int64_t(mxm::owned_hi_layer(h)) * L;
  out5[3] = h->glo ? int64_t(mxm::ghost_lo_layer(h)) * L : -1;
  out5[4] = h->ghi ? int64_t(mxm::ghost_hi_layer(h)) * L : -1;
  SLAB_END
}

int mxm_dg_slab_stage(void* handle, int s, double dt) {
  SLAB_BEGIN
  if (s < 0 || s > 2) throw mxm::ArgError("stage must be 0, 1 or 2");
  mxm::stage_only(h, s, dt);
  SLAB_END
}

int mxm_dg_nccl_unique_id(unsigned char* id128) {
  if (!id128) return MXM_DG_EINVAL;
  try {
    ncclUniqueId id;
    mxm::nck(mxm::nccl_api().get_unique_id(&id), "ncclGetUniqueId");
    static_assert(sizeof(id) == 128, "ncclUniqueId is 128 bytes");
    std::memcpy(id128, &id, sizeof(id));
    return MXM_DG_OK;
  } catch (std::exception& ex) {
    return create_error(ex, MXM_DG_EINVAL);
  }
}

int mxm_dg_slab_connect_nccl(void* handle, const unsigned char* id128) {
  SLAB_BEGIN
  if (!id128) throw mxm::ArgError("id128 must be non-null");
  if (h->nccl) throw mxm::ArgError("this part is connected already");
  ncclUniqueId id;
  std::memcpy(&id, id128, sizeof(id));
  std::unique_ptr<mxm::NcclLink> link(new mxm::NcclLink);
  mxm::nck(mxm::nccl_api().comm_init_rank(&link->comm, h->nparts, id, h->part), "ncclCommInitRank");
  h->nccl = link.release();
  SLAB_END
}

int mxm_dg_group_create(void* const* handles, int n, void** out) {
  if (!out) return MXM_DG_EINVAL;
  *out = nullptr;
  try {
    if (!handles || n < 1) throw mxm::ArgError("need n >= 1 handles");
    std::unique_ptr<Group> g(new Group);
    for (int r = 0; r < n; ++r) {
      Handle* h = (Handle*)handles[r];
      if (!h) throw mxm::ArgError("null handle");
      if (h->nparts != n || h->part != r) throw mxm::ArgError("handles must be parts 0..n-1 of one n-part slab decomposition, in order");
      const Handle* h0 = (Handle*)handles[0];
      if (h->P != h0->P || h->prec != h0->prec || h->NC != h0->NC || h->nx != h0->nx || h->ny != h0->ny ||
          h->nzg != h0->nzg || h->phys.kind != h0->phys.kind)
        throw mxm::ArgError("the parts differ in order, precision, physics or mesh");
      if (h->nccl) throw mxm::ArgError("a part connected to NCCL cannot join an in-process group");
      g->parts.push_back(h);
    }
    // Direct NVLink copies between the parts' GPUs where possible.  The
    // parts' state buffers come from each device's default memory pool
    // (stream-ordered allocation), whose access from other devices is set on
    // the pool (cudaMemPoolSetAccess); peer access of the contexts covers
    // cudaMalloc'd memory only, so both are granted.
    for (Handle* h : g->parts) {
      CK(cudaSetDevice(h->device));
      for (Handle* o : g->parts) {
        int can = 0;
        if (o->device != h->device && cudaDeviceCanAccessPeer(&can, h->device, o->device) == cudaSuccess && can) {
          const cudaError_t e = cudaDeviceEnablePeerAccess(o->device, 0);
          if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
          else CK(e);
          cudaMemPool_t pool;  // o's pool, readable and writable from h's device
          CK(cudaDeviceGetDefaultMemPool(&pool, o->device));
          cudaMemAccessDesc ad{};
          ad.location.type = cudaMemLocationTypeDevice;
          ad.location.id = h->device;
          ad.flags = cudaMemAccessFlagsProtReadWrite;
          CK(cudaMemPoolSetAccess(pool, &ad, 1));
        }
      }
      cudaEvent_t ev;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      g->ev.push_back(ev);
    }
    *out = g.release();
    return MXM_DG_OK;
  } catch (mxm::CudaError& ex) {
    return create_error(ex, MXM_DG_ECUDA);
  } catch (std::exception& ex) {
    return create_error(ex, MXM_DG_EINVAL);
  }
}

// Arguments every group step entry checks before it launches anything.
static void group_step_args(const Group* g, int nsteps) {
  if (nsteps < 0) throw mxm::ArgError("nsteps must be >= 0");
  for (Handle* h : g->parts)
    if (h->lim_on != g->parts[0]->lim_on) throw mxm::ArgError("the parts must agree on the limiter");
}

int mxm_dg_group_step_n(void* group, double dt, int nsteps) {
  Group* g = (Group*)group;
  if (!g) return MXM_DG_EINVAL;
  try {
    group_step_args(g, nsteps);
    g->step_n(dt, nsteps);
    return MXM_DG_OK;
  } catch (mxm::CudaError& ex) {
    g->err = ex.what();
    return MXM_DG_ECUDA;
  } catch (std::exception& ex) {
    g->err = ex.what();
    return MXM_DG_EINVAL;
  }
}

// Device time of `nsteps` group steps: every part's stream starts after an
// event on part 0's stream and part 0's stream waits for every part at the
// end, so the two timing events bracket all parts' work.
int mxm_dg_group_time_steps(void* group, double dt, int nsteps, double* ms) {
  Group* g = (Group*)group;
  if (!g || !ms) return MXM_DG_EINVAL;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  try {
    group_step_args(g, nsteps);
    Handle* h0 = g->parts[0];
    CK(cudaSetDevice(h0->device));
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    g->barrier();  // part 0's stream waits for its neighbours' work so far
    for (size_t r = 1; r < g->parts.size(); ++r) {
      CK(cudaSetDevice(g->parts[r]->device));
      CK(cudaEventRecord(g->ev[r], g->parts[r]->stream));
      CK(cudaSetDevice(h0->device));
      CK(cudaStreamWaitEvent(h0->stream, g->ev[r], 0));
    }
    CK(cudaSetDevice(h0->device));
    CK(cudaEventRecord(t0, h0->stream));
    for (size_t r = 1; r < g->parts.size(); ++r) {
      CK(cudaSetDevice(g->parts[r]->device));
      CK(cudaStreamWaitEvent(g->parts[r]->stream, t0, 0));
    }
    g->step_n(dt, nsteps);
    for (size_t r = 1; r < g->parts.size(); ++r) {
      CK(cudaSetDevice(g->parts[r]->device));
      CK(cudaEventRecord(g->ev[r], g->parts[r]->stream));
      CK(cudaSetDevice(h0->device));
      CK(cudaStreamWaitEvent(h0->stream, g->ev[r], 0));
    }
    CK(cudaSetDevice(h0->device));
    CK(cudaEventRecord(t1, h0->stream));
    CK(cudaEventSynchronize(t1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, t0, t1));
    *ms = f;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return MXM_DG_OK;
  } catch (mxm::CudaError& ex) {
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    g->err = ex.what();
    return MXM_DG_ECUDA;
  } catch (std::exception& ex) {
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    g->err = ex.what();
    return MXM_DG_EINVAL;
  }
}

int mxm_dg_group_synchronize(void* group) {
  Group* g = (Group*)group;
  if (!g) return MXM_DG_EINVAL;
  for (Handle* h : g->parts) {
    cudaSetDevice(h->device);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      g->err = cudaGetErrorString(e);
      return MXM_DG_ECUDA;
    }
  }
  return MXM_DG_OK;
}

int mxm_dg_group_last_error(void* group, char* buf, int len) {
  Group* g = (Group*)group;
  if (!g || !buf || len <= 0) return MXM_DG_EINVAL;
  std::snprintf(buf, size_t(len), "%s", g->err.c_str());
  return MXM_DG_OK;
}

int mxm_dg_group_destroy(void* group) {
  Group* g = (Group*)group;
  if (!g) return MXM_DG_OK;
  for (size_t r = 0; r < g->parts.size(); ++r) {
    cudaSetDevice(g->parts[r]->device);
    cudaStreamSynchronize(g->parts[r]->stream);
    cudaEventDestroy(g->ev[r]);
  }
  delete g;
  return MXM_DG_OK;
}

}  // extern "C"
