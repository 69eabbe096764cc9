// Batched engine of the C ABI (mxm_dg_batch_*): many independent solves of
// uneven mesh size and order advanced together, the whole SSPRK3 step
// (counter resets, stage kernels, limiter passes) captured once in a CUDA
// graph and replayed.
//  * 2D solves: one persistent stage launch per physics group and stage;
//    tile sizes (cells per tile) per (group, P) come from an autotuner that
//    times the batched stage kernel on the batch's own solves.
//  * 3D solves on the tensor-core stage (MIXED, MIXED_TF32): one launch per
//    (physics, order, operand kind) group and stage over the tiles of all
//    its solves (stage3d_tc_kernel's batched form); their limiter passes are
//    the single-solve ones, one pair per limited solve.
//  * other 3D solves (FP32 / FP64 SIMT stage): their single-solve launches,
//    in the same graph.
// Every solve gets its single-solve arithmetic, so batched results are
// bit-identical to the same solves stepped alone.
//
// The reference has no batching: each 2D solve runs its own driver loop
// (examples/euler_sod_2d_gpu.mojo, src/ssprk3.mojo:56-78).  Member solves are
// ordinary solver handles; their state stays in their own buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "batch2d.cuh"
#include "batch2d_launch.hpp"
#include "handle.hpp"
#include "ic.hpp"

namespace mxm {

struct BatchGroup {
  mxm_dg_physics_desc phys{};
  int NC = 0;
  int dim = 2;
  // 3D: tc = batched tensor-core tiles of order P and operand kind `kind`;
  // otherwise the members' single-solve launches
  bool tc = false;
  int P = 0, kind = 0;
  Stage3DArgs<float>* d_margs = nullptr;  // [3][members]: stage arguments
  KuhnTab3<float>* d_tabs = nullptr;      // [members]
  std::vector<int> members;  // indices into Batch::members
  int ec[6] = {0, 0, 0, 0, 0, 0};
  int4* d_items = nullptr;
  int nitems = 0;
  int4* d_litems = nullptr;  // limiter chunks of the limited members
  int nlitems = 0;
  int* d_counter = nullptr;  // [3]: one work counter per stage
  size_t smem = 0;
  int grid = 0;
  int qv = 0, a_len = 0, aoff[6] = {0, 0, 0, 0, 0, 0};
  const void* A[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// The limited 3D members of one component count: their cell-mean and theta
// passes as one launch each per stage, over chunks of kLim3Chunk elements.
struct Lim3Group {
  int NC = 0;
  std::vector<int> members;
  void* d_desc = nullptr;  // LimDesc3<R>[members]
  int4* d_items = nullptr;
  int nitems = 0;
};

struct Batch {
  int device = 0, nsm = 148;
  std::vector<Lim3Group> lim3;
  // the groups' stage launches of one stage run side by side on these
  // streams (fork / join by events inside the captured step)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev_side;
  cudaEvent_t ev_fork = nullptr;
  cudaStream_t stream = nullptr;
  size_t rbytes = 0;
  std::vector<Handle*> members;
  std::vector<double> dt;
  std::vector<BatchGroup> groups;
  void* d_solves = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool built = false, tuned = false;
  int* derr = nullptr;
  std::string err;
};

namespace {

constexpr int kLimChunk = 128;      // elements per limiter block
constexpr size_t kSmemCap = 200 * 1024;
const int kEcCandidates[] = {1, 2, 4, 8, 16, 32, 64};

size_t tab_bytes(size_t rb) {
  return rb == 8 ? (sizeof(KuhnTab2<double>) + 15) / 16 * 16 : (sizeof(KuhnTab2<float>) + 15) / 16 * 16;
}
int ntri_h(int P) { return (P + 1) * (P + 2) / 2; }
int klen2d(int P) { return 2 * ntri_h(P) + 3 * (P + 1); }

void release_graph(Batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->built = false;
}

void free_lim3(Batch* b) {
  for (auto& lg : b->lim3) {
    cudaFree(lg.d_desc);
    cudaFree(lg.d_items);
  }
  b->lim3.clear();
}

// component counts the batched 3D limiter is built for (the 17-component
// two-fluid state keeps its single-solve limiter launches)
bool lim3_batched_nc(int nc) { return nc == 1 || nc == 3 || nc == 5 || nc == 6 || nc == 9; }

template <class R>
void build_lim3(Batch* b) {
  free_lim3(b);
  for (size_t i = 0; i < b->members.size(); ++i) {
    const Handle* h = b->members[i];
    if (h->dim != 3 || !h->lim_on || !lim3_batched_nc(h->NC)) continue;
    Lim3Group* lg = nullptr;
    for (auto& x : b->lim3)
      if (x.NC == h->NC) lg = &x;
    if (!lg) {
      b->lim3.emplace_back();
      lg = &b->lim3.back();
      lg->NC = h->NC;
    }
    lg->members.push_back(int(i));
  }
  for (auto& lg : b->lim3) {
    std::vector<LimDesc3<R>> desc(lg.members.size());
    std::vector<int4> items;
    for (size_t j = 0; j < lg.members.size(); ++j) {
      const Handle* h = b->members[lg.members[j]];
      LimDesc3<R>& d = desc[j];
      std::memset(&d, 0, sizeof(d));
      d.a.avg = (R*)h->avg;
      d.a.w = (const R*)h->w;
      d.a.ne = h->ne;
      d.a.e0 = 0;
      d.a.e1 = h->ne;
      d.a.nx = h->nx; d.a.ny = h->ny; d.a.nz = h->nz;
      for (int k = 0; k < 6; ++k) d.a.bc[k] = h->bc[k];
      if (sizeof(R) == 4) {
        const float ef = float(h->lim_eps);  // as the single-solve limiter: eps2 = eps*eps in FP32
        d.a.eps2 = R(ef * ef);
      } else {
        d.a.eps2 = R(h->lim_eps * h->lim_eps);
      }
      for (int k = 0; k < 3; ++k) d.qs[k] = (R*)h->q[k];
      d.tab = sizeof(R) == 8 ? reinterpret_cast<const KuhnTab3<R>&>(h->t3d) : reinterpret_cast<const KuhnTab3<R>&>(h->t3f);
      d.P = h->P;
      for (int64_t e0 = 0; e0 < h->ne; e0 += kLim3Chunk)
        items.push_back(make_int4(int(j), int(e0), int(std::min<int64_t>(kLim3Chunk, h->ne - e0)), 0));
    }
    lg.nitems = int(items.size());
    CK(cudaMalloc(&lg.d_desc, desc.size() * sizeof(LimDesc3<R>)));
    CK(cudaMemcpy(lg.d_desc, desc.data(), desc.size() * sizeof(LimDesc3<R>), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&lg.d_items, items.size() * sizeof(int4)));
    CK(cudaMemcpy(lg.d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  }
}

template <class R, int NC>
cudaError_t lim3_launch_nc(const Lim3Group& lg, int which, cudaStream_t st) {
  const LimBatch3<R> lb{(const LimDesc3<R>*)lg.d_desc, lg.d_items, lg.nitems, which};
  avg3d_batch_kernel<R, NC><<<lg.nitems, 256, 0, st>>>(lb);
  theta3d_batch_kernel<R, NC><<<lg.nitems, 32 * kLim3Epb, 0, st>>>(lb);
  return cudaGetLastError();
}

template <class R>
cudaError_t lim3_launch(const Lim3Group& lg, int which, cudaStream_t st) {
  if (lg.nitems <= 0) return cudaSuccess;
  switch (lg.NC) {
    case 1: return lim3_launch_nc<R, 1>(lg, which, st);
    case 3: return lim3_launch_nc<R, 3>(lg, which, st);
    case 5: return lim3_launch_nc<R, 5>(lg, which, st);
    case 6: return lim3_launch_nc<R, 6>(lg, which, st);
    case 9: return lim3_launch_nc<R, 9>(lg, which, st);
  }
  return cudaErrorInvalidValue;
}

void free_group(BatchGroup& g) {
  cudaFree(g.d_items);
  cudaFree(g.d_litems);
  cudaFree(g.d_counter);
  cudaFree(g.d_margs);
  cudaFree(g.d_tabs);
  g.d_items = g.d_litems = nullptr;
  g.d_counter = nullptr;
  g.d_margs = nullptr;
  g.d_tabs = nullptr;
}

// During the capture of the step the 3D members' single-solve launches go to
// the batch stream (the members are idle while the batch owns them).
struct StreamSwap {
  std::vector<std::pair<Handle*, cudaStream_t>> saved;
  StreamSwap(Batch* b) {
    for (Handle* h : b->members)
      if (h->dim == 3) {
        saved.emplace_back(h, h->stream);
        h->stream = b->stream;
      }
  }
  ~StreamSwap() {
    for (auto& p : saved) p.first->stream = p.second;
  }
};

// Order of a 3D tensor-core group's tiles.  The batched kernel gives block
// b the contiguous item range [b n / G, (b + 1) n / G) of the launch's G
// blocks, so that a block rarely changes solve.  Within each solve's span
// the tiles are laid out so that, at every step k of the blocks' loops, the
// blocks working on that solve take consecutive tiles (the order of the
// single-solve kernel, whose blocks take every G-th tile): neighbouring
// tiles, whose y / z neighbour rows overlap, are then loaded together and
// stay in L2.  Each tile's arithmetic does not depend on the order.
void order_tc3_items(const Handle* h0, std::vector<int4>& items) {
  const int64_t n = int64_t(items.size());
  int G = 0;
  if (n < 2 || tc_group_grid(h0, int(n), &G) != cudaSuccess || G < 2) {
    cudaGetLastError();
    return;
  }
  std::vector<int> owner(size_t(n), 0), step(size_t(n), 0);
  for (int blk = 0; blk < G; ++blk)
    for (int64_t p = int64_t(blk) * n / G, hi = int64_t(blk + 1) * n / G, p0 = p; p < hi; ++p) {
      owner[size_t(p)] = blk;
      step[size_t(p)] = int(p - p0);
    }
  std::vector<int4> out(items.size());
  std::vector<int64_t> pos;
  for (int64_t s0 = 0; s0 < n;) {
    int64_t s1 = s0;
    while (s1 < n && items[size_t(s1)].x == items[size_t(s0)].x) ++s1;
    pos.resize(size_t(s1 - s0));
    for (int64_t p = s0; p < s1; ++p) pos[size_t(p - s0)] = p;
    std::stable_sort(pos.begin(), pos.end(), [&](int64_t a, int64_t c) {
      return step[size_t(a)] != step[size_t(c)] ? step[size_t(a)] < step[size_t(c)] : owner[size_t(a)] < owner[size_t(c)];
    });
    for (int64_t i = 0; i < s1 - s0; ++i) out[size_t(pos[size_t(i)])] = items[size_t(s0 + i)];
    s0 = s1;
  }
  items.swap(out);
}

// Tiles {member of the group, first cell, cells, 0} and per-stage arguments
// of a 3D tensor-core group.
void build_tc3(Batch* b, BatchGroup& g) {
  const int ng = int(g.members.size());
  const Handle* h0 = b->members[g.members[0]];
  const int ec = tc_tile_cubes(g.P, h0->NC, g.kind);
  if (ec < 1) throw ArgError("no tensor-core tile for this order and component count");
  std::vector<int4> items;
  std::vector<Stage3DArgs<float>> margs(size_t(3) * ng);
  std::vector<KuhnTab3<float>> tabs(ng);
  for (int j = 0; j < ng; ++j) {
    Handle* h = b->members[g.members[j]];
    for (int64_t c0 = h->cbeg; c0 < h->cend; c0 += ec)
      items.push_back(make_int4(j, int(c0), int(std::min<int64_t>(ec, h->cend - c0)), 0));
    for (int st = 0; st < 3; ++st) margs[size_t(st) * ng + j] = tc_stage_args(h, st, b->dt[g.members[j]], b->derr);
    tabs[j] = h->t3f;
  }
  order_tc3_items(h0, items);
  g.ec[g.P] = ec;
  g.nitems = int(items.size());
  CK(cudaMalloc(&g.d_items, std::max<size_t>(1, items.size()) * sizeof(int4)));
  CK(cudaMemcpy(g.d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&g.d_margs, margs.size() * sizeof(Stage3DArgs<float>)));
  CK(cudaMemcpy(g.d_margs, margs.data(), margs.size() * sizeof(Stage3DArgs<float>), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&g.d_tabs, tabs.size() * sizeof(KuhnTab3<float>)));
  CK(cudaMemcpy(g.d_tabs, tabs.data(), tabs.size() * sizeof(KuhnTab3<float>), cudaMemcpyHostToDevice));
}

template <class R>
void upload_solves(Batch* b) {
  std::vector<SolveDesc2<R>> sd(b->members.size());
  for (size_t i = 0; i < b->members.size(); ++i) {
    const Handle* h = b->members[i];
    SolveDesc2<R>& d = sd[i];
    std::memset(&d, 0, sizeof(d));
    d.tab = h->rbytes == 8 ? reinterpret_cast<const KuhnTab2<R>&>(h->t2d) : reinterpret_cast<const KuhnTab2<R>&>(h->t2f);
    for (int k = 0; k < 3; ++k) d.q[k] = (R*)h->q[k];
    d.avg = (R*)h->avg;
    d.w = (const R*)h->w;
    const double cs[3] = {1.0, 0.25, 2.0 / 3.0};
    for (int s = 0; s < 3; ++s) d.cdt[s] = R(cs[s] * b->dt[i]);
    if (sizeof(R) == 4) {
      const float ef = float(h->lim_eps);  // as the single-solve limiter: eps2 = eps*eps in FP32
      d.eps2 = R(ef * ef);
    } else {
      d.eps2 = R(h->lim_eps * h->lim_eps);
    }
    d.P = h->P;
    d.nx = h->nx;
    d.ny = h->ny;
    d.ncell = int(h->ncell);
    for (int k = 0; k < 4; ++k) d.bc[k] = h->bc[k];
    d.limiter = h->lim_on ? 1 : 0;
  }
  cudaFree(b->d_solves);
  b->d_solves = nullptr;
  CK(cudaMalloc(&b->d_solves, sd.size() * sizeof(SolveDesc2<R>)));
  CK(cudaMemcpy(b->d_solves, sd.data(), sd.size() * sizeof(SolveDesc2<R>), cudaMemcpyHostToDevice));
}

// tile items {solve, first cell, cells, P} of the group's members whose order
// is in `onlyP` (0 = all), heaviest P first
std::vector<int4> make_items(const Batch* b, const BatchGroup& g, const int* ec, int onlyP) {
  std::vector<int4> it;
  for (int P = 5; P >= 1; --P) {
    if (onlyP && P != onlyP) continue;
    for (int m : g.members) {
      const Handle* h = b->members[m];
      if (h->P != P) continue;
      const int E = ec[P];
      for (int c0 = 0; c0 < int(h->ncell); c0 += E) it.push_back(make_int4(m, c0, std::min(E, int(h->ncell) - c0), P));
    }
  }
  return it;
}

// shared-memory layout of the group's stage kernel for tile sizes ec[]
void layout(const Batch* b, BatchGroup& g, const int* ec) {
  bool present[6] = {false, false, false, false, false, false};
  for (int m : g.members) present[b->members[m]->P] = true;
  int off = 0, qv = 0, bmax = 0;
  for (int P = 1; P <= 5; ++P) {
    g.aoff[P] = 0;
    g.A[P] = nullptr;
    if (!present[P]) continue;
    g.aoff[P] = off;
    off += klen2d(P) * ntri_h(P);
    for (int m : g.members)
      if (b->members[m]->P == P) {
        g.A[P] = b->members[m]->A;
        break;
      }
    qv = std::max(qv, 2 * ec[P] * ntri_h(P) * g.NC);
    bmax = std::max(bmax, 2 * ec[P] * bstr2d(P, g.NC, b->rbytes));
  }
  g.a_len = (off + 3) / 4 * 4;
  g.qv = (qv + 3) / 4 * 4;
  g.smem = 32 + 2 * tab_bytes(b->rbytes) + size_t(g.a_len + 2 * g.qv + bmax) * b->rbytes;
}

template <class R>
Batch2DArgs<R> stage_args(const Batch* b, const BatchGroup& g, const int4* items, int nitems, int stage) {
  Batch2DArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.solves = (const SolveDesc2<R>*)b->d_solves;
  a.items = items;
  a.nitems = nitems;
  a.counter = g.d_counter + stage;
  a.stage = stage;
  for (int P = 0; P < 6; ++P) {
    a.A[P] = (const R*)g.A[P];
    a.aoff[P] = g.aoff[P];
  }
  a.a_len = g.a_len;
  a.qv = g.qv;
  a.err = b->derr;
  return a;
}

template <class R>
cudaError_t launch_group_stage(const Batch* b, const BatchGroup& g, const int4* items, int nitems, int stage,
                               int grid, size_t smem, cudaStream_t st = nullptr) {
  const Batch2DArgs<R> a = stage_args<R>(b, g, items, nitems, stage);
  return launch_stage2d_batch<R>(g.phys, a, grid, smem, st ? st : b->stream);
}

template <class R>
int grid_for(const Batch* b, const BatchGroup& g, size_t smem, int nitems) {
  int bps = 1;
  CK(stage2d_batch_blocks_per_sm<R>(g.phys, smem, &bps));
  int grid = b->nsm * bps;
  if (grid > nitems) grid = nitems;
  return grid < 1 ? 1 : grid;
}

// Autotune the cells per tile of every (group, P): time stage 0 of the
// group's members of that order (it writes only their q1 buffers) for each
// candidate that fits the shared-memory cap, keep the fastest.
template <class R>
void autotune(Batch* b) {
  upload_solves<R>(b);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (auto& g : b->groups) {
    if (g.dim == 3) continue;  // 3D tiles are fixed by the tensor-core shape
    if (!g.d_counter) CK(cudaMalloc(&g.d_counter, 3 * sizeof(int)));
    for (int P = 1; P <= 5; ++P) {
      bool any = false;
      for (int m : g.members) any = any || b->members[m]->P == P;
      if (!any) continue;
      double best = 1e30;
      int best_ec = 1;
      for (int E : kEcCandidates) {
        int ec[6] = {0, 0, 0, 0, 0, 0};
        ec[P] = E;
        BatchGroup t = g;  // shallow copy for the layout of this trial
        t.d_items = nullptr;
        layout(b, t, ec);
        if (t.smem > kSmemCap) continue;
        std::vector<int4> items = make_items(b, t, ec, P);
        int4* d_items = nullptr;
        CK(cudaMalloc(&d_items, items.size() * sizeof(int4)));
        CK(cudaMemcpy(d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
        const int grid = grid_for<R>(b, t, t.smem, int(items.size()));
        float tot = 0.f;
        for (int rep = 0; rep < 4; ++rep) {
          CK(cudaMemsetAsync(g.d_counter, 0, 3 * sizeof(int), b->stream));
          CK(cudaEventRecord(e0, b->stream));
          CK(launch_group_stage<R>(b, t, d_items, int(items.size()), 0, grid, t.smem));
          CK(cudaEventRecord(e1, b->stream));
          CK(cudaEventSynchronize(e1));
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          if (rep > 0) tot += ms;  // first launch warms up
        }
        cudaFree(d_items);
        if (tot < best) {
          best = tot;
          best_ec = E;
        }
      }
      g.ec[P] = best_ec;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuned = true;
}

template <class R>
void build(Batch* b) {
  release_graph(b);
  upload_solves<R>(b);
  for (auto& g : b->groups) {
    free_group(g);
    if (g.dim == 3) {
      if (g.tc) build_tc3(b, g);
      continue;
    }
    layout(b, g, g.ec);
    std::vector<int4> items = make_items(b, g, g.ec, 0);
    g.nitems = int(items.size());
    CK(cudaMalloc(&g.d_items, std::max<size_t>(1, items.size()) * sizeof(int4)));
    CK(cudaMemcpy(g.d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    std::vector<int4> lit;
    for (int m : g.members) {
      const Handle* h = b->members[m];
      if (!h->lim_on) continue;
      for (int64_t e0 = 0; e0 < h->ne; e0 += kLimChunk)
        lit.push_back(make_int4(m, int(e0), int(std::min<int64_t>(kLimChunk, h->ne - e0)), h->P));
    }
    g.nlitems = int(lit.size());
    if (!lit.empty()) {
      CK(cudaMalloc(&g.d_litems, lit.size() * sizeof(int4)));
      CK(cudaMemcpy(g.d_litems, lit.data(), lit.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&g.d_counter, 3 * sizeof(int)));
    g.grid = grid_for<R>(b, g, g.smem, g.nitems);
  }
  for (auto& g : b->groups)
    if (g.dim == 2 && g.nlitems > 0) CK(prepare_lim2d_batch<R>(g.NC));
  build_lim3<R>(b);
  // first-use set-up of the batched 3D kernels (kernel attributes,
  // occupancy) before the capture: an empty batch launches nothing
  for (auto& g : b->groups)
    if (g.dim == 3 && g.tc) {
      const Tc3Batch none{g.d_margs, g.d_tabs, g.d_items, 0};
      CK(launch_tc_group(b->members[g.members[0]], none, b->stream));
    }
  // side streams for the groups of a stage (a group's launch underfills the
  // GPU when its solves are few or small; groups of one stage are
  // independent)
  const int nside = int(std::min<size_t>(b->groups.size(), 8));
  while (int(b->side.size()) < nside) {
    cudaStream_t st;
    cudaEvent_t ev;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->side.push_back(st);
    b->ev_side.push_back(ev);
  }
  if (!b->ev_fork) CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  // one SSPRK3 step as a graph
  StreamSwap swap(b);
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t cap = cudaSuccess;
  for (auto& g : b->groups)
    if (cap == cudaSuccess && g.dim == 2) cap = cudaMemsetAsync(g.d_counter, 0, 3 * sizeof(int), b->stream);
  for (int s = 0; s < 3 && cap == cudaSuccess; ++s) {
    // fork: the batched group launches of the stage on the side streams
    const bool fork = nside > 1;
    if (fork) {
      cap = cudaEventRecord(b->ev_fork, b->stream);
      for (int i = 0; i < nside && cap == cudaSuccess; ++i) cap = cudaStreamWaitEvent(b->side[i], b->ev_fork, 0);
    }
    int gi = 0;
    for (auto& g : b->groups) {
      if (cap != cudaSuccess) break;
      cudaStream_t st = fork ? b->side[gi++ % nside] : b->stream;
      if (g.dim == 2) {
        cap = launch_group_stage<R>(b, g, g.d_items, g.nitems, s, g.grid, g.smem, st);
      } else if (g.tc) {
        const Tc3Batch bat{g.d_margs + size_t(s) * g.members.size(), g.d_tabs, g.d_items, g.nitems};
        cap = launch_tc_group(b->members[g.members[0]], bat, st);
      } else {  // single-solve launches on the batch stream
        try {
          for (int m : g.members) stage_only(b->members[m], s, b->dt[m]);
        } catch (CudaError& ex) {
          cap = ex.e;
        }
      }
    }
    if (fork) {  // join before the limiter passes
      for (int i = 0; i < nside && cap == cudaSuccess; ++i) {
        cap = cudaEventRecord(b->ev_side[i], b->side[i]);
        if (cap == cudaSuccess) cap = cudaStreamWaitEvent(b->stream, b->ev_side[i], 0);
      }
    }
    // 3D limiter passes: batched per component count; the two-fluid state
    // keeps its single-solve launches
    for (auto& lg : b->lim3)
      if (cap == cudaSuccess) cap = lim3_launch<R>(lg, stage_out(s), b->stream);
    for (auto& g : b->groups) {
      if (cap != cudaSuccess || g.dim != 3) continue;
      try {
        for (int m : g.members)
          if (b->members[m]->lim_on && !lim3_batched_nc(b->members[m]->NC))
            limit_buf(b->members[m], b->members[m]->q[stage_out(s)]);
      } catch (CudaError& ex) {
        cap = ex.e;
      }
    }
    for (auto& g : b->groups) {
      if (cap != cudaSuccess || g.dim != 2 || g.nlitems == 0) continue;
      LimBatch2DArgs<R> la;
      la.solves = (const SolveDesc2<R>*)b->d_solves;
      la.items = g.d_litems;
      la.nitems = g.nlitems;
      la.which = s == 0 ? 1 : (s == 1 ? 2 : 0);
      cap = launch_lim2d_batch<R>(g.NC, la, b->stream);
    }
  }
  // 2D GLM-MHD members: psi *= exp(-alpha_d dt) after the step, each with its own dt
  for (size_t i = 0; i < b->members.size() && cap == cudaSuccess; ++i) {
    const Handle* h = b->members[i];
    if (!glm_damped(h)) continue;
    cap = launch_scale_component(h->q[0], h->rbytes, h->ne * h->NP, h->NC, h->NC - 1, psi_decay(h, b->dt[i]),
                                 b->stream);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->stream, &graph);
  if (cap != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    throw CudaError(cap, "batched step capture");
  }
  CK(end);
  b->graph = graph;
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->built = true;
}

void ensure_built(Batch* b) {
  if (b->built) return;
  if (b->members.empty()) throw ArgError("the batch has no solves");
  // members must be idle before the batch stream uses their buffers
  for (Handle* h : b->members) CK(cudaStreamSynchronize(h->stream));
  if (b->rbytes == 8) {
    if (!b->tuned) autotune<double>(b);
    build<double>(b);
  } else {
    if (!b->tuned) autotune<float>(b);
    build<float>(b);
  }
}

void run_steps(Batch* b, int n) {
  for (int k = 0; k < n; ++k) CK(cudaGraphLaunch(b->exec, b->stream));
}

}  // namespace
}  // namespace mxm

using mxm::Batch;

#define BATCH_BEGIN                 \
  Batch* b = (Batch*)batch;         \
  if (!b) return MXM_DG_EINVAL;     \
  try {                             \
    cudaSetDevice(b->device);
#define BATCH_END                                                                \
  return MXM_DG_OK;                                                              \
  }                                                                              \
  catch (mxm::CudaError & ex) {                                                  \
    b->err = ex.what();                                                          \
    return ex.e == cudaErrorMemoryAllocation ? MXM_DG_ENOMEM : MXM_DG_ECUDA;     \
  }                                                                              \
  catch (std::exception & ex) {                                                  \
    b->err = ex.what();                                                          \
    return MXM_DG_EINVAL;                                                        \
  }

extern "C" {

int mxm_dg_batch_create(void** batch) {
  if (!batch) return MXM_DG_EINVAL;
  *batch = nullptr;
  std::unique_ptr<Batch> b(new Batch);
  if (cudaGetDevice(&b->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->derr, sizeof(int)) != cudaSuccess || cudaMemset(b->derr, 0, sizeof(int)) != cudaSuccess) {
    std::lock_guard<std::mutex> g(mxm::g_err_mu);
    mxm::g_create_err = "batch create: CUDA setup failed";
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaFree(b->derr);
    return MXM_DG_ECUDA;
  }
  *batch = b.release();
  return MXM_DG_OK;
}

int mxm_dg_batch_destroy(void* batch) {
  Batch* b = (Batch*)batch;
  if (!b) return MXM_DG_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  mxm::release_graph(b);
  for (auto& g : b->groups) mxm::free_group(g);
  mxm::free_lim3(b);
  for (size_t i = 0; i < b->side.size(); ++i) {
    cudaStreamDestroy(b->side[i]);
    cudaEventDestroy(b->ev_side[i]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  cudaFree(b->d_solves);
  cudaFree(b->derr);
  cudaStreamDestroy(b->stream);
  delete b;
  return MXM_DG_OK;
}

int mxm_dg_batch_add(void* batch, void* solver, double dt, int32_t* index) {
  BATCH_BEGIN
  mxm::Handle* h = (mxm::Handle*)solver;
  if (!h) throw mxm::ArgError("null solver handle");
  if (h->nparts > 1) throw mxm::ArgError("slab parts step through their group, not a batch");
  if (h->device != b->device) throw mxm::ArgError("solver lives on another device than the batch");
  if (!(dt > 0.0)) throw mxm::ArgError("dt must be positive");
  if (b->rbytes && h->rbytes != b->rbytes) throw mxm::ArgError("all solves of a batch share one precision");
  for (mxm::Handle* m : b->members)
    if (m == h) throw mxm::ArgError("solver already in the batch");
  b->rbytes = h->rbytes;
  const int id = int(b->members.size());
  b->members.push_back(h);
  b->dt.push_back(dt);
  // groups: 2D by physics; 3D tensor-core by (physics, order, operand
  // kind); the other 3D solves by physics
  const bool tc = h->dim == 3 && h->use_tc;
  int gi = -1;
  for (size_t k = 0; k < b->groups.size(); ++k) {
    const mxm::BatchGroup& g = b->groups[k];
    if (g.dim == h->dim && g.tc == tc && std::memcmp(&g.phys, &h->phys, sizeof(h->phys)) == 0 &&
        (!tc || (g.P == h->P && g.kind == h->tc_kind)))
      gi = int(k);
  }
  if (gi < 0) {
    b->groups.emplace_back();
    mxm::BatchGroup& g = b->groups.back();
    g.phys = h->phys;
    g.NC = h->NC;
    g.dim = h->dim;
    g.tc = tc;
    g.P = tc ? h->P : 0;
    g.kind = tc ? h->tc_kind : 0;
    gi = int(b->groups.size()) - 1;
  }
  b->groups[gi].members.push_back(id);
  mxm::release_graph(b);
  b->tuned = false;
  if (index) *index = id;
  BATCH_END
}

int mxm_dg_batch_autotune(void* batch) {
  BATCH_BEGIN
  if (b->members.empty()) throw mxm::ArgError("the batch has no solves");
  for (mxm::Handle* h : b->members) CK(cudaStreamSynchronize(h->stream));
  mxm::release_graph(b);
  if (b->rbytes == 8) mxm::autotune<double>(b);
  else mxm::autotune<float>(b);
  CK(cudaStreamSynchronize(b->stream));
  BATCH_END
}

int mxm_dg_batch_tile_cells(void* batch, int member, int32_t* cells) {
  BATCH_BEGIN
  if (member < 0 || member >= int(b->members.size()) || !cells) throw mxm::ArgError("member index out of range");
  mxm::ensure_built(b);
  for (auto& g : b->groups)
    for (int m : g.members)
      if (m == member) *cells = g.ec[b->members[m]->P];
  BATCH_END
}

int mxm_dg_batch_step(void* batch, int nsteps) {
  BATCH_BEGIN
  if (nsteps < 0) throw mxm::ArgError("nsteps >= 0");
  mxm::ensure_built(b);
  mxm::run_steps(b, nsteps);
  BATCH_END
}

int mxm_dg_batch_time_steps(void* batch, int nsteps, double* ms) {
  BATCH_BEGIN
  if (nsteps < 0 || !ms) throw mxm::ArgError("nsteps >= 0, ms non-null");
  mxm::ensure_built(b);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, b->stream));
  mxm::run_steps(b, nsteps);
  CK(cudaEventRecord(e1, b->stream));
  CK(cudaEventSynchronize(e1));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  BATCH_END
}

int mxm_dg_batch_synchronize(void* batch) {
  BATCH_BEGIN
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  int derr = 0;
  CK(cudaMemcpy(&derr, b->derr, sizeof(int), cudaMemcpyDeviceToHost));
  if (derr) {
    CK(cudaMemset(b->derr, 0, sizeof(int)));
    b->err = "a batched stage kernel's bounded wait for its state tile gave up";
    return MXM_DG_ETIMEDOUT;
  }
  BATCH_END
}

int mxm_dg_batch_dof_count(void* batch, int64_t* dof) {
  BATCH_BEGIN
  if (!dof) throw mxm::ArgError("dof non-null");
  int64_t n = 0;
  for (mxm::Handle* h : b->members) n += h->ne * h->NP * h->NC;
  *dof = n;
  BATCH_END
}

int mxm_dg_batch_launches_per_step(void* batch, int32_t* n) {
  BATCH_BEGIN
  if (!n) throw mxm::ArgError("n non-null");
  // per stage: one stage kernel per group, plus the two limiter passes of a
  // group with limited members
  // 3D: one batched launch per tensor-core group and stage, one launch per
  // other solve and stage, two limiter launches per component count of the
  // limited solves and stage (two per two-fluid limited solve and stage)
  int k = 0;
  std::vector<int> lim_nc;
  for (auto& g : b->groups) {
    if (g.dim == 3) {
      k += g.tc ? 3 : 3 * int(g.members.size());
      for (int m : g.members) {
        const mxm::Handle* h = b->members[m];
        if (!h->lim_on) continue;
        if (!mxm::lim3_batched_nc(h->NC)) k += 6;
        else if (std::find(lim_nc.begin(), lim_nc.end(), h->NC) == lim_nc.end()) lim_nc.push_back(h->NC);
      }
      continue;
    }
    bool lim = false;
    for (int m : g.members) lim = lim || b->members[m]->lim_on;
    k += 3 * (lim ? 3 : 1);
  }
  k += 6 * int(lim_nc.size());
  for (const mxm::Handle* h : b->members) k += mxm::glm_damped(h) ? 1 : 0;  // psi damping
  *n = k;
  BATCH_END
}

int mxm_dg_batch_last_error(void* batch, char* buf, int len) {
  if (!buf || len <= 0) return MXM_DG_EINVAL;
  std::string s;
  if (batch) s = ((Batch*)batch)->err;
  else {
    std::lock_guard<std::mutex> g(mxm::g_err_mu);
    s = mxm::g_create_err;
  }
  std::strncpy(buf, s.c_str(), size_t(len) - 1);
  buf[len - 1] = '\0';
  return MXM_DG_OK;
}

}  // extern "C"
