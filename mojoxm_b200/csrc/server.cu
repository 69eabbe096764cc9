// Serving loop of the C ABI (mxm_dg_server_*): continuous batching of
// independent solves on one GPU.  The reference has no serving layer; this
// sits on top of the same solver handles the Mojo driver would use.
//
// A scheduler thread owned by the server admits queued requests in arrival
// order while their device footprint fits the HBM budget and a slot is
// free, builds each admitted solve (handle, device IC fill) on its own
// stream, and keeps every running solve's stream fed with chunks of SSPRK3
// steps (at most two chunks in flight per solve), so solves that arrive while
// others run are admitted as memory frees up and their kernels overlap on the
// device.  A finished solve's state goes to the caller's host buffer, its
// memory is released and its latency (submit -> result on the host) is
// recorded.  Each solve's arithmetic is the single-solve arithmetic on its
// own buffers, so results do not depend on what else is running.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "handle.hpp"

namespace mxm {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  mxm_dg_mesh_desc mesh{};
  mxm_dg_physics_desc phys{};
  int P = 1, prec = 0, ic_kind = 0, nparams = 0, limiter = 0;
  double params[32] = {};
  double eps = 0.1, dt = 0.0;
  int nsteps = 0;
  void* out = nullptr;  // caller-owned host buffer (state bytes), may be null
  size_t bytes = 0;     // device footprint estimate
  // runtime
  Handle* h = nullptr;
  int enqueued = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int ev_head = 0, ev_count = 0;
  // one full chunk of SSPRK3 steps as a CUDA graph (captured after the first
  // chunk ran eagerly, replayed for every later full chunk)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  std::string err;
  Clock::time_point t_submit, t_admit, t_done;
  int64_t dof = 0;
};

struct Server {
  int device = 0;
  double budget = 0;
  int max_active = 0, chunk = 10;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  int64_t next_id = 1;
  std::deque<Request*> queue;
  std::vector<Request*> active;
  std::map<int64_t, std::unique_ptr<Request>> all;
  double bytes_in_use = 0, peak_bytes = 0;
  int peak_active = 0;
  std::vector<double> latencies_ms;
  Clock::time_point t_first_submit{}, t_last_done{};
  bool any_submit = false;
  double dof_stages_done = 0;
  std::string err;
};

namespace {

int nc_of(const mxm_dg_physics_desc& p, int dim) {
  return p.kind == MXM_DG_PHYS_ADVECTION ? 1
       : p.kind == MXM_DG_PHYS_EULER     ? (dim == 3 ? 5 : 4)
       : p.kind == MXM_DG_PHYS_MAXWELL   ? 6
       : p.kind == MXM_DG_PHYS_MHD       ? (dim == 3 ? 9 : 7)
       : p.kind == MXM_DG_PHYS_MHD_PLAIN ? 6
       : p.kind == MXM_DG_PHYS_TWO_FLUID ? 17
                                         : 3;
}

// device bytes a solve holds: three state buffers, the limiter means and
// nodal extrema, the operator and weights, plus a small fixed allowance
size_t footprint(const Request& r, int64_t* dof) {
  const int dim = r.mesh.dim, P = r.P;
  const int64_t ncell = int64_t(r.mesh.nx) * r.mesh.ny * (dim == 3 ? r.mesh.nz : 1);
  const int64_t ne = ncell * (dim == 3 ? 6 : 2);
  const int NP = dim == 3 ? (P + 1) * (P + 2) * (P + 3) / 6 : (P + 1) * (P + 2) / 2;
  const int NFP = dim == 3 ? (P + 1) * (P + 2) / 2 : P + 1;
  const int NC = nc_of(r.phys, dim);
  const size_t rb = r.prec == MXM_DG_PREC_F64 ? 8 : 4;
  const int K = dim == 3 ? 3 * NP + 4 * NFP : 2 * NP + 3 * NFP;
  *dof = ne * NP * NC;
  return size_t(3 * ne * NP * NC + ne * (NC + 2 * (dim == 3 ? NC : 1)) + K * NP + NP) * rb + (1 << 16);
}

void finish(Server* s, Request* r, bool ok) {
  // called by the worker without the lock held for the D2H copy
  if (ok && r->out) {
    cudaError_t e = cudaMemcpyAsync(r->out, r->h->q[0], r->h->qbytes(), cudaMemcpyDeviceToHost, r->h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->h->stream);
    if (e != cudaSuccess) {
      ok = false;
      r->err = std::string("result copy: ") + cudaGetErrorString(e);
    }
  } else if (r->h) {
    cudaStreamSynchronize(r->h->stream);
  }
  for (auto& ev : r->ev)
    if (ev) cudaEventDestroy(ev);
  if (r->exec) cudaGraphExecDestroy(r->exec);
  if (r->graph) cudaGraphDestroy(r->graph);
  r->exec = nullptr;
  r->graph = nullptr;
  if (r->h) destroy(r->h);
  r->h = nullptr;
  std::lock_guard<std::mutex> g(s->mu);
  r->t_done = Clock::now();
  r->state = ok ? 2 : 3;
  s->bytes_in_use -= double(r->bytes);
  if (ok) {
    s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
    s->t_last_done = r->t_done;
    s->dof_stages_done += 3.0 * double(r->dof) * r->nsteps;
  }
  s->cv_done.notify_all();
}

bool admit(Server* s, Request* r) {
  try {
    r->h = create(&r->mesh, &r->phys, r->P, r->prec);
    if (r->limiter) {
      r->h->lim_on = true;
      r->h->lim_eps = r->eps;
    }
    fill_ic(r->h, 0, r->ic_kind, r->params, r->nparams);
    for (auto& ev : r->ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return true;
  } catch (std::exception& ex) {
    r->err = ex.what();
    return false;
  }
}

void worker_main(Server* s) {
  cudaSetDevice(s->device);
  std::vector<Request*> finished;
  while (true) {
    std::vector<Request*> to_admit;
    {
      std::unique_lock<std::mutex> g(s->mu);
      if (s->stop) break;
      while (!s->queue.empty() && int(s->active.size() + to_admit.size()) < s->max_active &&
             s->bytes_in_use + double(s->queue.front()->bytes) <= s->budget) {
        Request* r = s->queue.front();
        s->queue.pop_front();
        s->bytes_in_use += double(r->bytes);
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
        r->state = 1;
        r->t_admit = Clock::now();
        to_admit.push_back(r);
      }
      if (to_admit.empty() && s->active.empty()) {
        s->cv_work.wait_for(g, std::chrono::milliseconds(2));
        continue;
      }
    }
    for (Request* r : to_admit) {
      if (admit(s, r)) {
        std::lock_guard<std::mutex> g(s->mu);
        s->active.push_back(r);
        s->peak_active = std::max(s->peak_active, int(s->active.size()));
      } else {
        finish(s, r, false);
      }
    }
    bool progress = !to_admit.empty();
    finished.clear();
    std::vector<Request*> act;
    {
      std::lock_guard<std::mutex> g(s->mu);
      act = s->active;
    }
    for (Request* r : act) {
      // retire completed chunks
      while (r->ev_count > 0) {
        const int tail = (r->ev_head - r->ev_count + 2) % 2;
        if (cudaEventQuery(r->ev[tail]) != cudaSuccess) break;
        --r->ev_count;
        progress = true;
      }
      if (r->enqueued < r->nsteps && r->ev_count < 2) {
        const int n = std::min(s->chunk, r->nsteps - r->enqueued);
        try {
          if (r->exec && n == s->chunk) {
            CK(cudaGraphLaunch(r->exec, r->h->stream));
          } else {
            step_n(r->h, r->dt, n);
            // after the first (eager) chunk, capture a full chunk once if
            // more full chunks follow: one launch per chunk from then on
            if (!r->exec && r->nsteps - r->enqueued - n >= 2 * s->chunk) {
              CK(cudaStreamBeginCapture(r->h->stream, cudaStreamCaptureModeThreadLocal));
              try {
                step_n(r->h, r->dt, s->chunk);
              } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(r->h->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
              }
              CK(cudaStreamEndCapture(r->h->stream, &r->graph));
              CK(cudaGraphInstantiate(&r->exec, r->graph, 0));
            }
          }
          CK(cudaEventRecord(r->ev[r->ev_head], r->h->stream));
        } catch (std::exception& ex) {
          r->err = ex.what();
          finished.push_back(r);
          continue;
        }
        r->ev_head = (r->ev_head + 1) % 2;
        ++r->ev_count;
        r->enqueued += n;
        progress = true;
      } else if (r->enqueued >= r->nsteps && r->ev_count == 0) {
        finished.push_back(r);
      }
    }
    for (Request* r : finished) {
      {
        std::lock_guard<std::mutex> g(s->mu);
        s->active.erase(std::find(s->active.begin(), s->active.end(), r));
      }
      finish(s, r, r->err.empty());
      progress = true;
    }
    if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  // shutdown: drain what is running, drop what is queued
  std::vector<Request*> act;
  {
    std::lock_guard<std::mutex> g(s->mu);
    act = s->active;
    s->active.clear();
  }
  for (Request* r : act) finish(s, r, false);
}

}  // namespace
}  // namespace mxm

using mxm::Server;

#define SERVER_BEGIN                \
  Server* s = (Server*)server;      \
  if (!s) return MXM_DG_EINVAL;     \
  try {
#define SERVER_END                                                               \
  return MXM_DG_OK;                                                              \
  }                                                                              \
  catch (std::exception & ex) {                                                  \
    std::lock_guard<std::mutex> g(s->mu);                                        \
    s->err = ex.what();                                                          \
    return MXM_DG_EINVAL;                                                        \
  }

extern "C" {

int mxm_dg_server_create(double hbm_budget_bytes, int max_active, int steps_per_chunk, void** server) {
  if (!server || !(hbm_budget_bytes > 0) || max_active < 1 || steps_per_chunk < 1) return MXM_DG_EINVAL;
  *server = nullptr;
  std::unique_ptr<Server> s(new Server);
  if (cudaGetDevice(&s->device) != cudaSuccess) return MXM_DG_ECUDA;
  s->budget = hbm_budget_bytes;
  s->max_active = max_active;
  s->chunk = steps_per_chunk;
  Server* raw = s.get();
  raw->worker = std::thread(mxm::worker_main, raw);
  *server = s.release();
  return MXM_DG_OK;
}

int mxm_dg_server_destroy(void* server) {
  Server* s = (Server*)server;
  if (!s) return MXM_DG_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    for (mxm::Request* r : s->queue) {
      r->state = 3;
      r->err = "server destroyed before the request ran";
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
  return MXM_DG_OK;
}

int mxm_dg_server_submit(void* server, const mxm_dg_mesh_desc* mesh, const mxm_dg_physics_desc* phys, int P,
                         int precision, int ic_kind, const double* ic_params, int nparams, int limiter,
                         double venkat_eps, double dt, int nsteps, void* out_host, int64_t* request_id) {
  SERVER_BEGIN
  if (!mesh || !phys || !request_id) throw mxm::ArgError("mesh, phys and request_id must be non-null");
  if (nparams < 0 || nparams > 32 || (nparams > 0 && !ic_params)) throw mxm::ArgError("nparams must be 0..32");
  if (!(dt > 0.0) || nsteps < 0) throw mxm::ArgError("dt > 0 and nsteps >= 0");
  if (P < 1 || P > 5 || (mesh->dim != 2 && mesh->dim != 3) || precision < 0 || precision > 2 || phys->kind < 0 ||
      phys->kind > MXM_DG_PHYS_TWO_FLUID || mesh->nx < 1 || mesh->ny < 1 || (mesh->dim == 3 && mesh->nz < 1))
    throw mxm::ArgError("order 1..5, dim 2 or 3, precision 0..2, physics kind 0..6, cell counts >= 1");
  std::unique_ptr<mxm::Request> r(new mxm::Request);
  r->mesh = *mesh;
  r->phys = *phys;
  r->P = P;
  r->prec = precision;
  r->ic_kind = ic_kind;
  r->nparams = nparams;
  for (int i = 0; i < nparams; ++i) r->params[i] = ic_params[i];
  r->limiter = limiter;
  r->eps = venkat_eps;
  r->dt = dt;
  r->nsteps = nsteps;
  r->out = out_host;
  r->bytes = mxm::footprint(*r, &r->dof);
  std::lock_guard<std::mutex> g(s->mu);
  if (double(r->bytes) > s->budget) throw mxm::ArgError("request larger than the server's HBM budget");
  r->id = s->next_id++;
  r->t_submit = mxm::Clock::now();
  if (!s->any_submit) {
    s->any_submit = true;
    s->t_first_submit = r->t_submit;
  }
  *request_id = r->id;
  s->queue.push_back(r.get());
  s->all[r->id] = std::move(r);
  s->cv_work.notify_all();
  SERVER_END
}

// MXM_DG_OK when finished (latency_ms = submit -> result on the host),
// MXM_DG_ENOTREADY while queued or running, MXM_DG_EINVAL for an unknown id,
// the request's failure code text in the server error otherwise.
int mxm_dg_server_poll(void* server, int64_t id, double* latency_ms) {
  Server* s = (Server*)server;
  if (!s) return MXM_DG_EINVAL;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return MXM_DG_EINVAL;
  mxm::Request* r = it->second.get();
  if (r->state < 2) return MXM_DG_ENOTREADY;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (r->state == 3) {
    s->err = "request " + std::to_string(id) + " failed: " + r->err;
    return MXM_DG_ECUDA;
  }
  return MXM_DG_OK;
}

int mxm_dg_server_wait(void* server, int64_t id, double timeout_s, double* latency_ms) {
  Server* s = (Server*)server;
  if (!s) return MXM_DG_EINVAL;
  {
    std::unique_lock<std::mutex> g(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return MXM_DG_EINVAL;
    mxm::Request* r = it->second.get();
    const auto deadline = mxm::Clock::now() + std::chrono::duration_cast<mxm::Clock::duration>(
                                                  std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9));
    while (r->state < 2)
      if (s->cv_done.wait_until(g, deadline) == std::cv_status::timeout && r->state < 2) return MXM_DG_ETIMEDOUT;
  }
  return mxm_dg_server_poll(server, id, latency_ms);
}

// out[0] completed, [1] failed, [2] p50 ms, [3] p99 ms, [4] mean ms,
// [5] solves/s (completed / (last completion - first submit)),
// [6] DOF·stage/s over the same span, [7] peak admitted bytes,
// [8] peak concurrent solves, [9] queued now, [10] running now
int mxm_dg_server_stats(void* server, double* out, int n) {
  Server* s = (Server*)server;
  if (!s || !out || n < 1) return MXM_DG_EINVAL;
  std::lock_guard<std::mutex> g(s->mu);
  std::vector<double> lat = s->latencies_ms;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) {
    if (lat.empty()) return 0.0;
    const double pos = p * (lat.size() - 1);
    const size_t i = size_t(pos);
    const double f = pos - double(i);
    return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat[i];
  };
  int failed = 0;
  for (auto& kv : s->all) failed += kv.second->state == 3;
  double mean = 0;
  for (double v : lat) mean += v;
  mean = lat.empty() ? 0 : mean / lat.size();
  const double span = lat.empty() ? 0 : std::chrono::duration<double>(s->t_last_done - s->t_first_submit).count();
  const double v[12] = {double(lat.size()), double(failed), pct(0.5), pct(0.99), mean,
                        span > 0 ? lat.size() / span : 0.0, span > 0 ? s->dof_stages_done / span : 0.0,
                        s->peak_bytes, double(s->peak_active), double(s->queue.size()), double(s->active.size()),
                        s->bytes_in_use};
  for (int i = 0; i < n && i < 12; ++i) out[i] = v[i];
  return MXM_DG_OK;
}

int mxm_dg_server_last_error(void* server, char* buf, int len) {
  Server* s = (Server*)server;
  if (!s || !buf || len <= 0) return MXM_DG_EINVAL;
  std::lock_guard<std::mutex> g(s->mu);
  std::strncpy(buf, s->err.c_str(), size_t(len) - 1);
  buf[len - 1] = '\0';
  return MXM_DG_OK;
}

}  // extern "C"
