// Serving: a request loop over HDG solves of this library's model on one GPU.
//
// Requests (Exasim's four datain blobs plus a precision mode) are queued as they arrive.
// `slots` host threads each drive one solve at a time on its own context and CUDA stream, so
// admitted solves overlap on the device.  Admission is by device-memory budget: the request
// at the head of the queue starts when a slot is free and its context fits in the budget
// (contexts held by finished requests, kept for reuse, are evicted oldest first to make
// room).  A finished request's context stays resident, keyed by its master, mesh, sol and
// app blobs without the physical parameters; a later request with the same key reuses it
// (exa_ctx_reset) and skips the set-up: connectivity, geometry, the q matrices and the
// device allocations.  Steady problems run Newton (solution.cpp:125-243); time-dependent
// ones run every DIRK step of their app (exasim.hpp:413-482).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "exa_batch.cuh"
#include "exa_solver.cuh"
#include "../../include/exasim_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

enum { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3 };

struct Request {
  long long id = 0;
  std::vector<double> app, master, mesh, sol;
  int precision = 0;
  double inner_tol = 1e-4, rtol = 0.0;
  unsigned long long key = 0;
  long long est = 0;
  int state = RQ_QUEUED;
  int status = EXA_OK;
  std::string msg;
  std::vector<double> udg, uh;
  Clock::time_point t_submit, t_start, t_end;
  int newton = 0, gmres = 0, reused = 0;
  double r0 = 0.0, r1 = 0.0;
};

struct Cached {
  unsigned long long key = 0;
  ExaCtx* c = nullptr;
  Clock::time_point last;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct exa_server {
  int device = 0;
  long long budget = 0;
  bool reuse = true;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<long long, std::shared_ptr<Request>> reqs;
  std::vector<Cached> idle;
  long long in_use = 0, peak = 0, next_id = 1;
  long long n_done = 0, n_failed = 0, n_created = 0, n_reused = 0, n_evicted = 0;
  int running = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  ExaBatcher* batcher = nullptr;  // batched GMRES across the running solves (exa_server_set_batching)
};

namespace {

void free_ctx(ExaCtx* c) {
  exa_ctx_free(*c);
  delete c;
}

// One solve on context c (created or reset by the caller); fills the request's results.
int run_solve(ExaCtx& c, Request& r) {
  EXA_TRY(exa_ctx_set_precision(c, r.precision));
  if (r.precision == 1) {
    c.mixed_inner_tol = r.inner_tol;
    c.mixed_rtol = r.rtol;
  }
  if (c.tdep == 1 && !c.dt.empty()) {
    std::vector<int> its(c.dt.size() * (size_t)std::max(1, c.nstage));
    EXA_TRY(exa_drv_dirk(c, (int)c.dt.size(), its.data(), (int)its.size()));
    for (int v : its) r.newton += v;
  } else {
    int it = 0;
    double nr = 0.0;
    EXA_TRY(exa_drv_newton(c, &it, &nr));
    r.newton = it;
  }
  r.gmres = c.total_gmres_iters;
  r.r0 = c.last_norm0;
  r.r1 = c.last_norm;
  const size_t nu = (size_t)c.P.npe * c.P.nc * c.P.ne, nh = (size_t)c.ndofuhat();
  r.udg.resize(nu);
  r.uh.resize(nh);
  EXA_CUDA(cudaMemcpyAsync(r.udg.data(), c.udg, sizeof(double) * nu, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaMemcpyAsync(r.uh.data(), c.uh, sizeof(double) * nh, cudaMemcpyDeviceToHost, c.st));
  EXA_CUDA(cudaStreamSynchronize(c.st));
  return EXA_OK;
}

void worker(exa_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    std::shared_ptr<Request> r;
    ExaCtx* ctx = nullptr;
    while (!r) {
      if (s->stop) return;
      if (!s->queue.empty()) {
        std::shared_ptr<Request> h = s->queue.front();
        auto it = s->reuse ? std::find_if(s->idle.begin(), s->idle.end(), [&](const Cached& q) { return q.key == h->key; })
                           : s->idle.end();
        if (it != s->idle.end()) {
          ctx = it->c;  // its bytes are already counted in in_use
          s->idle.erase(it);
          h->reused = 1;
          r = h;
        } else {
          // make room by evicting the least recently used idle contexts
          std::vector<ExaCtx*> evict;
          while (s->in_use + h->est > s->budget && !s->idle.empty()) {
            auto old = std::min_element(s->idle.begin(), s->idle.end(),
                                        [](const Cached& a, const Cached& b) { return a.last < b.last; });
            s->in_use -= old->c->alloc_bytes;
            evict.push_back(old->c);
            s->idle.erase(old);
            ++s->n_evicted;
          }
          // a request larger than the whole budget runs when nothing else holds memory
          if (s->in_use + h->est <= s->budget || s->in_use == 0) {
            s->in_use += h->est;
            r = h;
          }
          if (!evict.empty()) {
            lk.unlock();
            for (ExaCtx* e : evict) free_ctx(e);
            lk.lock();
          }
        }
        if (r) s->queue.pop_front();
      }
      if (!r) s->cv.wait(lk);
    }
    s->peak = std::max(s->peak, s->in_use);
    r->state = RQ_RUNNING;
    r->t_start = Clock::now();
    ++s->running;
    const bool fresh = (ctx == nullptr);
    lk.unlock();

    int st = EXA_OK;
    if (fresh) {
      ctx = new ExaCtx();
      st = exa_ctx_init(*ctx, r->app.data(), (long long)r->app.size(), r->master.data(), (long long)r->master.size(),
                        r->mesh.data(), (long long)r->mesh.size(), r->sol.data(), (long long)r->sol.size(), s->device);
    } else {
      st = exa_ctx_reset(*ctx, r->app.data(), (long long)r->app.size(), r->sol.data(), (long long)r->sol.size());
    }
    if (st == EXA_OK) {
      ctx->batcher = s->batcher;
      st = run_solve(*ctx, *r);
      ctx->batcher = nullptr;
    }
    std::string msg = st == EXA_OK ? std::string() : std::string(exa_get_error());
    const long long held = ctx->alloc_bytes;
    const bool keep = (st == EXA_OK && s->reuse);
    if (!keep) free_ctx(ctx);

    lk.lock();
    // the reservation becomes the context's actual size while it is kept, or is returned
    if (fresh) s->in_use -= r->est;
    else if (!keep) s->in_use -= held;
    if (keep) {
      if (fresh) s->in_use += held;
      s->idle.push_back(Cached{r->key, ctx, Clock::now()});
    }
    s->peak = std::max(s->peak, s->in_use);
    if (fresh) ++s->n_created;
    else ++s->n_reused;
    r->status = st;
    r->msg = msg;
    r->state = st == EXA_OK ? RQ_DONE : RQ_FAILED;
    r->t_end = Clock::now();
    r->app.clear(); r->app.shrink_to_fit();
    r->master.clear(); r->master.shrink_to_fit();
    r->mesh.clear(); r->mesh.shrink_to_fit();
    r->sol.clear(); r->sol.shrink_to_fit();
    if (st == EXA_OK) ++s->n_done;
    else ++s->n_failed;
    --s->running;
    s->cv.notify_all();
  }
}

}  // namespace

extern "C" {

int exa_server_create(int device, long long hbm_budget_bytes, int slots, int reuse_contexts, exa_server** out) {
  if (!out || slots < 1 || slots > 256 || hbm_budget_bytes <= 0) {
    exa_set_error("server: need an output handle, 1..256 slots and a positive memory budget");
    return EXA_ERR_ARG;
  }
  *out = nullptr;
  EXA_CUDA(cudaSetDevice(device));
  exa_server* s = new exa_server();
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->reuse = reuse_contexts != 0;
  for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker, s);
  *out = s;
  return EXA_OK;
}

int exa_server_submit(exa_server* s, const double* app, long long napp, const double* master, long long nmaster,
                      const double* mesh, long long nmesh, const double* sol, long long nsol, int precision,
                      double inner_tol, double rtol, long long* id) {
  if (!s || !id || !app || !master || !mesh || !sol || napp < 1 || nmaster < 1 || nmesh < 1 || nsol < 1) {
    exa_set_error("server submit: null handle, id or blob");
    return EXA_ERR_ARG;
  }
  if ((precision != 0 && precision != 1) || !(inner_tol > 0.0 && inner_tol < 1.0) || !(rtol >= 0.0 && rtol < 1.0)) {
    exa_set_error("server submit: precision 0 or 1, inner_tol in (0, 1), rtol in [0, 1)");
    return EXA_ERR_ARG;
  }
  const long long est = exa_ctx_estimate_bytes(app, napp, master, nmaster, mesh, nmesh, precision);
  if (est <= 0) {
    exa_set_error("server submit: malformed blobs");
    return EXA_ERR_ARG;
  }
  auto r = std::make_shared<Request>();
  r->app.assign(app, app + napp);
  r->master.assign(master, master + nmaster);
  r->mesh.assign(mesh, mesh + nmesh);
  r->sol.assign(sol, sol + nsol);
  r->precision = precision;
  r->inner_tol = inner_tol;
  r->rtol = rtol;
  r->est = est;
  r->key = exa_ctx_key(app, napp, master, nmaster, mesh, nmesh, sol, nsol) ^ (unsigned long long)precision;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(s->mu);
    r->id = s->next_id++;
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    *id = r->id;
  }
  s->cv.notify_all();
  return EXA_OK;
}

int exa_server_wait(exa_server* s, long long id, double timeout_s, long long* nudg, long long* nuh) {
  if (!s) {
    exa_set_error("server wait: null handle");
    return EXA_ERR_ARG;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    exa_set_error("server wait: unknown request %lld", id);
    return EXA_ERR_ARG;
  }
  std::shared_ptr<Request> r = it->second;
  auto done = [&] { return r->state == RQ_DONE || r->state == RQ_FAILED; };
  if (timeout_s < 0) s->cv.wait(lk, done);
  else if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    exa_set_error("server wait: request %lld still %s", id, r->state == RQ_QUEUED ? "queued" : "running");
    return EXA_ERR_TIMEOUT;
  }
  if (nudg) *nudg = (long long)r->udg.size();
  if (nuh) *nuh = (long long)r->uh.size();
  if (r->state == RQ_FAILED) {
    exa_set_error("request %lld failed: %s", id, r->msg.c_str());
    return r->status;
  }
  return EXA_OK;
}

int exa_server_fetch(exa_server* s, long long id, double* udg, long long nudg, double* uh, long long nuh,
                     double* info) {
  if (!s) {
    exa_set_error("server fetch: null handle");
    return EXA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    exa_set_error("server fetch: unknown request %lld", id);
    return EXA_ERR_ARG;
  }
  Request& r = *it->second;
  if (r.state != RQ_DONE && r.state != RQ_FAILED) {
    exa_set_error("server fetch: request %lld has not finished", id);
    return EXA_ERR_ARG;
  }
  if (r.state == RQ_DONE && ((udg && nudg != (long long)r.udg.size()) || (uh && nuh != (long long)r.uh.size()))) {
    exa_set_error("server fetch: result sizes are udg %zu, uh %zu", r.udg.size(), r.uh.size());
    return EXA_ERR_ARG;
  }
  if (udg && r.state == RQ_DONE) std::copy(r.udg.begin(), r.udg.end(), udg);
  if (uh && r.state == RQ_DONE) std::copy(r.uh.begin(), r.uh.end(), uh);
  if (info) {
    info[0] = ms_between(r.t_submit, r.t_start);  // queued
    info[1] = ms_between(r.t_start, r.t_end);     // set-up or reset, solve and read-back
    info[2] = ms_between(r.t_submit, r.t_end);    // latency
    info[3] = r.newton;
    info[4] = r.gmres;
    info[5] = r.r0;
    info[6] = r.r1;
    info[7] = r.reused;
  }
  const int status = r.state == RQ_DONE ? EXA_OK : r.status;
  s->reqs.erase(it);
  return status;
}

int exa_server_stats(exa_server* s, long long* out) {
  if (!s || !out) {
    exa_set_error("server stats: null argument");
    return EXA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  out[0] = (long long)s->queue.size();
  out[1] = s->running;
  out[2] = s->n_done;
  out[3] = s->n_failed;
  out[4] = s->in_use;
  out[5] = s->peak;
  out[6] = s->n_created;
  out[7] = s->n_reused;
  out[8] = (long long)s->idle.size();
  out[9] = s->n_evicted;
  return EXA_OK;
}

void exa_server_destroy(exa_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  for (auto& t : s->workers) t.join();
  cudaSetDevice(s->device);
  exa_batcher_destroy(s->batcher);
  for (auto& q : s->idle) free_ctx(q.c);
  s->idle.clear();
  delete s;
}

int exa_server_set_batching(exa_server* s, int capacity) {
  if (!s || capacity < 0) {
    exa_set_error("server batching: null server or negative capacity");
    return EXA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  if (s->running > 0 || !s->queue.empty()) {
    exa_set_error("server batching: set it before submitting requests");
    return EXA_ERR_ARG;
  }
  if (s->batcher) {
    exa_batcher_destroy(s->batcher);
    s->batcher = nullptr;
  }
  if (capacity > 0) EXA_TRY(exa_batcher_create(s->device, capacity, &s->batcher));
  return EXA_OK;
}

int exa_server_batch_stats(exa_server* s, long long* out) {
  if (!s || !out) {
    exa_set_error("server batch stats: null argument");
    return EXA_ERR_ARG;
  }
  out[0] = out[1] = out[2] = out[3] = 0;
  if (s->batcher) exa_batcher_stats(s->batcher, out);
  return EXA_OK;
}

}  // extern "C"
