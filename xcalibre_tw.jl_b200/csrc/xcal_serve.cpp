// Serving loop: a stream of independent SIMPLE cases on one GPU
// (include/xcal.h, xcal_serve_*).  No reference counterpart: the reference
// runs one case per Julia process (simple!, src/Solvers/Solvers_1_SIMPLE.jl:3-67).
//
// Design: submit() deep-copies the case (mesh through xcal_hmesh_from_desc,
// the case struct with its boundary tables, the initial fields) and queues
// it.  `slots` worker threads each own one context created with
// XCAL_FLAG_CLUSTER, so every run is a single hardware thread-block cluster
// on its own stream: runs of different workers overlap on the GPU without a
// grid-wide barrier that could wait on CTAs of another kernel.  A worker sets
// the case up on its context (host renumbering and layout, uploads, case
// set-up), runs SIMPLE to the tolerance or the iteration cap in one launch,
// reads the fields back and publishes the result.  Device buffers are
// stream-ordered, so set-up and clean-up of one worker do not synchronise
// the others.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/xcal.h"

namespace xcal {
void preload_programs();   // xcal_launch.cu
}

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
  int64_t ticket = 0;
  xcal_hmesh mesh = nullptr;
  xcal_case cfg{};
  std::vector<xcal_bc> bc[5];
  std::vector<double> U0, p0;
  int64_t n = 0;
  Clock::time_point t_submit, t_start;
  // result
  bool done = false;
  xcal_serve_result res{};
  std::vector<double> U, p;
  ~Job() {
    if (mesh) xcal_hmesh_free(mesh);
  }
};

}  // namespace

struct xcal_server_s {
  int device = 0;
  xcal_serve_cfg cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<int64_t, std::shared_ptr<Job>> jobs;
  std::vector<std::thread> workers;
  bool stop = false;
  int64_t next_ticket = 1;
  xcal_serve_stats st{};
  std::string init_err;
  int init_status = XCAL_OK;
  int started = 0;
};

namespace {

int run_case(xcal_ctx ctx, const xcal_serve_cfg &cfg, Job &j) {
  xcal_mesh_desc d;
  int st = xcal_hmesh_desc(j.mesh, &d);
  if (st) return st;
  const int64_t n = d.ncells;
  st = xcal_mesh_upload(ctx, &d, cfg.renumber);
  if (st) return st;
  st = xcal_case_setup(ctx, &j.cfg);
  if (st) return st;
  st = xcal_ctx_set_tolerance(ctx, cfg.tolerance);
  if (st) return st;
  for (int c = 0; c < 3; ++c) {
    st = xcal_field_set(ctx, XCAL_FIELD_UX + c, j.U0.data() + (size_t)c * n, n);
    if (st) return st;
  }
  st = xcal_field_set(ctx, XCAL_FIELD_P, j.p0.data(), n);
  if (st) return st;
  const auto t_setup = Clock::now();
  j.res.setup_ms = ms_between(j.t_start, t_setup);
  const int its = cfg.max_iterations;
  std::vector<double> R(4 * (size_t)its, 1.0);
  int32_t done = 0;
  st = xcal_simple_run(ctx, its, R.data(), R.data() + its, R.data() + 2 * (size_t)its, R.data() + 3 * (size_t)its,
                       nullptr, &done);
  xcal_last_run_stats(ctx, &j.res.run_ms, nullptr, 0);
  j.res.iterations = done;
  if (st) return st;   // XCAL_ERR_NAN: the case diverged and was stopped
  const int last = done > 0 ? done - 1 : 0;
  bool conv = done > 0;
  for (int c = 0; c < 4; ++c) {
    j.res.residual[c] = R[(size_t)c * its + last];
    if (c == 2 && d.dim == 2) continue;
    conv = conv && j.res.residual[c] <= cfg.tolerance;
  }
  j.res.converged = conv ? 1 : 0;
  j.U.assign(3 * (size_t)n, 0.0);
  j.p.assign((size_t)n, 0.0);
  for (int c = 0; c < 3; ++c) {
    st = xcal_field_get(ctx, XCAL_FIELD_UX + c, j.U.data() + (size_t)c * n, n);
    if (st) return st;
  }
  return xcal_field_get(ctx, XCAL_FIELD_P, j.p.data(), n);
}

void worker_main(xcal_server s) {
  xcal_ctx ctx = nullptr;
  int cst = xcal_ctx_create(s->device, XCAL_FLAG_CLUSTER | XCAL_FLAG_ABORT_ON_NAN, &ctx);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (cst != XCAL_OK && s->init_status == XCAL_OK) {
      s->init_status = cst;
      s->init_err = "worker context creation failed";
    }
    s->started += 1;
  }
  s->cv_done.notify_all();
  for (;;) {
    std::shared_ptr<Job> j;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->stop) break;
      j = s->queue.front();
      s->queue.pop_front();
      s->st.queued -= 1;
      s->st.running += 1;
    }
    j->t_start = Clock::now();
    j->res.queue_ms = ms_between(j->t_submit, j->t_start);
    j->res.ncells = (int32_t)j->n;
    int st = ctx ? run_case(ctx, s->cfg, *j) : cst;
    j->res.status = st;
    j->res.total_ms = ms_between(j->t_submit, Clock::now());
    {
      std::lock_guard<std::mutex> lk(s->mu);
      j->done = true;
      s->st.running -= 1;
      if (st == XCAL_OK) {
        s->st.completed += 1;
        s->st.cell_iterations += (double)j->n * j->res.iterations;
        s->st.run_ms += j->res.run_ms;
      } else {
        s->st.failed += 1;
      }
      // the mesh copy is no longer needed once the case has run
      if (j->mesh) {
        xcal_hmesh_free(j->mesh);
        j->mesh = nullptr;
      }
      j->U0.clear(); j->U0.shrink_to_fit();
      j->p0.clear(); j->p0.shrink_to_fit();
    }
    s->cv_done.notify_all();
  }
  if (ctx) xcal_ctx_destroy(ctx);
}

}  // namespace

extern "C" {

int xcal_serve_create(int device, const xcal_serve_cfg *cfg, xcal_server *out) {
  if (!cfg || !out) return XCAL_ERR_ARG;
  *out = nullptr;
  if (cfg->slots < 1 || cfg->slots > 64 || cfg->max_iterations < 1 || !(cfg->tolerance >= 0.0) ||
      cfg->renumber < XCAL_RENUMBER_NONE || cfg->renumber > XCAL_RENUMBER_COLOR)
    return XCAL_ERR_ARG;
  // load the program's builds before any case runs (see preload_programs)
  if (cudaSetDevice(device) != cudaSuccess) {
    (void)cudaGetLastError();
    return XCAL_ERR_CUDA;
  }
  xcal::preload_programs();
  auto *s = new xcal_server_s();
  s->device = device;
  s->cfg = *cfg;
  for (int i = 0; i < cfg->slots; ++i) s->workers.emplace_back(worker_main, s);
  int st;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->started == cfg->slots; });
    st = s->init_status;
  }
  if (st != XCAL_OK) {
    xcal_serve_destroy(s);
    return st;
  }
  *out = s;
  return XCAL_OK;
}

int xcal_serve_submit(xcal_server s, const xcal_mesh_desc *mesh, const xcal_case *cfg, const double *U0,
                      const double *p0, int64_t *ticket) {
  if (!s || !mesh || !cfg || !ticket) return XCAL_ERR_ARG;
  auto j = std::make_shared<Job>();
  j->t_submit = Clock::now();
  int st = xcal_hmesh_from_desc(mesh, &j->mesh, nullptr, 0);
  if (st) return st;
  j->n = mesh->ncells;
  j->cfg = *cfg;
  const xcal_bc *src[5] = {cfg->bc_U, cfg->bc_p, cfg->bc_k, cfg->bc_omega, cfg->bc_nut};
  const int32_t cnt[5] = {cfg->nbc_U, cfg->nbc_p, cfg->nbc_k, cfg->nbc_omega, cfg->nbc_nut};
  for (int k = 0; k < 5; ++k) {
    if (cnt[k] < 0 || (cnt[k] > 0 && !src[k])) return XCAL_ERR_ARG;
    if (cnt[k] > 0) j->bc[k].assign(src[k], src[k] + cnt[k]);
  }
  j->cfg.bc_U = j->bc[0].data(); j->cfg.bc_p = j->bc[1].data(); j->cfg.bc_k = j->bc[2].data();
  j->cfg.bc_omega = j->bc[3].data(); j->cfg.bc_nut = j->bc[4].data();
  j->U0.assign(3 * (size_t)j->n, 0.0);
  j->p0.assign((size_t)j->n, 0.0);
  if (U0) std::memcpy(j->U0.data(), U0, sizeof(double) * 3 * (size_t)j->n);
  if (p0) std::memcpy(j->p0.data(), p0, sizeof(double) * (size_t)j->n);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return XCAL_ERR_STATE;
    j->ticket = s->next_ticket++;
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    s->st.submitted += 1;
    s->st.queued += 1;
    *ticket = j->ticket;
  }
  s->cv_work.notify_one();
  return XCAL_OK;
}

int xcal_serve_poll(xcal_server s, int64_t ticket, int32_t wait_ms, xcal_serve_result *res, double *U, double *p) {
  if (!s || !res) return XCAL_ERR_ARG;
  std::shared_ptr<Job> j;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return XCAL_ERR_ARG;
    j = it->second;
    auto ready = [&] { return j->done; };
    if (wait_ms < 0) {
      s->cv_done.wait(lk, ready);
    } else if (wait_ms > 0) {
      s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
    }
    if (!j->done) return XCAL_PENDING;
    s->jobs.erase(it);
  }
  *res = j->res;
  if (U && !j->U.empty()) std::memcpy(U, j->U.data(), sizeof(double) * j->U.size());
  if (p && !j->p.empty()) std::memcpy(p, j->p.data(), sizeof(double) * j->p.size());
  return XCAL_OK;
}

int xcal_serve_stats_get(xcal_server s, xcal_serve_stats *st) {
  if (!s || !st) return XCAL_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  return XCAL_OK;
}

int xcal_serve_destroy(xcal_server s) {
  if (!s) return XCAL_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->st.queued = 0;
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto &t : s->workers)
    if (t.joinable()) t.join();
  delete s;
  return XCAL_OK;
}

}  // extern "C"
