// Serving loop: a stream of independent SIMPLE cases on one GPU in one
// persistent launch (include/xcal.h, xcal_serve_*).  No reference
// counterpart: the reference runs one case per Julia process (simple!,
// src/Solvers/Solvers_1_SIMPLE.jl:3-67).
//
// Design (continuous batching, packed):
//   * one persistent serving kernel (xcal_serve_kernel, cooperative launch, all
//     CTAs co-resident) runs for the server's lifetime; its CTAs poll per-CTA
//     mail words in pinned host memory;
//   * a case is admitted when its device footprint fits the server's device
//     arena (a region allocated once at start, so nothing is allocated or
//     freed on the device while the kernel runs); set-up threads build the
//     case's image on the host (renumbering, layout, BC tables, initial
//     fields) into pinned staging memory, with device pointers into its arena
//     region;
//   * the scheduler gives each ready case a group of CTAs sized by its tiles
//     (ceil(tiles / tiles_per_cta), at most max_ctas) and a barrier word; the
//     group copies the image in, runs SIMPLE to the case's tolerance or cap,
//     writes the results to pinned host memory and frees itself; the
//     scheduler then returns the memory, the CTAs and the barrier word, so
//     cases arriving while others run start as soon as CTAs and memory allow.
// There are no streams, copies or kernel launches besides the one serving
// launch while cases run, so no case's transfers can queue behind another
// case's run.
#include <algorithm>
#include <atomic>
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
#include "xcal_case.h"
#include "xcal_kernel.h"

namespace {

using Clock = std::chrono::steady_clock;
using xcal::CaseImage;
using xcal::ImageSink;
using xcal::ServeCtl;
using xcal::ServeJob;
using xcal::ServeMail;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// First-fit range allocator over [0, cap) with coalescing of freed ranges.
struct RangeAlloc {
  size_t cap = 0, used = 0, peak = 0;
  std::map<size_t, size_t> free;   // offset -> size
  void init(size_t c) {
    cap = c;
    used = peak = 0;
    free.clear();
    if (c) free[0] = c;
  }
  bool alloc(size_t bytes, size_t &off) {
    for (auto it = free.begin(); it != free.end(); ++it) {
      if (it->second < bytes) continue;
      off = it->first;
      const size_t rest = it->second - bytes;
      free.erase(it);
      if (rest) free[off + bytes] = rest;
      used += bytes;
      peak = std::max(peak, used);
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    used -= bytes;
    auto it = free.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free.erase(nx);
    }
    if (it != free.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free.erase(it);
      }
    }
  }
};

size_t up256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t SLOT_BYTES = 128;

struct Job {
  int64_t ticket = 0;
  xcal_hmesh mesh = nullptr;
  xcal_case cfg{};
  std::vector<xcal_bc> bc[5];
  std::vector<double> U0, p0;
  int64_t n = 0;
  Clock::time_point t_submit, t_setup0, t_run0;
  // image and placement
  CaseImage img;
  size_t dev_off = 0, dev_bytes = 0, host_off = 0, host_bytes = 0;
  ServeJob *sj = nullptr;   // in pinned host memory
  int *state = nullptr;     // sj->out_state (host view)
  double *oU = nullptr, *op = nullptr, *oR = nullptr;
  int *okry = nullptr;
  int k = 0, slot = -1;
  std::vector<int> ctas;
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
  int tiles_per_cta = 4, max_ctas = 64;
  // device arena, pinned host arena (with its device view), barrier words
  char *dev_arena = nullptr;
  char *host_arena = nullptr, *host_arena_dev = nullptr;
  RangeAlloc dalloc, halloc;
  // per slot, one 128-byte line: the group's barrier word, then its exit count
  char *slotmem = nullptr;
  std::vector<int> free_slots;
  // control records in pinned host memory
  ServeMail *mail = nullptr, *mail_dev = nullptr;
  ServeCtl *ctl = nullptr, *ctl_dev = nullptr;
  std::vector<unsigned long long> seq;
  int grid = 0;
  std::vector<char> cta_busy;
  int free_ctas = 0;
  cudaStream_t kstream = nullptr;
  cudaEvent_t kdone = nullptr;
  bool kernel_live = false;
  const void *kfn = nullptr;
  // queues and threads
  std::mutex mu;
  std::condition_variable cv_setup, cv_mem, cv_done, cv_sched;
  std::deque<std::shared_ptr<Job>> pending, ready;
  std::vector<std::shared_ptr<Job>> running;
  std::map<int64_t, std::shared_ptr<Job>> jobs;
  std::vector<std::thread> setup_threads;
  std::thread sched;
  bool stop = false;
  int64_t next_ticket = 1;
  xcal_serve_stats st{};
  std::string err;
};

namespace {

int choose_k(xcal_server s, int ntiles) {
  int k = (ntiles + s->tiles_per_cta - 1) / s->tiles_per_cta;
  return std::max(1, std::min(std::min(k, s->max_ctas), s->grid));
}

// Image of one case: measure pass, admission (device and host footprint),
// build pass into the allocated regions, job record.
int setup_job(xcal_server s, Job &j) {
  xcal_mesh_desc d;
  int st = xcal_hmesh_desc(j.mesh, &d);
  if (st) return st;
  xcal_case cfg = j.cfg;
  cfg.precision = s->cfg.precision;
  const int iters = s->cfg.max_iterations;
  std::string e;
  ImageSink meas;
  CaseImage tmp;
  st = xcal::build_case_image(&d, s->cfg.renumber, &cfg, j.U0.data(), j.p0.data(), s->cfg.tolerance, iters,
                              s->max_ctas, meas, tmp, e);
  if (st) return st;
  if (tmp.ns != s->cfg.dim) return XCAL_ERR_UNSUPPORTED;
  if (cfg.model != XCAL_MODEL_LAMINAR) return XCAL_ERR_UNSUPPORTED;
  meas.finish_measure();
  const int64_t n = tmp.n;
  const int ns = tmp.ns;
  const size_t out_bytes = up256(sizeof(ServeJob)) + up256(sizeof(double) * n * ns) + up256(sizeof(double) * n) +
                           up256(sizeof(double) * 4 * iters) + up256(sizeof(int) * 5 * iters) + 256;
  j.dev_bytes = meas.total();
  j.host_bytes = meas.copy_size + out_bytes;
  if (j.dev_bytes > s->dalloc.cap || j.host_bytes > s->halloc.cap) return XCAL_ERR_OOM;
  {
    // admission by footprint: wait until the case fits both arenas
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
      if (s->stop) return XCAL_ERR_STATE;
      size_t doff = 0, hoff = 0;
      if (s->dalloc.alloc(j.dev_bytes, doff)) {
        if (s->halloc.alloc(j.host_bytes, hoff)) {
          j.dev_off = doff;
          j.host_off = hoff;
          break;
        }
        s->dalloc.release(doff, j.dev_bytes);
      }
      s->cv_mem.wait(lk);
    }
  }
  ImageSink b = meas;
  b.dev_base = s->dev_arena + j.dev_off;
  b.host_img = s->host_arena + j.host_off;
  st = xcal::build_case_image(&d, s->cfg.renumber, &cfg, j.U0.data(), j.p0.data(), s->cfg.tolerance, iters,
                              s->max_ctas, b, j.img, e);
  if (st || b.copy_off > b.copy_size || b.zero_off > b.zero_size || b.scratch_off > b.scratch_size) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->dalloc.release(j.dev_off, j.dev_bytes);
    s->halloc.release(j.host_off, j.host_bytes);
    s->cv_mem.notify_all();
    return st ? st : XCAL_ERR_STATE;
  }
  // job record and result areas after the image in the host region
  char *h = s->host_arena + j.host_off + b.copy_size;
  auto dev_of = [&](const void *p) { return s->host_arena_dev + ((const char *)p - s->host_arena); };
  j.sj = (ServeJob *)h;
  h += up256(sizeof(ServeJob));
  j.oU = (double *)h;
  h += up256(sizeof(double) * n * ns);
  j.op = (double *)h;
  h += up256(sizeof(double) * n);
  j.oR = (double *)h;
  h += up256(sizeof(double) * 4 * iters);
  j.okry = (int *)h;
  h += up256(sizeof(int) * 5 * iters);
  j.state = (int *)h;
  std::memset(j.state, 0, sizeof(int) * 4);
  ServeJob &J = *j.sj;
  std::memset(&J, 0, sizeof(J));
  J.prm = j.img.prm;
  J.src = (const uint4 *)dev_of(s->host_arena + j.host_off);
  J.dst = (uint4 *)(s->dev_arena + j.dev_off);
  J.copy16 = b.copy_size / 16;
  J.zero16 = b.zero_size / 16;
  J.iters = iters;
  J.prog = xcal::PROG_SIMPLE;
  J.out_U = (double *)dev_of(j.oU);
  J.out_p = (double *)dev_of(j.op);
  J.out_R = (double *)dev_of(j.oR);
  J.out_kry = (int *)dev_of(j.okry);
  J.out_state = (int *)dev_of(j.state);
  j.k = choose_k(s, j.img.ntiles);
  return XCAL_OK;
}

void finish_job(xcal_server s, Job &j, int status) {
  // caller holds s->mu
  j.res.status = status;
  j.res.total_ms = ms_between(j.t_submit, Clock::now());
  j.done = true;
  if (status == XCAL_OK) {
    s->st.completed += 1;
    s->st.cell_iterations += (double)j.n * j.res.iterations;
    s->st.run_ms += j.res.run_ms;
  } else {
    s->st.failed += 1;
  }
  if (j.mesh) {
    xcal_hmesh_free(j.mesh);
    j.mesh = nullptr;
  }
  j.U0.clear();
  j.U0.shrink_to_fit();
  j.p0.clear();
  j.p0.shrink_to_fit();
  j.img.perm.clear();
  j.img.perm.shrink_to_fit();
}

void setup_main(xcal_server s) {
  for (;;) {
    std::shared_ptr<Job> j;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_setup.wait(lk, [&] { return s->stop || !s->pending.empty(); });
      if (s->stop) return;
      j = s->pending.front();
      s->pending.pop_front();
    }
    j->t_setup0 = Clock::now();
    j->res.queue_ms = ms_between(j->t_submit, j->t_setup0);
    const int st = setup_job(s, *j);
    std::lock_guard<std::mutex> lk(s->mu);
    j->res.setup_ms = ms_between(j->t_setup0, Clock::now());
    if (st != XCAL_OK) {
      s->st.queued -= 1;
      finish_job(s, *j, st);
      s->cv_done.notify_all();
      continue;
    }
    s->ready.push_back(j);
    s->cv_sched.notify_all();
  }
}

// Results of a finished group: fields back to the caller's order.
void collect(xcal_server s, Job &j) {
  const int *state = j.state;
  const int dn = state[0], berr = state[1], nonfin = state[2];
  const int64_t n = j.img.n;
  const int ns = j.img.ns;
  j.res.iterations = dn;
  j.res.run_ms = ms_between(j.t_run0, Clock::now());
  j.U.assign(3 * (size_t)n, 0.0);
  j.p.assign((size_t)n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t dv = j.img.perm[i];
    for (int d = 0; d < ns; ++d) j.U[(size_t)d * n + i] = j.oU[(size_t)dv * ns + d];
    if (ns == 2) j.U[(size_t)2 * n + i] = j.U0[(size_t)2 * n + i];
    j.p[i] = j.op[dv];
  }
  const int last = dn > 0 ? dn - 1 : 0;
  bool conv = dn > 0;
  for (int c = 0; c < 4; ++c) {
    j.res.residual[c] = dn > 0 ? j.oR[(size_t)last * 4 + c] : 1.0;
    if (c == 2 && ns == 2) continue;
    conv = conv && j.res.residual[c] <= s->cfg.tolerance;
  }
  j.res.converged = conv ? 1 : 0;
  int status = XCAL_OK;
  if (berr) status = XCAL_ERR_TIMEOUT;
  else if (nonfin) status = XCAL_ERR_NAN;
  finish_job(s, j, status);
}

void release_job(xcal_server s, Job &j) {
  // caller holds s->mu
  for (int c : j.ctas) {
    s->cta_busy[c] = 0;
    s->free_ctas += 1;
  }
  j.ctas.clear();
  if (j.slot >= 0) s->free_slots.push_back(j.slot);
  j.slot = -1;
  s->dalloc.release(j.dev_off, j.dev_bytes);
  s->halloc.release(j.host_off, j.host_bytes);
  s->cv_mem.notify_all();
}

// Gives the job its CTAs and barrier word, then posts the mail (job pointer,
// group index and size first, the sequence word last with release order).
void post(xcal_server s, Job &j) {
  const int slot = s->free_slots.back();
  s->free_slots.pop_back();
  j.slot = slot;
  j.sj->prm.bar = (xcal::Bar *)(s->slotmem + SLOT_BYTES * slot);
  j.sj->exits = (unsigned *)(s->slotmem + SLOT_BYTES * slot + 64);
  j.ctas.clear();
  for (int c = 0; c < s->grid && (int)j.ctas.size() < j.k; ++c)
    if (!s->cta_busy[c]) {
      s->cta_busy[c] = 1;
      j.ctas.push_back(c);
    }
  s->free_ctas -= j.k;
  ServeJob *jd = (ServeJob *)(s->host_arena_dev + ((char *)j.sj - s->host_arena));
  for (int v = 0; v < j.k; ++v) {
    ServeMail &m = s->mail[j.ctas[v]];
    m.job = jd;
    m.vbid = v;
    m.nblk = j.k;
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  for (int v = 0; v < j.k; ++v) {
    const int c = j.ctas[v];
    __atomic_store_n(&s->mail[c].seq, ++s->seq[c], __ATOMIC_RELEASE);
  }
  j.t_run0 = Clock::now();
  s->st.queued -= 1;
  s->st.running += 1;
}

void sched_main(xcal_server s) {
  auto last_hb = Clock::now();
  for (;;) {
    std::unique_lock<std::mutex> lk(s->mu);
    const auto now = Clock::now();
    if (ms_between(last_hb, now) >= 2.0) {
      __atomic_add_fetch(&s->ctl->heartbeat, 1ull, __ATOMIC_RELEASE);
      last_hb = now;
    }
    // finished groups
    bool changed = false;
    for (size_t q = 0; q < s->running.size();) {
      Job &j = *s->running[q];
      if (__atomic_load_n(j.state + 3, __ATOMIC_ACQUIRE) == 1) {
        collect(s, j);
        release_job(s, j);
        s->st.running -= 1;
        s->running.erase(s->running.begin() + q);
        changed = true;
      } else {
        ++q;
      }
    }
    // the serving launch ended (idle limit or a fault): cases in flight cannot finish
    if (s->kernel_live && cudaEventQuery(s->kdone) != cudaErrorNotReady) {
      s->kernel_live = false;
      for (auto &jp : s->running) {
        jp->res.run_ms = ms_between(jp->t_run0, Clock::now());
        finish_job(s, *jp, XCAL_ERR_CUDA);
        release_job(s, *jp);
        s->st.running -= 1;
      }
      s->running.clear();
      changed = true;
    }
    // start ready cases in arrival order while CTAs allow; a case that does
    // not fit yet is passed over for smaller ones until it has waited 50 ms
    if (s->kernel_live) {
      for (auto it = s->ready.begin(); it != s->ready.end();) {
        Job &j = **it;
        if (j.k <= s->free_ctas && !s->free_slots.empty()) {
          post(s, j);
          s->running.push_back(*it);
          it = s->ready.erase(it);
          changed = true;
          continue;
        }
        if (ms_between(j.t_submit, now) > 50.0 + j.res.queue_ms + j.res.setup_ms) break;
        ++it;
      }
    }
    if (changed) s->cv_done.notify_all();
    if (s->stop && s->running.empty() && s->ready.empty()) return;
    s->cv_sched.wait_for(lk, std::chrono::microseconds(changed ? 0 : 100));
  }
}

int launch_server_kernel(xcal_server s) {
  void *args[2] = {(void *)&s->mail_dev, (void *)&s->ctl_dev};
  cudaError_t e = cudaLaunchCooperativeKernel(s->kfn, dim3(s->grid), dim3(xcal::TPB), args, 0, s->kstream);
  if (e != cudaSuccess) return XCAL_ERR_CUDA;
  if (cudaEventRecord(s->kdone, s->kstream) != cudaSuccess) return XCAL_ERR_CUDA;
  s->kernel_live = true;
  return XCAL_OK;
}

void release_resources(xcal_server s) {
  if (s->kstream) cudaStreamSynchronize(s->kstream);
  if (s->dev_arena) cudaFree(s->dev_arena);
  if (s->slotmem) cudaFree(s->slotmem);
  if (s->host_arena) cudaFreeHost(s->host_arena);
  if (s->mail) cudaFreeHost(s->mail);
  if (s->ctl) cudaFreeHost(s->ctl);
  if (s->kdone) cudaEventDestroy(s->kdone);
  if (s->kstream) cudaStreamDestroy(s->kstream);
}

}  // namespace

extern "C" {

int xcal_serve_create(int device, const xcal_serve_cfg *cfg, xcal_server *out) {
  if (!cfg || !out) return XCAL_ERR_ARG;
  *out = nullptr;
  if (cfg->slots < 1 || cfg->slots > 4096 || cfg->max_iterations < 1 || !(cfg->tolerance >= 0.0) ||
      cfg->renumber < XCAL_RENUMBER_NONE || cfg->renumber > XCAL_RENUMBER_COLOR ||
      (cfg->precision != XCAL_PREC_FP64 && cfg->precision != XCAL_PREC_MIXED) || (cfg->dim != 2 && cfg->dim != 3) ||
      cfg->tiles_per_cta < 0 || cfg->max_ctas < 0 || cfg->setup_threads < 0 || cfg->setup_threads > 64 ||
      !(cfg->device_bytes >= 0.0) || !(cfg->host_bytes >= 0.0))
    return XCAL_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    (void)cudaGetLastError();
    return XCAL_ERR_CUDA;
  }
  auto *s = new xcal_server_s();
  s->device = device;
  s->cfg = *cfg;
  if (cfg->tiles_per_cta > 0) s->tiles_per_cta = cfg->tiles_per_cta;
  if (cfg->max_ctas > 0) s->max_ctas = cfg->max_ctas;
  s->kfn = xcal::serve_kernel_ptr(cfg->dim, cfg->precision == XCAL_PREC_MIXED);
  s->grid = xcal::serve_grid(cfg->dim, cfg->precision == XCAL_PREC_MIXED, device);
  if (!s->kfn || s->grid < 1) {
    delete s;
    return XCAL_ERR_CUDA;
  }
  s->max_ctas = std::min(s->max_ctas, s->grid);
  size_t freeb = 0, totb = 0;
  if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) {
    delete s;
    return XCAL_ERR_CUDA;
  }
  size_t dbytes = cfg->device_bytes > 0.0 ? (size_t)cfg->device_bytes : (size_t)(0.5 * (double)freeb);
  dbytes = std::min(dbytes, (size_t)(0.9 * (double)freeb)) / 256 * 256;   // never more than asked for
  const size_t hbytes = up256(cfg->host_bytes > 0.0 ? (size_t)cfg->host_bytes : ((size_t)4 << 30));
  const int nslots = std::min(cfg->slots, s->grid);
  bool ok = cudaMalloc(&s->dev_arena, dbytes) == cudaSuccess &&
            cudaMalloc(&s->slotmem, SLOT_BYTES * nslots) == cudaSuccess &&
            cudaHostAlloc(&s->host_arena, hbytes, cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess &&
            cudaHostAlloc(&s->mail, sizeof(ServeMail) * s->grid, cudaHostAllocMapped | cudaHostAllocPortable) ==
                cudaSuccess &&
            cudaHostAlloc(&s->ctl, sizeof(ServeCtl), cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess &&
            cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&s->kdone, cudaEventDisableTiming) == cudaSuccess;
  if (ok) {
    void *p = nullptr;
    ok = cudaHostGetDevicePointer(&p, s->host_arena, 0) == cudaSuccess;
    s->host_arena_dev = (char *)p;
    ok = ok && cudaHostGetDevicePointer(&p, s->mail, 0) == cudaSuccess;
    s->mail_dev = (ServeMail *)p;
    ok = ok && cudaHostGetDevicePointer(&p, s->ctl, 0) == cudaSuccess;
    s->ctl_dev = (ServeCtl *)p;
  }
  if (ok) {
    ok = cudaMemsetAsync(s->slotmem, 0, SLOT_BYTES * nslots, s->kstream) == cudaSuccess &&
         cudaStreamSynchronize(s->kstream) == cudaSuccess;
  }
  if (!ok) {
    (void)cudaGetLastError();
    release_resources(s);
    delete s;
    return XCAL_ERR_OOM;
  }
  std::memset(s->mail, 0, sizeof(ServeMail) * s->grid);
  std::memset(s->ctl, 0, sizeof(ServeCtl));
  s->ctl->idle_limit_ns = 10ull * 1000 * 1000 * 1000;   // 10 s without a heartbeat
  s->seq.assign(s->grid, 0ull);
  s->cta_busy.assign(s->grid, 0);
  s->free_ctas = s->grid;
  for (int k = nslots - 1; k >= 0; --k) s->free_slots.push_back(k);
  s->dalloc.init(dbytes);
  s->halloc.init(hbytes);
  if (launch_server_kernel(s) != XCAL_OK) {
    (void)cudaGetLastError();
    release_resources(s);
    delete s;
    return XCAL_ERR_CUDA;
  }
  const int nsetup = cfg->setup_threads > 0 ? cfg->setup_threads
                                            : std::max(2, std::min(8, (int)std::thread::hardware_concurrency() / 2));
  for (int i = 0; i < nsetup; ++i) s->setup_threads.emplace_back(setup_main, s);
  s->sched = std::thread(sched_main, s);
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
    s->pending.push_back(j);
    s->st.submitted += 1;
    s->st.queued += 1;
    *ticket = j->ticket;
  }
  s->cv_setup.notify_one();
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
  res->ncells = (int32_t)j->n;
  if (U && !j->U.empty()) std::memcpy(U, j->U.data(), sizeof(double) * j->U.size());
  if (p && !j->p.empty()) std::memcpy(p, j->p.data(), sizeof(double) * j->p.size());
  return XCAL_OK;
}

int xcal_serve_stats_get(xcal_server s, xcal_serve_stats *st) {
  if (!s || !st) return XCAL_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  st->device_bytes = (double)s->dalloc.cap;
  st->device_bytes_peak = (double)s->dalloc.peak;
  st->grid_ctas = s->grid;
  return XCAL_OK;
}

int xcal_serve_destroy(xcal_server s) {
  if (!s) return XCAL_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    // cases not started yet are dropped; running ones finish
    for (auto &j : s->pending) finish_job(s, *j, XCAL_ERR_STATE);
    s->st.queued -= (int64_t)s->pending.size();
    s->pending.clear();
    for (auto &j : s->ready) {
      finish_job(s, *j, XCAL_ERR_STATE);
      s->dalloc.release(j->dev_off, j->dev_bytes);
      s->halloc.release(j->host_off, j->host_bytes);
    }
    s->st.queued -= (int64_t)s->ready.size();
    s->ready.clear();
  }
  s->cv_setup.notify_all();
  s->cv_mem.notify_all();
  s->cv_sched.notify_all();
  for (auto &t : s->setup_threads)
    if (t.joinable()) t.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto &j : s->ready) {
      finish_job(s, *j, XCAL_ERR_STATE);
      s->dalloc.release(j->dev_off, j->dev_bytes);
      s->halloc.release(j->host_off, j->host_bytes);
    }
    s->ready.clear();
  }
  if (s->sched.joinable()) s->sched.join();
  __atomic_store_n(&s->ctl->shutdown, 1u, __ATOMIC_RELEASE);
  s->cv_done.notify_all();
  release_resources(s);
  delete s;
  return XCAL_OK;
}

}  // extern "C"
