// C ABI of libxcal.so (include/xcal.h): contexts, mesh upload, case set-up,
// field transfer, runs of the persistent device program, standalone solves.
#include <cuda_runtime.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/xcal.h"
#include "host_mesh.h"
#include "xcal_case.h"
#include "xcal_kernel.h"
#include "xcal_ops.h"

using namespace xcal;

namespace {

// Device allocations of one context, released together.  They are ordered
// on the context's stream (cudaMallocAsync/cudaFreeAsync): a plain cudaFree
// would synchronise the whole device and stall the runs of other contexts
// (the serving loop keeps several in flight on one GPU).
struct DevBuf {
  std::vector<void *> ptrs;
  cudaStream_t stream = nullptr;
  ~DevBuf() { release(); }
  void release() {
    for (void *p : ptrs) cudaFreeAsync(p, stream);
    ptrs.clear();
  }
  template <class T>
  T *alloc(size_t n) {
    if (n == 0) n = 1;
    void *p = nullptr;
    if (cudaMallocAsync(&p, n * sizeof(T), stream) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T *)p;
  }
};

}  // namespace

struct xcal_ctx_s {
  int device = 0;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evrun = nullptr;   // cluster-mode contexts: blocking-sync event for the run wait
  std::string err;
  bool have_mesh = false, have_case = false;
  HostMesh user, mesh;
  std::vector<int64_t> perm;   // user cell -> device cell
  Prep prep;
  int ns = 2;
  int mode = SYNC_GRID, nblocks = 1;
  int occ = 0;                 // program build: 0 = 2 CTAs/SM, 1 = 4 CTAs/SM (xcal_kernel.h)
  DevBuf mbuf, cbuf, rbuf;     // mesh, case, run buffers
  KParams hp;
  double conv = 1e-7;          // SIMPLE stop tolerance
  int run_cap = 0;
  double last_ms = 0.0;
  double *pin = nullptr;       // pinned staging, one region of n values per field
  size_t pin_n = 0;
  cudaEvent_t pin_ev[7] = {};  // last copy out of each pinned field region
  bool pin_busy[7] = {};
  int *d_perm = nullptr;       // caller cell -> device cell (device copy, int32)
  double *d_stage = nullptr;   // device staging, one region of n values per field
  void *rpin = nullptr;        // pinned run-result staging (barrier word, count, R, Krylov counts)
  size_t rpin_n = 0;
  std::vector<BcEntry> tabU, tabP;
  std::vector<xcal_bc> bcU_host;   // the case's U conditions (post-processing)
  unsigned long long *d_phase = nullptr;            // per-phase timers of the last run (device)
  unsigned long long phase[2 * NPH] = {};           // cycles, counts of the last run
};

struct xcal_hmesh_s {
  HostMesh M;
};

// Host staging buffers.  Ordinary contexts use pinned memory (asynchronous
// copies).  Cluster-mode contexts (the serving loop) use ordinary heap
// memory: allocating or freeing pinned memory can wait for work already
// queued on the device, i.e. for other contexts' runs of several seconds,
// while pageable copies are staged by the driver without such a wait.
static cudaError_t stage_alloc(xcal_ctx c, void **p, size_t bytes) {
  if (c->flags & XCAL_FLAG_CLUSTER) {
    *p = std::malloc(std::max(bytes, (size_t)1));
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}
static void stage_free(xcal_ctx c, void *p) {
  if (!p) return;
  if (c->flags & XCAL_FLAG_CLUSTER) std::free(p);
  else cudaFreeHost(p);
}

static int fail(xcal_ctx c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}
#define CUDA_TRY(c, x)                                                            \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) return fail(c, XCAL_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Blocking copy on the context's stream (the stream-ordered allocations are
// only ordered with that stream).
static cudaError_t copy_sync(xcal_ctx c, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, c->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(c->stream);
}

// Zero a device range with a copy-engine transfer rather than a memset
// kernel: a memset kernel would have to wait for a free SM while other
// contexts' persistent programs occupy the GPU (serving), a copy does not.
// A pageable source is staged before cudaMemcpyAsync returns, so the zero
// buffer may be reused at once.
static cudaError_t zero_dev(xcal_ctx c, void *dst, size_t bytes) {
  static thread_local std::vector<char> zeros;
  if (zeros.size() < bytes) zeros.assign(bytes, 0);
  return cudaMemcpyAsync(dst, zeros.data(), bytes, cudaMemcpyHostToDevice, c->stream);
}

template <class T>
static int upload(xcal_ctx c, DevBuf &buf, T *&dst, const std::vector<T> &src) {
  dst = buf.alloc<T>(src.size());
  if (!dst) return fail(c, XCAL_ERR_OOM, "device allocation failed");
  if (!src.empty()) CUDA_TRY(c, copy_sync(c, dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return XCAL_OK;
}
template <class T>
static int upload_c(xcal_ctx c, DevBuf &buf, const T *&dst, const std::vector<T> &src) {
  T *d = nullptr;
  int st = upload(c, buf, d, src);
  dst = d;
  return st;
}
#define TRY(x)              \
  do {                      \
    int s_ = (x);           \
    if (s_ != XCAL_OK) return s_; \
  } while (0)

// Sink of an ordinary context: every array is a stream-ordered allocation of
// the given buffer set, uploaded (blocking) or zero-filled on the context's
// stream as it is created.
namespace {
struct DevSink : Sink {
  xcal_ctx c;
  DevBuf &B;
  int st = XCAL_OK;
  std::string msg;
  DevSink(xcal_ctx c_, DevBuf &B_) : c(c_), B(B_) {}
  char *get(size_t bytes) {
    char *p = B.alloc<char>(bytes);
    if (!p && st == XCAL_OK) {
      st = XCAL_ERR_OOM;
      msg = "device allocation failed";
    }
    return p;
  }
  void cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess && st == XCAL_OK) {
      st = XCAL_ERR_CUDA;
      msg = std::string(what) + ": " + cudaGetErrorString(e);
    }
  }
  void *put(const void *src, size_t bytes) override {
    char *p = get(bytes);
    if (p && src && bytes) cuda(copy_sync(c, p, src, bytes, cudaMemcpyHostToDevice), "upload");
    return p;
  }
  void *zeros(size_t bytes) override {
    char *p = get(bytes);
    if (p && bytes) cuda(zero_dev(c, p, bytes), "zero fill");
    return p;
  }
  void *scratch(size_t bytes) override { return get(bytes); }
  bool ok() const override { return st == XCAL_OK; }
  int error() const override { return st; }
  std::string message() const override { return msg; }
};
}  // namespace

// CG with a two-level DILU can apply M^{-1} inside its x/r phase by
// recomputing neighbour values (2 instead of 3 grid barriers per iteration,
// identical results).  On B200 the extra chain of dependent L2 gathers costs
// more than the barrier it saves (47,385-cell BFS: 1.73 vs 1.48 ms per SIMPLE
// iteration; 128^3 cavity: 44 vs 33 ms), so it is off unless XCAL_CG_FUSE=1.
static int choose_cg_fuse(int ntiles, int nblocks) {
  const char *f = getenv("XCAL_CG_FUSE");
  (void)ntiles; (void)nblocks;
  return f ? atoi(f) != 0 : 0;
}

// Grid-barrier wait limit and expected extra arrivals, read on every run:
// XCAL_BARRIER_TIMEOUT_US (default 2 s) bounds one wait; XCAL_BARRIER_EXTRA
// (default 0) makes every wait expect that many arrivals beyond the launch's
// CTAs, so that it can end only by its limit (the test of the timeout path).
static void barrier_knobs(KParams &h) {
  const char *t = getenv("XCAL_BARRIER_TIMEOUT_US");
  const char *x = getenv("XCAL_BARRIER_EXTRA");
  const long long us = t ? atoll(t) : 0;
  h.bar_timeout_ns = us > 0 ? (unsigned long long)us * 1000ull : 0ull;
  h.bar_extra = x ? std::max(0, std::min(atoi(x), 1 << 20)) : 0;
}

static void choose_launch_mode(xcal_ctx c, int n);

// Launch forms chosen by xcal_autotune, per mesh class: (components, tiles
// bucket = floor(log2 tiles), row width, precision).  A context whose mesh
// falls in a tuned class starts with the tuned form (the environment
// overrides of choose_launch_mode still win).  All forms compute the same
// values; only the time differs.
struct TuneKey {
  int ns, bucket, W, prec;
  bool operator<(const TuneKey &o) const {
    return std::tie(ns, bucket, W, prec) < std::tie(o.ns, o.bucket, o.W, o.prec);
  }
};
struct TuneChoice {
  int mode, occ, nblocks, cg_fuse;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneChoice> g_tune;

static TuneKey tune_key(xcal_ctx c, int prec) {
  const int ntiles = (c->prep.n + TILE - 1) / TILE;
  int b = 0;
  while ((2 << b) <= ntiles) ++b;
  return TuneKey{c->ns, b, c->prep.W, prec};
}

static void choose_launch(xcal_ctx c, int n, KParams &h) {
  choose_launch_mode(c, n);
  h.cg_fuse = choose_cg_fuse((n + TILE - 1) / TILE, c->nblocks);
}

// A tuned form for this context's class, unless the environment forces one.
static void apply_tuned(xcal_ctx c, int prec) {
  if (getenv("XCAL_SYNC") || getenv("XCAL_OCC") || getenv("XCAL_NBLOCKS") || getenv("XCAL_CG_FUSE")) return;
  if (c->flags & XCAL_FLAG_CLUSTER) return;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(c, prec));
  if (it == g_tune.end()) return;
  c->mode = it->second.mode;
  c->occ = it->second.occ;
  c->nblocks = it->second.nblocks;
  c->hp.cg_fuse = it->second.cg_fuse;
}

// Build of the persistent program for a grid launch: the 4-CTA/SM build once
// the mesh has more tiles per CTA of the 2-CTA/SM grid than a threshold (the
// phases are then memory-latency rather than barrier bound).  Measured on
// B200, ms per SIMPLE iteration (2-CTA / 4-CTA build), 296-CTA grid:
//   3D: cavity 32^3 (128 tiles) 0.86 / 0.96; 48^3 (432) 1.71 / 1.62;
//       64^3 (1024) 3.56 / 2.93; 96^3 (3456) 15.4 / 11.8; 128^3 (8192) 39.6 / 27.7
//   2D: BFS 47k (186) 1.50 / 1.73; BFS 104k (407) 1.97 / 1.96; flat plate k-omega
//       150k (586) 2.68 / 2.77; cavity 400^2 (625) 2.53 / 2.71; BFS 190k (741)
//       2.80 / 2.73; BFS 416k (1625) 4.62 / 3.95; cavity 800^2 (2500) 6.86 / 6.42
// so the threshold is 1 tile per CTA in 3D and 3 in 2D.  XCAL_OCC=2 or 4
// forces one.  Both builds compute the same values.
static int choose_occ(xcal_ctx c, int ntiles) {
  const char *o = getenv("XCAL_OCC");
  if (o) return atoi(o) == 4 ? 1 : 0;
  if (c->ns < 2) return 0;
  const int maxco2 = max_coresident_blocks(c->ns, 0, c->device);
  const int per_cta = (c->ns == 3) ? 1 : 3;
  return ntiles > per_cta * std::max(maxco2, 1) ? 1 : 0;
}

static void choose_launch_mode(xcal_ctx c, int n) {
  int ntiles = (n + TILE - 1) / TILE;
  const char *m = getenv("XCAL_SYNC");
  const char *nbv = getenv("XCAL_NBLOCKS");
  int ns = c->ns;
  c->occ = 0;
  if (!(c->flags & XCAL_FLAG_CLUSTER) && !(m && (!strcmp(m, "block") || !strcmp(m, "cluster"))))
    c->occ = choose_occ(c, ntiles);
  int maxco = max_coresident_blocks(ns, c->occ, c->device);
  if (m && !strcmp(m, "block")) { c->mode = SYNC_BLOCK; c->nblocks = 1; return; }
  if ((c->flags & XCAL_FLAG_CLUSTER) && !m) {   // one hardware cluster: safe beside other kernels
    // the 4-CTA/SM build once the cluster's CTAs hold more tiles each than
    // the grid threshold of choose_occ (large cases of a serving stream)
    const char *o = getenv("XCAL_OCC");
    const int mc0 = max_cluster_blocks(ns, 0);
    if (o) c->occ = (atoi(o) == 4 && ns >= 2) ? 1 : 0;
    else c->occ = (ns >= 2 && ntiles > ((ns == 3) ? 1 : 3) * mc0) ? 1 : 0;
    c->mode = SYNC_CLUSTER;
    c->nblocks = std::max(1, std::min(max_cluster_blocks(ns, c->occ), ntiles));
    return;
  }
  if (m && !strcmp(m, "cluster")) {
    c->mode = SYNC_CLUSTER;
    int mc = max_cluster_blocks(ns);
    c->nblocks = nbv ? std::max(1, std::min(mc, atoi(nbv))) : mc;
    return;
  }
  if (m && !strcmp(m, "grid")) {
    c->mode = SYNC_GRID;
    c->nblocks = nbv ? std::max(1, std::min(maxco, atoi(nbv))) : std::max(1, maxco);
    return;
  }
  // One CTA per 256-row tile: a hardware cluster barrier while the tiles fit
  // one cluster, a grid barrier over co-resident CTAs beyond that.
  int mc = max_cluster_blocks(ns);
  if (ntiles <= mc) {
    c->mode = SYNC_CLUSTER;
    c->nblocks = std::max(1, ntiles);
    c->occ = 0;
  } else {
    c->mode = SYNC_GRID;
    c->nblocks = std::max(1, std::min(maxco, ntiles));
  }
  (void)ntiles;
}

extern "C" {

int xcal_version(int *major, int *minor) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  return XCAL_OK;
}

int xcal_ctx_create(int device, uint32_t flags, xcal_ctx *out) {
  if (!out) return XCAL_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return XCAL_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return XCAL_ERR_CUDA;
  auto *c = new xcal_ctx_s();
  c->device = device;
  c->flags = flags;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return XCAL_ERR_CUDA;
  }
  c->mbuf.stream = c->cbuf.stream = c->rbuf.stream = c->stream;
  // Contexts of the serving loop wait for their (long) runs asleep: a host
  // thread spinning in a stream synchronisation for the seconds a case runs
  // would take a core from the threads setting other cases up.  Short waits
  // (uploads, read-backs) keep spinning, where a wake-up would cost more.
  if ((flags & XCAL_FLAG_CLUSTER) &&
      cudaEventCreateWithFlags(&c->evrun, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess) {
    delete c;
    return XCAL_ERR_CUDA;
  }
  for (auto &e : c->pin_ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      delete c;
      return XCAL_ERR_CUDA;
    }
  // Keep freed stream-ordered memory in the device's pool: with the default
  // release threshold (0) every synchronisation would hand it back and the
  // next set-up would map fresh memory again.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = c;
  return XCAL_OK;
}

int xcal_ctx_destroy(xcal_ctx c) {
  if (!c) return XCAL_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->rbuf.release();
  c->cbuf.release();
  c->d_phase = nullptr;
  c->mbuf.release();
  stage_free(c, c->pin);
  stage_free(c, c->rpin);
  for (auto &e : c->pin_ev)
    if (e) cudaEventDestroy(e);
  if (c->evrun) cudaEventDestroy(c->evrun);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return XCAL_OK;
}

int xcal_ctx_set_tolerance(xcal_ctx c, double tol) {
  if (!c) return XCAL_ERR_ARG;
  if (!(tol >= 0.0)) return fail(c, XCAL_ERR_ARG, "tolerance must be >= 0");
  c->conv = tol;
  return XCAL_OK;
}

int xcal_last_error(xcal_ctx c, char *buf, size_t n) {
  if (!c || !buf || !n) return XCAL_ERR_ARG;
  snprintf(buf, n, "%s", c->err.c_str());
  return XCAL_OK;
}

// ----------------------------------------------------------- host meshes
int xcal_hmesh_build_unv(const char *path, double scale, xcal_hmesh *out, char *err, size_t nerr) {
  if (!path || !out) return XCAL_ERR_ARG;
  auto *h = new xcal_hmesh_s();
  std::string e;
  int st = build_unv(path, scale, h->M, e);
  if (st) {
    if (err && nerr) snprintf(err, nerr, "%s", e.c_str());
    delete h;
    return st;
  }
  *out = h;
  return XCAL_OK;
}

int xcal_hmesh_counts(xcal_hmesh h, int64_t *c) {
  if (!h || !c) return XCAL_ERR_ARG;
  const HostMesh &M = h->M;
  c[0] = M.nc; c[1] = M.nf; c[2] = M.nbf; c[3] = (int64_t)M.cf_face.size(); c[4] = (int64_t)M.pname.size();
  c[5] = (int64_t)M.pfaces.size(); c[6] = M.nnodes; c[7] = (int64_t)M.names.size();
  return XCAL_OK;
}

static void fill_desc(const HostMesh &M, xcal_mesh_desc *d);

int xcal_hmesh_desc(xcal_hmesh h, xcal_mesh_desc *d) {
  if (!h || !d) return XCAL_ERR_ARG;
  fill_desc(h->M, d);
  return XCAL_OK;
}

static void fill_desc(const HostMesh &M, xcal_mesh_desc *d) {
  d->ncells = M.nc; d->nfaces = M.nf; d->nbfaces = M.nbf; d->dim = M.dim;
  d->cell_centre = M.cc.data(); d->cell_volume = M.cvol.data();
  d->cell_faces_ptr = M.x_cfp.data(); d->cell_faces = M.x_cf.data(); d->cell_neighbours = M.x_cn.data();
  d->cell_nsign = M.cf_sign.data(); d->face_owner = M.x_own.data(); d->face_centre = M.fc.data();
  d->face_normal = M.fn.data(); d->face_e = M.fe.data(); d->face_area = M.farea.data();
  d->face_delta = M.fdelta.data(); d->face_weight = M.fweight.data();
  d->npatches = (int64_t)M.pname.size(); d->patch_ptr = M.pptr.data(); d->patch_faces = M.x_pf.data();
  d->patch_cells = M.x_pc.data();
  d->nnodes = M.cn_ptr.empty() ? 0 : M.nnodes;
  d->node_coords = M.nodes.empty() ? nullptr : M.nodes.data();
  d->cell_nodes_ptr = M.x_cnp.empty() ? nullptr : M.x_cnp.data();
  d->cell_nodes = M.x_cnode.empty() ? nullptr : M.x_cnode.data();
}

int xcal_hmesh_patch_names(xcal_hmesh h, char *buf, size_t n) {
  if (!h || !buf || !n) return XCAL_ERR_ARG;
  snprintf(buf, n, "%s", h->M.names.c_str());
  return XCAL_OK;
}

int xcal_hmesh_free(xcal_hmesh h) {
  delete h;
  return XCAL_OK;
}

int xcal_hmesh_from_desc(const xcal_mesh_desc *d, xcal_hmesh *out, char *err, size_t nerr) {
  if (!d || !out) return XCAL_ERR_ARG;
  auto *h = new xcal_hmesh_s();
  std::string e;
  int st = mesh_from_desc(d, h->M, e);
  if (st) {
    if (err && nerr) snprintf(err, nerr, "%s", e.c_str());
    delete h;
    return st;
  }
  *out = h;
  return XCAL_OK;
}

int xcal_hmesh_renumber(xcal_hmesh m, int32_t mode, xcal_hmesh *out, int64_t *perm) {
  if (!m || !out) return XCAL_ERR_ARG;
  if (mode < XCAL_RENUMBER_NONE || mode > XCAL_RENUMBER_COLOR) return XCAL_ERR_ARG;
  std::vector<int64_t> p;
  renumber_perm(m->M, mode, p);
  auto *h = new xcal_hmesh_s();
  apply_perm(m->M, p, mode != XCAL_RENUMBER_NONE, h->M);
  h->M.pname = m->M.pname;
  h->M.prepare_export();
  if (perm) for (size_t i = 0; i < p.size(); ++i) perm[i] = p[i] + 1;
  *out = h;
  return XCAL_OK;
}

int xcal_hmesh_csr(xcal_hmesh m, int64_t *nnz, int32_t *rp, int32_t *col, int32_t *fl, int32_t *bl, int32_t *nl) {
  if (!m) return XCAL_ERR_ARG;
  Prep P;
  std::string e;
  int st = prepare(m->M, P, e);
  if (st) return st;
  if (nnz) *nnz = P.nnz;
  if (rp) std::copy(P.row_ptr.begin(), P.row_ptr.end(), rp);
  if (col) std::copy(P.col.begin(), P.col.end(), col);
  if (fl) std::copy(P.flev.begin(), P.flev.begin() + P.n, fl);
  if (bl) std::copy(P.blev.begin(), P.blev.begin() + P.n, bl);
  if (nl) { nl[0] = P.nfl; nl[1] = P.nbl; }
  return XCAL_OK;
}

// ------------------------------------------------------------ device mesh
}  // extern "C"

// Host side of a mesh upload: validation, renumbering, device layout and the
// launch form; fills the context's mesh, permutation and layout (no device work).
static int mesh_prepare(xcal_ctx c, const xcal_mesh_desc *d, int32_t renumber) {
  std::string e;
  int st = mesh_from_desc(d, c->user, e);
  if (st) return fail(c, st, e);
  renumber_perm(c->user, renumber, c->perm);
  apply_perm(c->user, c->perm, renumber != XCAL_RENUMBER_NONE, c->mesh);
  st = prepare(c->mesh, c->prep, e);
  if (st) return fail(c, st, e);
  c->ns = (c->mesh.dim == 3) ? 3 : 2;
  KParams &h = c->hp;
  memset(&h, 0, sizeof(h));
  const Prep &P = c->prep;
  h.n = P.n; h.nf = P.nf; h.nbf = P.nbf; h.dim = c->mesh.dim; h.ntiles = P.np / TILE;
  h.nfl = P.nfl; h.nbl = P.nbl; h.np = P.np; h.Wf = P.Wf;
  return XCAL_OK;
}

// Device arrays of the mesh: geometry (SoA), face lists, boundary lists,
// level sets and the shared ELL pattern of the matrices.
static int mesh_arrays(xcal_ctx c, Sink &S) {
  const HostMesh &M = c->mesh;
  const Prep &P = c->prep;
  KParams &h = c->hp;
  std::vector<double> cx(P.n), cy(P.n), cz(P.n), fx(P.nf), fy(P.nf), fz(P.nf), nx(P.nf), ny(P.nf), nz(P.nf);
  for (int i = 0; i < P.n; ++i) { cx[i] = M.cc[3 * i]; cy[i] = M.cc[3 * i + 1]; cz[i] = M.cc[3 * i + 2]; }
  for (int f = 0; f < P.nf; ++f) {
    fx[f] = M.fc[3 * f]; fy[f] = M.fc[3 * f + 1]; fz[f] = M.fc[3 * f + 2];
    nx[f] = M.fn[3 * f]; ny[f] = M.fn[3 * f + 1]; nz[f] = M.fn[3 * f + 2];
  }
  h.vol = S.put_v(M.cvol); h.ccx = S.put_v(cx); h.ccy = S.put_v(cy); h.ccz = S.put_v(cz);
  h.area = S.put_v(M.farea); h.delta = S.put_v(M.fdelta); h.wgt = S.put_v(M.fweight);
  h.fnx = S.put_v(nx); h.fny = S.put_v(ny); h.fnz = S.put_v(nz);
  h.fcx = S.put_v(fx); h.fcy = S.put_v(fy); h.fcz = S.put_v(fz);
  h.o1 = S.put_v(P.o1); h.o2 = S.put_v(P.o2);
  h.f_face = S.put_v(P.f_face); h.f_nbr = S.put_v(P.f_nbr); h.f_pos = S.put_v(P.f_pos);
  h.f_sign = S.put_v(P.f_sign); h.f_first = S.put_v(P.f_first);
  h.cb_ptr = S.put_v(P.cb_ptr); h.cb_face = S.put_v(P.cb_face);
  h.flev = S.put_v(P.flev); h.blev = S.put_v(P.blev);
  const int *ecol = S.put_v(P.e_col), *etpos = S.put_v(P.e_tpos), *edpos = S.put_v(P.dpos);
  for (Mat *A : {&h.AU, &h.AP}) { A->col = ecol; A->tpos = etpos; A->dpos = edpos; A->W = P.W; A->np = P.np; }
  if (!S.ok()) return fail(c, S.error(), S.message());
  return XCAL_OK;
}

extern "C" {

int xcal_mesh_upload(xcal_ctx c, const xcal_mesh_desc *d, int32_t renumber) {
  if (!c) return XCAL_ERR_ARG;
  if (renumber < XCAL_RENUMBER_NONE || renumber > XCAL_RENUMBER_COLOR) return fail(c, XCAL_ERR_ARG, "bad renumber mode");
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->have_mesh = c->have_case = false;
  c->cbuf.release();
  c->d_phase = nullptr;
  c->rbuf.release();
  c->mbuf.release();
  c->run_cap = 0;
  TRY(mesh_prepare(c, d, renumber));
  DevSink S(c, c->mbuf);
  TRY(mesh_arrays(c, S));
  choose_launch(c, c->prep.n, c->hp);
  {
    std::vector<int> p32(c->perm.begin(), c->perm.end());
    c->d_perm = S.put_v(p32);
    if (!S.ok()) return fail(c, S.error(), S.message());
  }
  c->have_mesh = true;
  return XCAL_OK;
}

int xcal_mesh_permutation(xcal_ctx c, int64_t *perm, int64_t n) {
  if (!c || !perm) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "no mesh");
  if (n != c->user.nc) return fail(c, XCAL_ERR_ARG, "size mismatch");
  for (int64_t i = 0; i < n; ++i) perm[i] = c->perm[i] + 1;
  return XCAL_OK;
}

int xcal_mesh_export(xcal_ctx c, int64_t *cfp, int64_t *cf, int64_t *cn, int64_t *cs, int64_t *own,
                     double *cc, double *cv, double *fc, double *fn, double *fe, double *fa, double *fd,
                     double *fw, int64_t *pf, int64_t *pc) {
  if (!c) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "no mesh");
  const HostMesh &M = c->mesh;
  auto cp = [](auto *dst, const auto &v) { if (dst) std::copy(v.begin(), v.end(), dst); };
  cp(cfp, M.x_cfp); cp(cf, M.x_cf); cp(cn, M.x_cn); cp(cs, M.cf_sign); cp(own, M.x_own);
  cp(cc, M.cc); cp(cv, M.cvol); cp(fc, M.fc); cp(fn, M.fn); cp(fe, M.fe); cp(fa, M.farea);
  cp(fd, M.fdelta); cp(fw, M.fweight); cp(pf, M.x_pf); cp(pc, M.x_pc);
  return XCAL_OK;
}

int xcal_mesh_csr(xcal_ctx c, int64_t *nnz, int32_t *rp, int32_t *col, int32_t *fl, int32_t *bl, int32_t *nl) {
  if (!c) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "no mesh");
  const Prep &P = c->prep;
  if (nnz) *nnz = P.nnz;
  if (rp) std::copy(P.row_ptr.begin(), P.row_ptr.end(), rp);
  if (col) std::copy(P.col.begin(), P.col.end(), col);
  if (fl) std::copy(P.flev.begin(), P.flev.begin() + P.n, fl);
  if (bl) std::copy(P.blev.begin(), P.blev.begin() + P.n, bl);
  if (nl) { nl[0] = P.nfl; nl[1] = P.nbl; }
  return XCAL_OK;
}

// -------------------------------------------------------------- case setup
static int build_bc(xcal_ctx c, Sink &S, const xcal_bc *bcs, int nbc, FieldBC &out,
                    std::vector<BcEntry> &tab, bool vector, const char *what) {
  const HostMesh &M = c->mesh;
  int n = (int)M.nc, nbf = (int)M.nbf;
  if (nbc < 0 || (nbc > 0 && !bcs)) return fail(c, XCAL_ERR_ARG, std::string("bad BC list for ") + what);
  tab.assign(std::max(nbc, 1), BcEntry());
  std::vector<int> cnt(n + 1, 0), fbc(std::max(nbf, 1), -1);
  for (int b = 0; b < nbc; ++b) {
    const xcal_bc &x = bcs[b];
    if (x.patch < 0 || x.patch >= (int)M.pname.size()) return fail(c, XCAL_ERR_ARG, std::string("BC patch out of range for ") + what);
    if (x.type < XCAL_BC_DIRICHLET || x.type > XCAL_BC_NUTWALL) return fail(c, XCAL_ERR_ARG, std::string("bad BC type for ") + what);
    BcEntry &e = tab[b];
    e.type = x.type; e.pad = 0;
    for (int d = 0; d < 3; ++d) e.v[d] = vector ? x.value[d] : x.value[0];
    e.kappa = x.kappa; e.beta1 = x.beta1; e.cmu = x.cmu; e.B = x.B; e.E = x.E;
    // y_plus_laminar(E, kappa) and cmu^0.25 (RANSModels_kOmega.jl:322-331), host libm
    double yl = 11.0;
    for (int it = 0; it < 10; ++it) yl = std::log(std::max(yl * x.E, 1.0)) / x.kappa;
    e.ylam = yl;
    e.c25 = std::pow(x.cmu, 0.25);
    for (int64_t k = M.pptr[x.patch]; k < M.pptr[x.patch + 1]; ++k) {
      cnt[M.pcells[k] + 1]++;
      fbc[M.pfaces[k]] = b;
    }
  }
  std::vector<int> ptr(n + 1, 0);
  for (int i = 0; i < n; ++i) ptr[i + 1] = ptr[i] + cnt[i + 1];
  std::vector<int> face(std::max(ptr[n], 1)), bcid(std::max(ptr[n], 1));
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int b = 0; b < nbc; ++b) {
    const xcal_bc &x = bcs[b];
    for (int64_t k = M.pptr[x.patch]; k < M.pptr[x.patch + 1]; ++k) {
      int cell = (int)M.pcells[k];
      face[fill[cell]] = (int)M.pfaces[k];
      bcid[fill[cell]] = b;
      fill[cell]++;
    }
  }
  out.tab = S.put_v(tab); out.a_ptr = S.put_v(ptr);
  out.a_face = S.put_v(face); out.a_bc = S.put_v(bcid);
  out.fbc = S.put_v(fbc);
  if (!S.ok()) return fail(c, S.error(), S.message());
  return XCAL_OK;
}

constexpr int GMRES_MAX = 1000;   // GMRES basis limit (no restart: itmax vectors)

static int check_solver(xcal_ctx c, const xcal_solver_cfg &s, const char *what) {
  if (s.solver != XCAL_SOLVER_CG && s.solver != XCAL_SOLVER_BICGSTAB && s.solver != XCAL_SOLVER_GMRES)
    return fail(c, XCAL_ERR_UNSUPPORTED, std::string("solver not available for ") + what);
  if (s.preconditioner < XCAL_PRECON_DILU || s.preconditioner > XCAL_PRECON_ILU0)
    return fail(c, XCAL_ERR_UNSUPPORTED, std::string("preconditioner not available for ") + what);
  if (s.itmax < 0) return fail(c, XCAL_ERR_ARG, std::string("itmax < 0 for ") + what);
  if (s.solver == XCAL_SOLVER_GMRES && s.itmax > GMRES_MAX)
    return fail(c, XCAL_ERR_UNSUPPORTED, std::string("GMRES itmax above 1000 for ") + what);
  return XCAL_OK;
}

// GMRES work space of one Krylov work set (basis of gmax+1 vectors of m values,
// per-CTA Givens scratch, packed R) and ILU(0) factor storage.
}  // extern "C"
template <class T, class AllocT>
static void gmres_alloc(KWorkT<T> &w, int gmax, size_t m, int ns, int nblocks, AllocT allocT,
                        double *&gws, double *&gR, const std::function<double *(size_t)> &allocD) {
  w.gmax = gmax;
  if (gmax <= 0) return;
  w.V = allocT((size_t)(gmax + 1) * m);
  if (!gws) gws = allocD((size_t)std::max(nblocks, 1) * ns * 4 * (gmax + 1));
  if (!gR) gR = allocD((size_t)ns * gmax * (gmax + 1) / 2);
  w.gws = gws;
  w.gR = gR;
}
extern "C" {

static int check_case(xcal_ctx c, const xcal_case *cfg) {
  if (cfg->model != XCAL_MODEL_LAMINAR && cfg->model != XCAL_MODEL_KOMEGA) return fail(c, XCAL_ERR_ARG, "unknown model");
  const bool turb = (cfg->model == XCAL_MODEL_KOMEGA);
  if (turb) {
    TRY(check_solver(c, cfg->solver_k, "k"));
    TRY(check_solver(c, cfg->solver_omega, "omega"));
    if (!(cfg->solver_k.relax > 0.0) || !(cfg->solver_omega.relax > 0.0)) return fail(c, XCAL_ERR_ARG, "relaxation factors must be > 0");
    if (c->ns == 3) return fail(c, XCAL_ERR_UNSUPPORTED, "k-omega is a 2D model in the reference");
  }
  if (cfg->precision != XCAL_PREC_FP64 && cfg->precision != XCAL_PREC_MIXED) return fail(c, XCAL_ERR_ARG, "unknown precision");
  TRY(check_solver(c, cfg->solver_U, "U"));
  TRY(check_solver(c, cfg->solver_p, "p"));
  if (cfg->schemes_U.time == XCAL_TIME_EULER && !(cfg->dt > 0.0)) return fail(c, XCAL_ERR_ARG, "Euler time scheme needs dt > 0");
  if (!(cfg->solver_U.relax > 0.0) || !(cfg->solver_p.relax > 0.0)) return fail(c, XCAL_ERR_ARG, "relaxation factors must be > 0");
  return XCAL_OK;
}

// Device arrays of a case (set_solver/set_schemes/@assign! state, equation
// storage, Krylov work sets, fields).  U0 (3 x n, caller order) and p0 give
// initial fields; null: zero fields (ScalarField/VectorField constructors),
// set later through xcal_field_set.
static int case_arrays(xcal_ctx c, const xcal_case *cfg, Sink &B, const double *U0, const double *p0) {
  const bool turb = (cfg->model == XCAL_MODEL_KOMEGA);
  KParams &h = c->hp;
  int n = c->prep.n, nf = c->prep.nf, NS = c->ns;
  size_t nnz = (size_t)c->prep.W * c->prep.np;
  TRY(build_bc(c, B, cfg->bc_U, cfg->nbc_U, h.bcU, c->tabU, true, "U"));
  c->bcU_host.assign(cfg->bc_U, cfg->bc_U + cfg->nbc_U);
  TRY(build_bc(c, B, cfg->bc_p, cfg->nbc_p, h.bcP, c->tabP, false, "p"));
  h.model = cfg->model;
  if (turb) {
    std::vector<BcEntry> tk, tw, tn;
    TRY(build_bc(c, B, cfg->bc_k, cfg->nbc_k, h.bcK, tk, false, "k"));
    TRY(build_bc(c, B, cfg->bc_omega, cfg->nbc_omega, h.bcW, tw, false, "omega"));
    TRY(build_bc(c, B, cfg->bc_nut, cfg->nbc_nut, h.bcN, tn, false, "nut"));
    h.kK.solver = cfg->solver_k.solver; h.kK.itmax = cfg->solver_k.itmax; h.kK.atol = cfg->solver_k.atol; h.kK.rtol = cfg->solver_k.rtol;
    h.kW.solver = cfg->solver_omega.solver; h.kW.itmax = cfg->solver_omega.itmax; h.kW.atol = cfg->solver_omega.atol; h.kW.rtol = cfg->solver_omega.rtol;
    h.precK = cfg->solver_k.preconditioner; h.precW = cfg->solver_omega.preconditioner;
    h.divK = cfg->schemes_k.divergence; h.divW = cfg->schemes_omega.divergence;
    h.timeK = cfg->schemes_k.time; h.timeW = cfg->schemes_omega.time;
    h.aK = cfg->solver_k.relax; h.aW = cfg->solver_omega.relax;
  }
  h.div = cfg->schemes_U.divergence; h.time = cfg->schemes_U.time; h.grad = cfg->schemes_p.gradient;
  h.dt = cfg->dt; h.nu = cfg->nu; h.aU = cfg->solver_U.relax; h.aP = cfg->solver_p.relax;
  h.has_pref = cfg->has_pref ? 1 : 0; h.pref = cfg->pref;
  h.ref_cell = (int)c->perm[0];   // setReference!(p_eqn, pref, 1): the caller's first cell
  h.kU.solver = cfg->solver_U.solver; h.kU.itmax = cfg->solver_U.itmax; h.kU.atol = cfg->solver_U.atol; h.kU.rtol = cfg->solver_U.rtol;
  h.kP.solver = cfg->solver_p.solver; h.kP.itmax = cfg->solver_p.itmax; h.kP.atol = cfg->solver_p.atol; h.kP.rtol = cfg->solver_p.rtol;
  h.AU.precon = cfg->solver_U.preconditioner; h.AP.precon = cfg->solver_p.preconditioner;
  auto A = [&](size_t cnt) { return B.scratch_n<double>(cnt); };
  auto Z = [&](size_t cnt) { return B.zeros_n<double>(cnt); };
  // initial fields in device numbering (interleaved U), or zeros
  if (U0 && p0) {
    std::vector<double> u((size_t)n * NS), pp(n), uz(n);
    for (int i = 0; i < n; ++i) {
      const int64_t dv = c->perm[i];
      for (int d = 0; d < NS; ++d) u[(size_t)dv * NS + d] = U0[(size_t)d * n + i];
      uz[dv] = U0[(size_t)2 * n + i];
      pp[dv] = p0[i];
    }
    h.U = B.put_v(u); h.Uz2 = B.put_v(uz); h.p = B.put_v(pp);
  } else {
    h.U = Z((size_t)n * NS); h.Uz2 = Z(n); h.p = Z(n);
  }
  h.gp = Z((size_t)n * NS);
  h.AU.val = Z(nnz); h.AU.Dpiv = A(n); h.AU.Dinv = A(n);
  h.AP.val = Z(nnz); h.AP.Dpiv = A(n); h.AP.Dinv = A(n);
  h.bU = Z((size_t)n * NS); h.bP = Z(n);
  h.H = A((size_t)n * NS); h.rD = A(n); h.divH = A(n);
  h.mdot = A(nf); h.nueff = A(nf); h.rDf = A(nf); h.pf = A(nf); h.UfH = A((size_t)nf * NS);
  for (int k = 0; k < 2; ++k) {
    KWork *w = (k == 0) ? &h.wU : &h.wP;
    size_t m = (k == 0) ? (size_t)n * NS : (size_t)n;
    w->x = A(m); w->s = A(m); w->t = A(m); w->q = A(m);
    for (int b = 0; b < 2; ++b) { w->r[b] = A(m); w->p[b] = A(m); w->v[b] = A(m); }
  }
  h.part = A((size_t)2 * MAXK * h.ntiles);   // two buffers, used in turn
  // ILU(0) factors and GMRES work space where a solver asks for them (k and
  // omega reuse the pressure matrix and work set)
  auto is_ilu = [](const xcal_solver_cfg &sc) { return sc.preconditioner == XCAL_PRECON_ILU0; };
  auto gm = [](const xcal_solver_cfg &sc) { return sc.solver == XCAL_SOLVER_GMRES ? sc.itmax : 0; };
  const bool iluU = is_ilu(cfg->solver_U);
  const bool iluP = is_ilu(cfg->solver_p) || (turb && (is_ilu(cfg->solver_k) || is_ilu(cfg->solver_omega)));
  const int gmU = gm(cfg->solver_U);
  const int gmP = std::max(gm(cfg->solver_p), turb ? std::max(gm(cfg->solver_k), gm(cfg->solver_omega)) : 0);
  h.AU.fval = iluU ? A(nnz) : nullptr;
  h.AP.fval = iluP ? A(nnz) : nullptr;
  double *gwsU = nullptr, *gRU = nullptr, *gwsP = nullptr, *gRP = nullptr;
  std::function<double *(size_t)> allocD = [&](size_t cnt) { return A(cnt); };
  gmres_alloc(h.wU, gmU, (size_t)n * NS, NS, c->nblocks, A, gwsU, gRU, allocD);
  gmres_alloc(h.wP, gmP, (size_t)n, 1, c->nblocks, A, gwsP, gRP, allocD);
  h.prec = cfg->precision;
  if (h.prec == XCAL_PREC_MIXED) {
    auto F = [&](size_t cnt) { return B.scratch_n<float>(cnt); };
    for (int k = 0; k < 2; ++k) {
      MatT<float> &M32 = (k == 0) ? h.AU32 : h.AP32;
      const Mat &M64 = (k == 0) ? h.AU : h.AP;
      M32.col = M64.col; M32.tpos = M64.tpos; M32.dpos = M64.dpos; M32.W = M64.W; M32.np = M64.np;
      M32.precon = M64.precon;
      M32.val = B.zeros_n<float>(nnz); M32.Dpiv = F(n); M32.Dinv = F(n);   // padding zero, as in FP64
      M32.fval = M64.fval ? F(nnz) : nullptr;
      KWorkT<float> *w = (k == 0) ? &h.wU32 : &h.wP32;
      size_t m = (k == 0) ? (size_t)n * NS : (size_t)n;
      w->x = F(m); w->s = F(m); w->t = F(m); w->q = F(m);
      for (int b = 0; b < 2; ++b) { w->r[b] = F(m); w->p[b] = F(m); w->v[b] = F(m); }
      const KWork &w64 = (k == 0) ? h.wU : h.wP;
      double *g1 = w64.gws, *g2 = w64.gR;
      gmres_alloc(*w, w64.gmax, m, (k == 0) ? NS : 1, c->nblocks, F, g1, g2, allocD);
    }
  }
  if (turb) {
    h.k = Z(n); h.w = Z(n); h.nut = Z(n); h.nutf = Z(nf);
    h.nueffk = A(nf); h.nueffw = A(nf);
    h.Dk = A(n); h.Dw = A(n); h.Pk = A(n); h.Pw = A(n); h.G = A((size_t)n * 9);
  }
  h.done = B.zeros_n<int>(1);
  if (!B.ok()) return fail(c, B.error(), B.message());
  return XCAL_OK;
}

int xcal_case_setup(xcal_ctx c, const xcal_case *cfg) {
  if (!c || !cfg) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "xcal_case_setup before xcal_mesh_upload");
  CUDA_TRY(c, cudaSetDevice(c->device));
  TRY(check_case(c, cfg));
  c->have_case = false;
  c->cbuf.release();
  c->d_phase = nullptr;
  c->rbuf.release();
  c->run_cap = 0;
  KParams &h = c->hp;
  int n = c->prep.n;
  apply_tuned(c, cfg->precision);
  DevSink B(c, c->cbuf);
  TRY(case_arrays(c, cfg, B, nullptr, nullptr));
  h.bar = B.scratch_n<Bar>(1);
  if (!B.ok()) return fail(c, B.error(), B.message());
  if (!c->pin || c->pin_n < (size_t)n * 7) {
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    stage_free(c, c->pin);
    c->pin = nullptr;
    CUDA_TRY(c, stage_alloc(c, (void **)&c->pin, sizeof(double) * n * 7));
    c->pin_n = (size_t)n * 7;
  }
  for (bool &b : c->pin_busy) b = false;
  c->d_stage = c->cbuf.alloc<double>((size_t)n * 7);
  if (!c->d_stage) return fail(c, XCAL_ERR_OOM, "device allocation failed");
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->have_case = true;
  return XCAL_OK;
}

// ------------------------------------------------------------------ fields
static int field_target(xcal_ctx c, int32_t field, double *&base, int &stride, int &off) {
  KParams &h = c->hp;
  int NS = c->ns;
  switch (field) {
    case XCAL_FIELD_UX: base = h.U; stride = NS; off = 0; return XCAL_OK;
    case XCAL_FIELD_UY: base = h.U; stride = NS; off = 1; return XCAL_OK;
    case XCAL_FIELD_UZ:
      if (NS == 3) { base = h.U; stride = 3; off = 2; } else { base = h.Uz2; stride = 1; off = 0; }
      return XCAL_OK;
    case XCAL_FIELD_P: base = h.p; stride = 1; off = 0; return XCAL_OK;
    case XCAL_FIELD_K: case XCAL_FIELD_OMEGA: case XCAL_FIELD_NUT:
      if (h.model != XCAL_MODEL_KOMEGA) return fail(c, XCAL_ERR_STATE, "turbulence fields need the k-omega model");
      base = (field == XCAL_FIELD_K) ? h.k : (field == XCAL_FIELD_OMEGA) ? h.w : h.nut;
      stride = 1; off = 0;
      return XCAL_OK;
    default: return fail(c, XCAL_ERR_ARG, "unknown field");
  }
}

// Field transfer.  A context's fields live in device numbering, components
// interleaved.  Ordinary contexts copy the caller's array contiguously
// (pinned staging, one region per field) and scatter/gather with a small
// kernel applying the permutation; xcal_field_set returns without waiting
// for the copy.  Cluster-mode contexts (the serving loop) keep to copy
// engines only (a kernel could wait for SMs held by other contexts' runs):
// the permutation is applied on the host and every copy is contiguous, a
// vector component by a read-modify-write of the whole interleaved array.
int xcal_field_set(xcal_ctx c, int32_t field, const double *host, int64_t n) {
  if (!c || !host) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_field_set before xcal_case_setup");
  if (n != c->user.nc) return fail(c, XCAL_ERR_ARG, "field size mismatch");
  double *base; int stride, off;
  TRY(field_target(c, field, base, stride, off));
  CUDA_TRY(c, cudaSetDevice(c->device));
  double *hs = c->pin + (size_t)field * n;
  if (c->pin_busy[field]) {
    CUDA_TRY(c, cudaEventSynchronize(c->pin_ev[field]));
    c->pin_busy[field] = false;
  }
  if ((c->flags & XCAL_FLAG_CLUSTER) && stride == 1) {
    for (int64_t i = 0; i < n; ++i) hs[c->perm[i]] = host[i];
    CUDA_TRY(c, cudaMemcpyAsync(base, hs, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  } else if (c->flags & XCAL_FLAG_CLUSTER) {
    // one component of the interleaved vector array: read-modify-write of the
    // whole array with contiguous copies (a strided copy moves 8-byte rows)
    double *hv = c->pin;   // regions of ux, uy, uz: room for n*stride values
    for (int f = 0; f < 3; ++f)
      if (c->pin_busy[f]) {
        CUDA_TRY(c, cudaEventSynchronize(c->pin_ev[f]));
        c->pin_busy[f] = false;
      }
    const size_t bytes = sizeof(double) * (size_t)n * stride;
    CUDA_TRY(c, cudaMemcpyAsync(hv, base, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < n; ++i) hv[(size_t)c->perm[i] * stride + off] = host[i];
    CUDA_TRY(c, cudaMemcpyAsync(base, hv, bytes, cudaMemcpyHostToDevice, c->stream));
    for (int f = 0; f < 3; ++f) {
      CUDA_TRY(c, cudaEventRecord(c->pin_ev[f], c->stream));
      c->pin_busy[f] = true;
    }
    return XCAL_OK;
  } else {
    std::memcpy(hs, host, sizeof(double) * n);
    double *ds = c->d_stage + (size_t)field * n;
    CUDA_TRY(c, cudaMemcpyAsync(ds, hs, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, launch_field_scatter((int)n, ds, c->d_perm, base + off, stride, c->stream));
  }
  CUDA_TRY(c, cudaEventRecord(c->pin_ev[field], c->stream));
  c->pin_busy[field] = true;
  return XCAL_OK;
}

int xcal_field_get(xcal_ctx c, int32_t field, double *host, int64_t n) {
  if (!c || !host) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_field_get before xcal_case_setup");
  if (n != c->user.nc) return fail(c, XCAL_ERR_ARG, "field size mismatch");
  double *base; int stride, off;
  TRY(field_target(c, field, base, stride, off));
  CUDA_TRY(c, cudaSetDevice(c->device));
  double *hs = c->pin + (size_t)field * n;
  if (c->flags & XCAL_FLAG_CLUSTER) {
    // contiguous copy of the whole (interleaved) array, component picked here
    double *hv = (stride == 1) ? hs : c->pin;
    if (stride != 1)
      for (int f = 0; f < 3; ++f)
        if (c->pin_busy[f]) {
          CUDA_TRY(c, cudaEventSynchronize(c->pin_ev[f]));
          c->pin_busy[f] = false;
        }
    CUDA_TRY(c, cudaMemcpyAsync(hv, base, sizeof(double) * (size_t)n * stride, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < n; ++i) host[i] = hv[(size_t)c->perm[i] * stride + off];
  } else {
    double *ds = c->d_stage + (size_t)field * n;
    CUDA_TRY(c, launch_field_gather((int)n, base + off, c->d_perm, ds, stride, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(hs, ds, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    std::memcpy(host, hs, sizeof(double) * n);
  }
  c->pin_busy[field] = false;
  return XCAL_OK;
}

// -------------------------------------------------------------------- runs
static int run_program(xcal_ctx c, int prog, int32_t iters, double *Rux, double *Ruy, double *Ruz,
                       double *Rp, int32_t *kry, int32_t *done) {
  if (!c) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "run before xcal_case_setup");
  if (iters < 0) return fail(c, XCAL_ERR_ARG, "iterations < 0");
  CUDA_TRY(c, cudaSetDevice(c->device));
  KParams &h = c->hp;
  if (iters > c->run_cap) {
    c->rbuf.release();
    h.R = c->rbuf.alloc<double>((size_t)iters * 4);
    h.kry = c->rbuf.alloc<int>((size_t)iters * 5);
    if (!h.R || !h.kry) return fail(c, XCAL_ERR_OOM, "device allocation failed");
    c->run_cap = iters;
  }
  std::vector<double> ones((size_t)std::max(iters, 1) * 4, 1.0);
  CUDA_TRY(c, cudaMemcpyAsync(h.R, ones.data(), sizeof(double) * iters * 4, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(h.kry, 0, sizeof(int) * iters * 5, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(h.bar, 0, sizeof(Bar), c->stream));
  CUDA_TRY(c, cudaMemsetAsync(h.done, 0, sizeof(int), c->stream));
  h.mode = c->mode;
  h.conv = c->conv;
  h.abort_nan = (c->flags & XCAL_FLAG_ABORT_ON_NAN) ? 1 : 0;
  barrier_knobs(h);
  h.phase = nullptr;
  if (c->flags & XCAL_FLAG_PHASE_TIMERS) {
    if (!c->d_phase) {
      c->d_phase = c->cbuf.alloc<unsigned long long>(2 * NPH);
      if (!c->d_phase) return fail(c, XCAL_ERR_OOM, "device allocation failed");
    }
    CUDA_TRY(c, cudaMemsetAsync(c->d_phase, 0, sizeof(unsigned long long) * 2 * NPH, c->stream));
    h.phase = c->d_phase;
  }
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
  if (iters > 0)
    CUDA_TRY(c, launch_program(c->ns, h.prec == XCAL_PREC_MIXED, c->occ, c->mode, c->nblocks, &h, prog, iters,
                               c->stream));
  CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
  // results: one pinned block, one synchronisation
  const size_t nR = (size_t)std::max(iters, 1) * 4, nK = (size_t)std::max(iters, 1) * 5;
  const size_t nPh = 2 * NPH;
  const size_t need = sizeof(Bar) + 16 + sizeof(unsigned long long) * nPh + sizeof(double) * nR + sizeof(int) * nK;
  if (!c->rpin || c->rpin_n < need) {
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    stage_free(c, c->rpin);
    c->rpin = nullptr;
    CUDA_TRY(c, stage_alloc(c, &c->rpin, need));
    c->rpin_n = need;
  }
  Bar *hb = (Bar *)c->rpin;
  int *hdn = (int *)((char *)c->rpin + sizeof(Bar));
  unsigned long long *hph = (unsigned long long *)((char *)c->rpin + sizeof(Bar) + 16);
  double *R = (double *)(hph + nPh);
  int *K = (int *)(R + nR);
  CUDA_TRY(c, cudaMemcpyAsync(hb, h.bar, sizeof(Bar), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(hdn, h.done, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (h.phase)
    CUDA_TRY(c, cudaMemcpyAsync(hph, h.phase, sizeof(unsigned long long) * nPh, cudaMemcpyDeviceToHost, c->stream));
  if (iters > 0) {
    CUDA_TRY(c, cudaMemcpyAsync(R, h.R, sizeof(double) * iters * 4, cudaMemcpyDeviceToHost, c->stream));
    if (kry) CUDA_TRY(c, cudaMemcpyAsync(K, h.kry, sizeof(int) * iters * 5, cudaMemcpyDeviceToHost, c->stream));
  }
  if (c->evrun) {
    CUDA_TRY(c, cudaEventRecord(c->evrun, c->stream));
    CUDA_TRY(c, cudaEventSynchronize(c->evrun));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  const Bar bar = *hb;
  const int dn = *hdn;
  if (h.phase) std::copy(hph, hph + nPh, c->phase);
  else std::fill(c->phase, c->phase + nPh, 0ull);
  for (int i = 0; i < iters; ++i) {
    if (Rux) Rux[i] = R[4 * i];
    if (Ruy) Ruy[i] = R[4 * i + 1];
    if (Ruz) Ruz[i] = R[4 * i + 2];
    if (Rp) Rp[i] = R[4 * i + 3];
  }
  if (kry) std::copy(K, K + (size_t)iters * 5, kry);
  if (done) *done = dn;
  if (bar.err) return fail(c, XCAL_ERR_TIMEOUT, "device barrier timed out");
  if (bar.nonfinite)
    return fail(c, XCAL_ERR_NAN, "non-finite residual at iteration " + std::to_string(dn) + "; run stopped");
  return XCAL_OK;
}

int xcal_simple_run(xcal_ctx c, int32_t iters, double *Rux, double *Ruy, double *Ruz, double *Rp,
                    int32_t *kry, int32_t *done) {
  return run_program(c, PROG_SIMPLE, iters, Rux, Ruy, Ruz, Rp, kry, done);
}

int xcal_piso_run(xcal_ctx c, int32_t iters, double *Rux, double *Ruy, double *Ruz, double *Rp,
                  int32_t *kry, int32_t *done) {
  return run_program(c, PROG_PISO, iters, Rux, Ruy, Ruz, Rp, kry, done);
}

// ---------------------------------------------------------------- tuning
int xcal_autotune(xcal_ctx c, int32_t iters, xcal_tune_result *out) {
  if (!c || !out) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_autotune before xcal_case_setup");
  if (iters < 1 || iters > 1000) return fail(c, XCAL_ERR_ARG, "iterations must be 1..1000");
  if (c->flags & XCAL_FLAG_CLUSTER) return fail(c, XCAL_ERR_STATE, "cluster contexts keep their launch form");
  CUDA_TRY(c, cudaSetDevice(c->device));
  KParams &h = c->hp;
  const int n = c->prep.n, NS = c->ns;
  const int ntiles = (n + TILE - 1) / TILE;
  const bool gmres = h.wU.gmax > 0 || h.wP.gmax > 0;
  const int setup_ctas = c->nblocks;   // GMRES per-CTA scratch was sized for this many CTAs
  struct Cand {
    int mode, occ, nblocks, cg_fuse;
  };
  std::vector<Cand> cands;
  cands.push_back({c->mode, c->occ, c->nblocks, h.cg_fuse});   // the heuristic's form first
  auto add = [&](int mode, int occ, int nb, int fuse) {
    nb = std::max(1, nb);
    if (gmres && nb > setup_ctas) return;
    for (const Cand &k : cands)
      if (k.mode == mode && k.occ == occ && k.nblocks == nb && k.cg_fuse == fuse) return;
    cands.push_back({mode, occ, nb, fuse});
  };
  for (int occ = 0; occ <= (NS >= 2 ? 1 : 0); ++occ) {
    const int maxco = max_coresident_blocks(NS, occ, c->device);
    if (maxco < 1) continue;
    add(SYNC_GRID, occ, std::min(maxco, ntiles), 0);
    add(SYNC_GRID, occ, std::min(maxco / 2, ntiles), 0);
  }
  const int mc = max_cluster_blocks(NS, 0);
  if (ntiles <= mc) add(SYNC_CLUSTER, 0, ntiles, 0);
  if (h.kP.solver == XCAL_SOLVER_CG && h.AP.precon == XCAL_PRECON_DILU && h.nfl == 2)
    add(cands[0].mode, cands[0].occ, cands[0].nblocks, 1 - cands[0].cg_fuse);
  // fields the runs change, restored before every candidate and at the end
  DevBuf B;
  B.stream = c->stream;
  std::vector<std::pair<double *, size_t>> state = {{h.U, (size_t)n * NS}, {h.p, (size_t)n}};
  if (h.model == XCAL_MODEL_KOMEGA) {
    state.push_back({h.k, (size_t)n});
    state.push_back({h.w, (size_t)n});
    state.push_back({h.nut, (size_t)n});
  }
  std::vector<double *> saved;
  for (auto &f : state) {
    double *d = B.alloc<double>(f.second);
    if (!d) return fail(c, XCAL_ERR_OOM, "device allocation failed");
    CUDA_TRY(c, cudaMemcpyAsync(d, f.first, sizeof(double) * f.second, cudaMemcpyDeviceToDevice, c->stream));
    saved.push_back(d);
  }
  auto restore = [&]() -> int {
    for (size_t q = 0; q < state.size(); ++q)
      CUDA_TRY(c, cudaMemcpyAsync(state[q].first, saved[q], sizeof(double) * state[q].second,
                                  cudaMemcpyDeviceToDevice, c->stream));
    return XCAL_OK;
  };
  double best = 1e300, first = 0.0;
  size_t best_k = 0;
  const double conv = c->conv;
  c->conv = 0.0;   // time whole iterations: no early stop
  int st = XCAL_OK;
  for (size_t k = 0; k < cands.size() && st == XCAL_OK; ++k) {
    c->mode = cands[k].mode;
    c->occ = cands[k].occ;
    c->nblocks = cands[k].nblocks;
    h.cg_fuse = cands[k].cg_fuse;
    st = restore();
    if (st == XCAL_OK) st = run_program(c, PROG_SIMPLE, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (st == XCAL_OK) st = restore();
    if (st == XCAL_OK) st = run_program(c, PROG_SIMPLE, iters, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (st != XCAL_OK) break;
    const double ms = c->last_ms / iters;
    if (k == 0) first = ms;
    if (ms < best) {
      best = ms;
      best_k = k;
    }
  }
  c->conv = conv;
  const Cand &b = cands[best_k];
  c->mode = b.mode;
  c->occ = b.occ;
  c->nblocks = b.nblocks;
  h.cg_fuse = b.cg_fuse;
  const int rs = restore();
  if (st != XCAL_OK) return st;
  TRY(rs);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(c, h.prec)] = TuneChoice{b.mode, b.occ, b.nblocks, b.cg_fuse};
  }
  out->mode = b.mode;
  out->ctas = b.nblocks;
  out->ctas_per_sm = b.occ ? 4 : 2;
  out->cg_fused = b.cg_fuse;
  out->candidates = (int32_t)cands.size();
  out->ms_per_iteration = best;
  out->ms_default = first;
  return XCAL_OK;
}

int xcal_last_run_stats(xcal_ctx c, double *ms, double *phase, int32_t nph) {
  if (!c) return XCAL_ERR_ARG;
  if (ms) *ms = c->last_ms;
  for (int i = 0; phase && i < nph; ++i) phase[i] = (i < NPH) ? (double)c->phase[i] : 0.0;
  return XCAL_OK;
}

int xcal_last_run_phases(xcal_ctx c, int32_t nph, double *cycles, int64_t *count) {
  if (!c || nph < 0) return XCAL_ERR_ARG;
  for (int i = 0; i < nph; ++i) {
    if (cycles) cycles[i] = (i < NPH) ? (double)c->phase[i] : 0.0;
    if (count) count[i] = (i < NPH) ? (int64_t)c->phase[NPH + i] : 0;
  }
  return XCAL_OK;
}

int xcal_equation_get(xcal_ctx c, int32_t which, double *vals, double *b0, double *b1, double *b2) {
  if (!c) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "no case");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const KParams &h = c->hp;
  int n = c->prep.n, nnz = c->prep.nnz, NS = c->ns;
  size_t ne = (size_t)c->prep.W * c->prep.np;
  std::vector<double> ell(ne);
  auto to_csr = [&](const double *dev) -> int {
    CUDA_TRY(c, copy_sync(c, ell.data(), dev, sizeof(double) * ne, cudaMemcpyDeviceToHost));
    for (int k = 0; k < nnz; ++k) vals[k] = ell[c->prep.csr2ell[k]];
    return XCAL_OK;
  };
  if (which == 0) {
    if (vals) TRY(to_csr(h.AU.val));
    std::vector<double> b((size_t)n * NS);
    CUDA_TRY(c, copy_sync(c, b.data(), h.bU, sizeof(double) * n * NS, cudaMemcpyDeviceToHost));
    double *dst[3] = {b0, b1, b2};
    for (int d = 0; d < NS; ++d)
      if (dst[d]) for (int i = 0; i < n; ++i) dst[d][i] = b[(size_t)i * NS + d];
    return XCAL_OK;
  }
  if (which == 1) {
    if (vals) TRY(to_csr(h.AP.val));
    if (b0) CUDA_TRY(c, copy_sync(c, b0, h.bP, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return XCAL_OK;
  }
  return fail(c, XCAL_ERR_ARG, "which must be 0 (momentum) or 1 (pressure)");
}

// -------------------------------------------------------- standalone solve
int xcal_linear_solve(xcal_ctx c, int32_t solver, int32_t precon, int64_t n64, const int32_t *row_ptr,
                      const int32_t *col, const double *val, const double *b, double *x, int32_t itmax,
                      double atol, double rtol, int32_t *niter, double *final_rnorm) {
  if (!c || !row_ptr || !col || !val || !b || !x || n64 <= 0 || n64 > (1 << 30)) return XCAL_ERR_ARG;
  {
    xcal_solver_cfg sc{};
    sc.solver = solver; sc.preconditioner = precon; sc.itmax = itmax;
    TRY(check_solver(c, sc, "xcal_linear_solve"));
  }
  CUDA_TRY(c, cudaSetDevice(c->device));
  int n = (int)n64;
  if (row_ptr[0] != 0) return fail(c, XCAL_ERR_ARG, "row_ptr[0] must be 0");
  for (int i = 0; i < n; ++i) {
    if (row_ptr[i + 1] < row_ptr[i]) return fail(c, XCAL_ERR_ARG, "row_ptr not monotone");
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
      if (col[k] < 0 || col[k] >= n) return fail(c, XCAL_ERR_ARG, "column out of range");
      if (k > row_ptr[i] && col[k] <= col[k - 1]) return fail(c, XCAL_ERR_ARG, "columns not strictly ascending");
    }
  }
  int nnz = row_ptr[n];
  std::vector<int> rp(row_ptr, row_ptr + n + 1), cl(col, col + nnz), dg(n, -1), ts(nnz, -1);
  auto find = [&](int r, int cc) -> int {
    auto bb = cl.begin() + rp[r], ee = cl.begin() + rp[r + 1];
    auto it = std::lower_bound(bb, ee, cc);
    return (it != ee && *it == cc) ? (int)(it - cl.begin()) : -1;
  };
  for (int i = 0; i < n; ++i) {
    dg[i] = find(i, i);
    if (dg[i] < 0) return fail(c, XCAL_ERR_ARG, "missing diagonal entry");
  }
  for (int r = 0; r < n; ++r)
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      ts[k] = find(cl[k], r);
      if (ts[k] < 0) return fail(c, XCAL_ERR_ARG, "pattern not symmetric");
    }
  std::vector<int> fl(n, 0), bl(n, 0);
  for (int i = 0; i < n; ++i) { int l = 0; for (int k = rp[i]; k < dg[i]; ++k) l = std::max(l, fl[cl[k]] + 1); fl[i] = l; }
  for (int i = n - 1; i >= 0; --i) { int l = 0; for (int k = dg[i] + 1; k < rp[i + 1]; ++k) l = std::max(l, bl[cl[k]] + 1); bl[i] = l; }
  int nfl = 1, nbl = 1;
  for (int i = 0; i < n; ++i) { nfl = std::max(nfl, fl[i] + 1); nbl = std::max(nbl, bl[i] + 1); }
  int W = 0;
  for (int i = 0; i < n; ++i) W = std::max(W, rp[i + 1] - rp[i]);
  int np = ((n + TILE - 1) / TILE) * TILE;
  std::vector<int> ecol((size_t)W * np, -1), etp((size_t)W * np, -1), edp(np, 0), c2e(nnz);
  std::vector<double> ev((size_t)W * np, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      size_t e = (size_t)(k - rp[i]) * np + i;
      ecol[e] = cl[k]; ev[e] = val[k]; c2e[k] = (int)e;
    }
  for (int i = 0; i < n; ++i) {
    edp[i] = c2e[dg[i]];
    for (int k = rp[i]; k < rp[i + 1]; ++k) etp[c2e[k]] = c2e[ts[k]];
  }
  fl.resize(np, 0);
  bl.resize(np, 0);
  DevBuf B;
  B.stream = c->stream;
  KParams h;
  memset(&h, 0, sizeof(h));
  h.n = n; h.ntiles = np / TILE; h.np = np;
  TRY(upload_c(c, B, h.flev, fl)); TRY(upload_c(c, B, h.blev, bl));
  h.nfl = nfl; h.nbl = nbl;
  TRY(upload_c(c, B, h.AU.col, ecol)); TRY(upload_c(c, B, h.AU.tpos, etp)); TRY(upload_c(c, B, h.AU.dpos, edp));
  h.AU.W = W; h.AU.np = np;
  std::vector<double> bb(b, b + n), xx(x, x + n);
  TRY(upload(c, B, h.AU.val, ev));
  TRY(upload(c, B, h.sb, bb));
  TRY(upload(c, B, h.U, xx));
  h.AU.precon = precon;
  bool ok = true;
  auto A = [&](size_t cnt) { double *p = B.alloc<double>(cnt); if (!p) ok = false; return p; };
  h.AU.Dpiv = A(n); h.AU.Dinv = A(n);
  h.AU.fval = (precon == XCAL_PRECON_ILU0) ? A(ev.size()) : nullptr;
  KWork &w = h.wU;
  w.x = A(n); w.s = A(n); w.t = A(n); w.q = A(n);
  for (int k = 0; k < 2; ++k) { w.r[k] = A(n); w.p[k] = A(n); w.v[k] = A(n); }
  h.part = A((size_t)2 * MAXK * h.ntiles);   // two buffers, used in turn
  h.solve_out = A(2);
  h.bar = B.alloc<Bar>(1);
  h.done = B.alloc<int>(1);
  KParams *dp = B.alloc<KParams>(1);
  if (!ok || !h.bar || !h.done || !dp) return fail(c, XCAL_ERR_OOM, "device allocation failed");
  h.solve_solver = solver; h.solve_itmax = itmax; h.solve_atol = atol; h.solve_rtol = rtol;
  int mode, nb;
  {
    int saved_ns = c->ns, saved_mode = c->mode, saved_nb = c->nblocks, saved_occ = c->occ;
    c->ns = 1;
    choose_launch(c, n, h);
    mode = c->mode; nb = c->nblocks;
    c->ns = saved_ns; c->mode = saved_mode; c->nblocks = saved_nb; c->occ = saved_occ;
  }
  h.mode = mode;
  if (solver == XCAL_SOLVER_GMRES) {
    double *g1 = nullptr, *g2 = nullptr;
    std::function<double *(size_t)> allocD = [&](size_t cnt) { return A(cnt); };
    gmres_alloc(h.wU, itmax, (size_t)n, 1, nb, A, g1, g2, allocD);
    if (!ok) return fail(c, XCAL_ERR_OOM, "device allocation failed");
  }
  CUDA_TRY(c, cudaMemsetAsync(h.bar, 0, sizeof(Bar), c->stream));
  barrier_knobs(h);
  CUDA_TRY(c, launch_program(1, 0, 0, mode, nb, &h, PROG_SOLVE, 1, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  Bar bar;
  double so[2];
  CUDA_TRY(c, copy_sync(c, &bar, h.bar, sizeof(Bar), cudaMemcpyDeviceToHost));
  CUDA_TRY(c, copy_sync(c, so, h.solve_out, sizeof(so), cudaMemcpyDeviceToHost));
  CUDA_TRY(c, copy_sync(c, x, h.U, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (niter) *niter = (int32_t)so[0];
  if (final_rnorm) *final_rnorm = so[1];
  if (bar.err) return fail(c, XCAL_ERR_TIMEOUT, "device barrier timed out");
  return XCAL_OK;
}

// ------------------------------------------------------ operator level
}  // extern "C"

// The context's ELL values of a CSR matrix on its pattern (xcal_mesh_csr order).
static void ell_of_csr(xcal_ctx c, const double *vals, std::vector<double> &ell) {
  const Prep &P = c->prep;
  ell.assign((size_t)P.W * P.np, 0.0);
  for (int k = 0; k < P.nnz; ++k) ell[P.csr2ell[k]] = vals[k];
}

extern "C" {

int xcal_assemble(xcal_ctx c, const xcal_term *terms, int32_t nterms, const xcal_source *sources, int32_t nsources,
                  const xcal_bc *bcs, int32_t nbc, int32_t comp, const double *phi, const double *prev, double dt,
                  double *vals, double *b) {
  if (!c) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "xcal_assemble before xcal_mesh_upload");
  if (!terms || nterms < 1 || nsources < 0 || (nsources > 0 && !sources) || nbc < 0 || (nbc > 0 && !bcs) ||
      comp < 0 || comp > 2 || !vals || !b)
    return fail(c, XCAL_ERR_ARG, "bad xcal_assemble arguments");
  const int n = c->prep.n, nf = c->prep.nf;
  bool si_wall = false, euler = false;
  for (int t = 0; t < nterms; ++t) {
    const xcal_term &T = terms[t];
    if (T.kind < XCAL_TERM_TIME || T.kind > XCAL_TERM_SI) return fail(c, XCAL_ERR_ARG, "unknown term kind");
    if (T.kind != XCAL_TERM_TIME && !T.flux) return fail(c, XCAL_ERR_ARG, "term without its flux field");
    if (T.kind == XCAL_TERM_DIVERGENCE && T.scheme != XCAL_DIV_LINEAR && T.scheme != XCAL_DIV_UPWIND)
      return fail(c, XCAL_ERR_UNSUPPORTED, "divergence scheme not available");
    if (T.kind == XCAL_TERM_LAPLACIAN && T.scheme != XCAL_LAP_LINEAR)
      return fail(c, XCAL_ERR_UNSUPPORTED, "laplacian scheme not available");
    if (T.kind == XCAL_TERM_TIME && T.scheme == XCAL_TIME_EULER) euler = true;
    if (T.kind == XCAL_TERM_SI) si_wall = true;
  }
  for (int q = 0; q < nsources; ++q)
    if (!sources[q].field) return fail(c, XCAL_ERR_ARG, "source without its field");
  if (euler && (!prev || !(dt > 0.0))) return fail(c, XCAL_ERR_ARG, "the Euler term needs prev and dt > 0");
  if (si_wall && nbc > 0 && !phi) return fail(c, XCAL_ERR_ARG, "the Si term's wall condition needs phi");
  CUDA_TRY(c, cudaSetDevice(c->device));
  DevBuf B;
  B.stream = c->stream;
  DevSink S(c, B);
  std::vector<OpTerm> dt_(nterms);
  for (int t = 0; t < nterms; ++t) {
    const xcal_term &T = terms[t];
    dt_[t].kind = T.kind;
    dt_[t].scheme = T.scheme;
    dt_[t].sign = T.sign;
    const size_t len = (T.kind == XCAL_TERM_SI) ? n : nf;
    dt_[t].flux = (T.kind == XCAL_TERM_TIME) ? nullptr : (const double *)S.put(T.flux, sizeof(double) * len);
  }
  std::vector<OpSource> ds(std::max(nsources, 1));
  for (int q = 0; q < nsources; ++q) {
    ds[q].sign = sources[q].sign;
    ds[q].field = (const double *)S.put(sources[q].field, sizeof(double) * n);
  }
  const OpTerm *dterms = S.put_v(dt_);
  const OpSource *dsrc = S.put_v(ds);
  const double *dphi = phi ? (const double *)S.put(phi, sizeof(double) * n) : S.zeros_n<double>(n);
  const double *dprev = prev ? (const double *)S.put(prev, sizeof(double) * n) : S.zeros_n<double>(n);
  FieldBC bc{};
  std::vector<BcEntry> tab;
  TRY(build_bc(c, S, bcs, nbc, bc, tab, true, "the equation"));
  double *dval = S.zeros_n<double>((size_t)c->prep.W * c->prep.np);
  double *db = S.zeros_n<double>(n);
  if (!S.ok()) return fail(c, S.error(), S.message());
  CUDA_TRY(c, launch_assemble_terms(c->hp, dterms, nterms, dsrc, nsources, bc, nbc > 0 ? 1 : 0, comp, dphi, dprev,
                                    dt, dval, db, c->stream));
  std::vector<double> ell((size_t)c->prep.W * c->prep.np);
  CUDA_TRY(c, copy_sync(c, ell.data(), dval, sizeof(double) * ell.size(), cudaMemcpyDeviceToHost));
  CUDA_TRY(c, copy_sync(c, b, db, sizeof(double) * n, cudaMemcpyDeviceToHost));
  for (int k = 0; k < c->prep.nnz; ++k) vals[k] = ell[c->prep.csr2ell[k]];
  return XCAL_OK;
}

int xcal_spmv(xcal_ctx c, const double *vals, const double *x, double *y) {
  if (!c || !vals || !x || !y) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "xcal_spmv before xcal_mesh_upload");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const int n = c->prep.n;
  std::vector<double> ell;
  ell_of_csr(c, vals, ell);
  DevBuf B;
  B.stream = c->stream;
  DevSink S(c, B);
  Mat A = c->hp.AU;
  A.val = S.put_v(ell);
  const double *dx = (const double *)S.put(x, sizeof(double) * n);
  double *dy = S.scratch_n<double>(n);
  if (!S.ok()) return fail(c, S.error(), S.message());
  CUDA_TRY(c, launch_spmv(A, n, dx, dy, c->stream));
  CUDA_TRY(c, copy_sync(c, y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return XCAL_OK;
}

int xcal_dilu(xcal_ctx c, const double *vals, const double *r, double *y) {
  if (!c || !vals || !r || !y) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "xcal_dilu before xcal_mesh_upload");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const int n = c->prep.n;
  std::vector<double> ell;
  ell_of_csr(c, vals, ell);
  DevBuf B;
  B.stream = c->stream;
  DevSink S(c, B);
  Mat A = c->hp.AU;
  A.val = S.put_v(ell);
  A.Dpiv = S.scratch_n<double>(n);
  A.Dinv = S.scratch_n<double>(n);
  A.fval = nullptr;
  A.precon = XCAL_PRECON_DILU;
  const double *dr = (const double *)S.put(r, sizeof(double) * n);
  double *dy = S.zeros_n<double>(n);
  if (!S.ok()) return fail(c, S.error(), S.message());
  CUDA_TRY(c, launch_dilu(A, n, c->hp.flev, c->hp.blev, c->hp.nfl, c->hp.nbl, dr, dy, c->stream));
  CUDA_TRY(c, copy_sync(c, y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return XCAL_OK;
}

int xcal_grad(xcal_ctx c, const double *phi, const xcal_bc *bcs, int32_t nbc, double *grad) {
  if (!c || !phi || !grad || nbc < 0 || (nbc > 0 && !bcs)) return XCAL_ERR_ARG;
  if (!c->have_mesh) return fail(c, XCAL_ERR_STATE, "xcal_grad before xcal_mesh_upload");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const int n = c->prep.n, nf = c->prep.nf;
  DevBuf B;
  B.stream = c->stream;
  DevSink S(c, B);
  FieldBC bc{};
  std::vector<BcEntry> tab;
  TRY(build_bc(c, S, bcs, nbc, bc, tab, false, "the gradient"));
  const double *dphi = (const double *)S.put(phi, sizeof(double) * n);
  double *pf = S.scratch_n<double>(nf);
  double *dg = S.scratch_n<double>((size_t)3 * n);
  if (!S.ok()) return fail(c, S.error(), S.message());
  CUDA_TRY(c, launch_grad(c->hp, bc, dphi, pf, dg, c->stream));
  CUDA_TRY(c, copy_sync(c, grad, dg, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
  return XCAL_OK;
}

// ------------------------------------------------------------- residual!
static int check_csr(xcal_ctx c, int n, const int32_t *rp, const int32_t *col) {
  if (rp[0] != 0) return fail(c, XCAL_ERR_ARG, "row_ptr[0] must be 0");
  for (int i = 0; i < n; ++i) {
    if (rp[i + 1] < rp[i]) return fail(c, XCAL_ERR_ARG, "row_ptr not monotone");
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      if (col[k] < 0 || col[k] >= n) return fail(c, XCAL_ERR_ARG, "column out of range");
      if (k > rp[i] && col[k] <= col[k - 1]) return fail(c, XCAL_ERR_ARG, "columns not strictly ascending");
    }
  }
  return XCAL_OK;
}

int xcal_residual(xcal_ctx c, int64_t n64, const int32_t *row_ptr, const int32_t *col, const double *val,
                  const double *x, const double *b, double *R) {
  if (!c || !row_ptr || !col || !val || !x || !b || !R || n64 <= 0 || n64 > (1 << 30)) return XCAL_ERR_ARG;
  CUDA_TRY(c, cudaSetDevice(c->device));
  int n = (int)n64;
  TRY(check_csr(c, n, row_ptr, col));
  int nnz = row_ptr[n];
  int ntiles = (n + TILE - 1) / TILE;
  DevBuf B;
  B.stream = c->stream;
  std::vector<int> rp(row_ptr, row_ptr + n + 1), cl(col, col + nnz);
  std::vector<double> vv(val, val + nnz), xx(x, x + n), bb(b, b + n);
  int *drp, *dcl;
  double *dv, *dx, *db;
  TRY(upload(c, B, drp, rp)); TRY(upload(c, B, dcl, cl)); TRY(upload(c, B, dv, vv));
  TRY(upload(c, B, dx, xx)); TRY(upload(c, B, db, bb));
  double *part = B.alloc<double>((size_t)2 * ntiles), *out = B.alloc<double>(1);
  if (!part || !out) return fail(c, XCAL_ERR_OOM, "device allocation failed");
  CUDA_TRY(c, launch_residual(n, drp, dcl, dv, dx, db, part, out, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(R, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return XCAL_OK;
}

// Allocation-free residual!: same kernels as xcal_residual, device pointers in
// and out, partial sums in the library's fixed scratch array (no cudaMalloc,
// cudaFree or other allocation).  The first call on a device resolves the
// scratch address; make it before any stream capture.  Calls that overlap on
// the GPU (other threads, other contexts) share the scratch and race.
int xcal_residual_noalloc(xcal_ctx c, int64_t n64, const int32_t *d_row_ptr, const int32_t *d_col,
                          const double *d_val, const double *d_x, const double *d_b, double *d_R) {
  if (!c) return XCAL_ERR_ARG;
  if (!d_row_ptr || !d_col || !d_val || !d_x || !d_b || !d_R) return fail(c, XCAL_ERR_ARG, "null device pointer");
  if (n64 <= 0) return fail(c, XCAL_ERR_ARG, "n must be positive");
  if (n64 > (int64_t)noalloc_max_rows())
    return fail(c, XCAL_ERR_ARG, "n = " + std::to_string(n64) + " exceeds the allocation-free limit of " +
                                     std::to_string(noalloc_max_rows()) + " rows");
  CUDA_TRY(c, cudaSetDevice(c->device));
  double *scratch = nullptr;
  int *bad = nullptr;
  CUDA_TRY(c, noalloc_scratch(c->device, &scratch, &bad));
  CUDA_TRY(c, cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  CUDA_TRY(c, launch_residual((int)n64, d_row_ptr, d_col, d_val, d_x, d_b, scratch, d_R, c->stream, bad));
  int hbad = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (hbad)
    return fail(c, XCAL_ERR_ARG, std::string("CSR out of bounds:") + ((hbad & 1) ? " row_ptr range" : "") +
                                     ((hbad & 2) ? " column index" : "") + " (those entries were skipped)");
  return XCAL_OK;
}


// ------------------------------------------------------- post-processing
static void put_num(std::string &out, double v) {
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof(buf), v);
  out.append(buf, r.ptr);
}

int xcal_vtk_write(const char *name, const xcal_mesh_desc *d, int32_t nfields, const char *const *labels,
                   const int32_t *ncomp, const double *const *data) {
  if (!name || !d || nfields < 0 || (nfields > 0 && (!labels || !ncomp || !data))) return XCAL_ERR_ARG;
  if (d->nnodes <= 0 || !d->node_coords || !d->cell_nodes_ptr || !d->cell_nodes) return XCAL_ERR_UNSUPPORTED;
  for (int f = 0; f < nfields; ++f)
    if (!labels[f] || !data[f] || (ncomp[f] != 1 && ncomp[f] != 3)) return XCAL_ERR_ARG;
  const int64_t nc = d->ncells, nn = d->nnodes;
  std::string out;
  out.reserve((size_t)(nn * 60 + nc * 40 * (2 + nfields)));
  out += "# vtk DataFile Version 3.0\njCFD simulation data\nASCII\nDATASET UNSTRUCTURED_GRID\n";
  out += "POINTS " + std::to_string(nn) + " double\n";
  for (int64_t i = 0; i < nn; ++i) {
    put_num(out, d->node_coords[3 * i]); out += ' ';
    put_num(out, d->node_coords[3 * i + 1]); out += ' ';
    put_num(out, d->node_coords[3 * i + 2]); out += '\n';
  }
  const int64_t total = d->cell_nodes_ptr[nc] - d->cell_nodes_ptr[0];
  out += "CELLS " + std::to_string(nc) + " " + std::to_string(total + nc) + "\n";
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t b = d->cell_nodes_ptr[c] - 1, e = d->cell_nodes_ptr[c + 1] - 1;
    out += std::to_string(e - b) + " ";          // println(io, nNodes, " ", nodes): nodes = " id0 id1 ..."
    for (int64_t k = b; k < e; ++k) {
      if (d->cell_nodes[k] < 1 || d->cell_nodes[k] > nn) return XCAL_ERR_MESH;
      out += ' ';
      out += std::to_string(d->cell_nodes[k] - 1);
    }
    out += '\n';
  }
  out += "CELL_TYPES " + std::to_string(nc) + "\n";
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t k = d->cell_nodes_ptr[c + 1] - d->cell_nodes_ptr[c];
    out += (k == 3) ? "5\n" : (k == 4) ? "9\n" : "7\n";
  }
  out += "CELL_DATA " + std::to_string(nc) + "\n";
  for (int f = 0; f < nfields; ++f) {
    const double *v = data[f];
    if (ncomp[f] == 1) {
      out += std::string("SCALARS ") + labels[f] + " double 1\nLOOKUP_TABLE CellColors\n";
      for (int64_t c = 0; c < nc; ++c) { put_num(out, v[c]); out += '\n'; }
    } else {
      out += std::string("VECTORS ") + labels[f] + " double\n";
      for (int64_t c = 0; c < nc; ++c) {
        put_num(out, v[c]); out += ' ';
        put_num(out, v[nc + c]); out += ' ';
        put_num(out, v[2 * nc + c]); out += '\n';
      }
    }
  }
  FILE *fp = fopen((std::string(name) + ".vtk").c_str(), "wb");
  if (!fp) return XCAL_ERR_IO;
  const size_t w = fwrite(out.data(), 1, out.size(), fp);
  const int cl = fclose(fp);
  return (w == out.size() && cl == 0) ? XCAL_OK : XCAL_ERR_IO;
}

static int host_fields(xcal_ctx c, std::vector<double> &U, std::vector<double> &p, std::vector<double> *nut) {
  const int64_t n = c->user.nc;
  U.assign(3 * (size_t)n, 0.0);
  p.assign((size_t)n, 0.0);
  for (int d = 0; d < 3; ++d) TRY(xcal_field_get(c, XCAL_FIELD_UX + d, U.data() + (size_t)d * n, n));
  TRY(xcal_field_get(c, XCAL_FIELD_P, p.data(), n));
  if (nut) {
    nut->assign((size_t)n, 0.0);
    if (c->hp.model == XCAL_MODEL_KOMEGA) TRY(xcal_field_get(c, XCAL_FIELD_NUT, nut->data(), n));
  }
  return XCAL_OK;
}

int xcal_model2vtk(xcal_ctx c, const char *name) {
  if (!c || !name) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_model2vtk before xcal_case_setup");
  std::vector<double> U, p, k, w, nut;
  TRY(host_fields(c, U, p, nullptr));
  std::vector<const char *> labels = {"U", "p"};
  std::vector<int32_t> nco = {3, 1};
  std::vector<const double *> data = {U.data(), p.data()};
  if (c->hp.model == XCAL_MODEL_KOMEGA) {
    const int64_t n = c->user.nc;
    k.resize(n); w.resize(n); nut.resize(n);
    TRY(xcal_field_get(c, XCAL_FIELD_K, k.data(), n));
    TRY(xcal_field_get(c, XCAL_FIELD_OMEGA, w.data(), n));
    TRY(xcal_field_get(c, XCAL_FIELD_NUT, nut.data(), n));
    labels.insert(labels.end(), {"k", "omega", "nut"});
    nco.insert(nco.end(), {1, 1, 1});
    data.insert(data.end(), {k.data(), w.data(), nut.data()});
  }
  xcal_mesh_desc d;
  fill_desc(c->user, &d);
  const int st = xcal_vtk_write(name, &d, (int32_t)labels.size(), labels.data(), nco.data(), data.data());
  if (st == XCAL_ERR_UNSUPPORTED) return fail(c, st, "mesh has no node coordinates (xcal_mesh_desc.nnodes = 0)");
  if (st) return fail(c, st, "VTK write failed");
  return XCAL_OK;
}

// Dirichlet value of U on a patch (the reference looks it up in U.BCs)
static int patch_Uw(xcal_ctx c, int32_t patch, double Uw[3]) {
  for (const xcal_bc &b : c->bcU_host)
    if (b.patch == patch) {
      if (b.type != XCAL_BC_DIRICHLET) return fail(c, XCAL_ERR_ARG, "patch has no Dirichlet U condition");
      for (int d = 0; d < 3; ++d) Uw[d] = b.value[d];
      return XCAL_OK;
    }
  return fail(c, XCAL_ERR_ARG, "patch has no U condition");
}

int xcal_wall_shear_stress(xcal_ctx c, int32_t patch, double *tau, double *pos, int64_t cap, int64_t *count) {
  if (!c || !count) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_wall_shear_stress before xcal_case_setup");
  const HostMesh &M = c->user;
  if (patch < 0 || patch >= (int32_t)M.pname.size()) return fail(c, XCAL_ERR_ARG, "patch index out of range");
  const int64_t a = M.pptr[patch], b = M.pptr[patch + 1];
  *count = b - a;
  if (!tau || !pos || cap < b - a) return fail(c, XCAL_ERR_ARG, "output arrays smaller than the patch");
  double Uw[3];
  TRY(patch_Uw(c, patch, Uw));
  std::vector<double> U, p, nut;
  TRY(host_fields(c, U, p, &nut));
  const int64_t n = M.nc;
  for (int64_t i = a; i < b; ++i) {
    const int64_t f = M.pfaces[i], cell = M.pcells[i];
    const double *nrm = &M.fn[3 * f];
    double ud[3], up[3];
    for (int d = 0; d < 3; ++d) ud[d] = U[(size_t)d * n + cell] - Uw[d];
    const double dn = (ud[0] * nrm[0] + ud[1] * nrm[1]) + ud[2] * nrm[2];
    for (int d = 0; d < 3; ++d) up[d] = ud[d] - dn * nrm[d];
    const double nueff = c->hp.nu + nut[cell];
    for (int d = 0; d < 3; ++d) {
      tau[3 * (i - a) + d] = (up[d] / M.fdelta[f]) * nueff;
      pos[3 * (i - a) + d] = M.fc[3 * f + d];
    }
  }
  return XCAL_OK;
}

int xcal_pressure_force(xcal_ctx c, int32_t patch, double rho, double F[3]) {
  if (!c || !F) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_pressure_force before xcal_case_setup");
  const HostMesh &M = c->user;
  if (patch < 0 || patch >= (int32_t)M.pname.size()) return fail(c, XCAL_ERR_ARG, "patch index out of range");
  std::vector<double> U, p;
  TRY(host_fields(c, U, p, nullptr));
  double s[3] = {0.0, 0.0, 0.0};
  for (int64_t i = M.pptr[patch]; i < M.pptr[patch + 1]; ++i) {
    const int64_t f = M.pfaces[i], cell = M.pcells[i];
    for (int d = 0; d < 3; ++d) s[d] += p[cell] * (M.farea[f] * M.fn[3 * f + d]);
  }
  for (int d = 0; d < 3; ++d) F[d] = rho * s[d];
  return XCAL_OK;
}

int xcal_viscous_force(xcal_ctx c, int32_t patch, double rho, double F[3]) {
  if (!c || !F) return XCAL_ERR_ARG;
  if (!c->have_case) return fail(c, XCAL_ERR_STATE, "xcal_viscous_force before xcal_case_setup");
  const HostMesh &M = c->user;
  if (patch < 0 || patch >= (int32_t)M.pname.size()) return fail(c, XCAL_ERR_ARG, "patch index out of range");
  double Uw[3];
  TRY(patch_Uw(c, patch, Uw));
  std::vector<double> U, p, nut;
  TRY(host_fields(c, U, p, &nut));
  const int64_t n = M.nc;
  double s[3] = {0.0, 0.0, 0.0};
  for (int64_t i = M.pptr[patch]; i < M.pptr[patch + 1]; ++i) {
    const int64_t f = M.pfaces[i], cell = M.pcells[i];
    const double *nrm = &M.fn[3 * f];
    double ud[3];
    for (int d = 0; d < 3; ++d) ud[d] = U[(size_t)d * n + cell] - Uw[d];
    const double dn = (ud[0] * nrm[0] + ud[1] * nrm[1]) + ud[2] * nrm[2];
    for (int d = 0; d < 3; ++d) {
      const double g = (ud[d] - dn * nrm[d]) / M.fdelta[f];
      s[d] += g * M.farea[f] * (c->hp.nu + nut[cell]);
    }
  }
  for (int d = 0; d < 3; ++d) F[d] = rho * s[d];
  return XCAL_OK;
}

}  // extern "C"

// ------------------------------------------------------- serving images
namespace xcal {

int build_case_image(const xcal_mesh_desc *mesh, int renumber, const xcal_case *cfg, const double *U0,
                     const double *p0, double tolerance, int iters, int gmres_ctas, Sink &sink, CaseImage &out,
                     std::string &err) {
  if (!mesh || !cfg || !U0 || !p0 || iters < 1 || gmres_ctas < 1) {
    err = "bad case image arguments";
    return XCAL_ERR_ARG;
  }
  xcal_ctx_s c;   // host-side context: no stream, no device work
  c.flags = XCAL_FLAG_CLUSTER;
  int st = mesh_prepare(&c, mesh, renumber);
  if (st == XCAL_OK) st = check_case(&c, cfg);
  if (st == XCAL_OK) {
    c.mode = SYNC_GRID;
    c.nblocks = gmres_ctas;   // GMRES per-CTA scratch
    st = mesh_arrays(&c, sink);
  }
  if (st == XCAL_OK) st = case_arrays(&c, cfg, sink, U0, p0);
  if (st != XCAL_OK) {
    err = c.err;
    return st;
  }
  KParams &h = c.hp;
  // run arrays: residual histories start at 1.0 as in the reference, Krylov counts at 0
  std::vector<double> ones((size_t)iters * 4, 1.0);
  h.R = sink.put_v(ones);
  h.kry = sink.zeros_n<int>((size_t)iters * 5);
  if (!sink.ok()) {
    err = sink.message();
    return sink.error();
  }
  h.conv = tolerance;
  h.abort_nan = 1;
  h.mode = SYNC_GRID;
  h.cg_fuse = 0;
  h.phase = nullptr;
  h.bar = nullptr;   // the serving loop gives the case a barrier word when it starts
  out.prm = h;
  out.ns = c.ns;
  out.n = c.prep.n;
  out.ntiles = h.ntiles;
  out.perm = c.perm;
  return XCAL_OK;
}

}  // namespace xcal
