// Launch of the persistent device program (xcal_kernel.cu instantiations):
// block, cluster or cooperative grid launch, and the occupancy queries the
// launch configuration uses.
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "xcal_device.cuh"
#include "xcal_kernel.h"

namespace xcal {

const void *program_kernel_d1();
const void *program_kernel_d2();
const void *program_kernel_d3();
const void *program_kernel_f2();
const void *program_kernel_f3();
const void *program_kernel_d2o();
const void *program_kernel_d3o();
const void *program_kernel_f2o();
const void *program_kernel_f3o();
const void *serve_kernel_d2o();
const void *serve_kernel_d3o();
const void *serve_kernel_f2o();
const void *serve_kernel_f3o();

// Serving kernel of a dimension and precision (4-CTA/SM builds).
const void *serve_kernel_ptr(int ns, int mixed) {
  if (ns == 2) return mixed ? serve_kernel_f2o() : serve_kernel_d2o();
  if (ns == 3) return mixed ? serve_kernel_f3o() : serve_kernel_d3o();
  return nullptr;
}

// CTAs of the serving launch: every CTA that can be resident at once (a
// cooperative launch of this size is guaranteed co-resident).
int serve_grid(int ns, int mixed, int device) {
  const void *fn = serve_kernel_ptr(ns, mixed);
  if (!fn) return 0;
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, TPB, 0) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

const void *program_kernel_ptr(int ns, int mixed, int occ) {
  if (ns == 1) return program_kernel_d1();
  if (ns == 2) {
    if (occ) return mixed ? program_kernel_f2o() : program_kernel_d2o();
    return mixed ? program_kernel_f2() : program_kernel_d2();
  }
  if (occ) return mixed ? program_kernel_f3o() : program_kernel_d3o();
  return mixed ? program_kernel_f3() : program_kernel_d3();
}

// Non-portable cluster sizes are allowed once per kernel and device; the
// attribute is process-wide state, so there is no reason to set it again on
// every launch (and a serving loop launches from many threads at once).
static cudaError_t allow_large_clusters(const void *fn) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, bool> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({fn, dev})) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess) done[{fn, dev}] = true;
  return e;
}

cudaError_t launch_program(int ns, int mixed, int occ, int mode, int nblocks, const KParams *hparams, int prog,
                           int iters, cudaStream_t stream) {
  const void *fn = program_kernel_ptr(ns, mixed, occ);
  void *args[3];
  args[0] = (void *)hparams;
  args[1] = (void *)&prog;
  args[2] = (void *)&iters;
  if (mode == SYNC_BLOCK) return cudaLaunchKernel(fn, dim3(1), dim3(TPB), args, 0, stream);
  if (mode == SYNC_CLUSTER) {
    cudaError_t e = allow_large_clusters(fn);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(TPB);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = nblocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
  }
  return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(TPB), args, 0, stream);
}

// Load every build of the program on the current device now.  With lazy
// module loading a build is loaded on its first query or launch, and loading
// can wait for kernels already running on the device; a serving loop, whose
// runs overlap, loads them all before its first case.
void preload_programs() {
  for (int ns = 1; ns <= 3; ++ns)
    for (int mixed = 0; mixed <= 1; ++mixed)
      for (int occ = 0; occ <= 1; ++occ) {
        if (ns == 1 && (mixed || occ)) continue;
        cudaFuncAttributes a;
        if (cudaFuncGetAttributes(&a, program_kernel_ptr(ns, mixed, occ)) != cudaSuccess) (void)cudaGetLastError();
      }
}

// Occupancy probes: a failed query counts as zero and its error is consumed
// here, so that it is not reported later by an unrelated call that reads the
// runtime's last error.
int max_coresident_blocks(int ns, int occ, int device) {
  int per_sm = 0, sms = 0, per_sm32 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, program_kernel_ptr(ns, 0, occ), TPB, 0) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    per_sm = 0;
  }
  if (ns >= 2) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, program_kernel_ptr(ns, 1, occ), TPB, 0) !=
        cudaSuccess) {
      (void)cudaGetLastError();
      per_sm32 = 0;
    }
    per_sm = std::min(per_sm, per_sm32);
  }
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    (void)cudaGetLastError();
    sms = 0;
  }
  return per_sm * sms;
}

static int probe_cluster_blocks(int ns, int occ);

// Largest cluster of the program that fits an empty device, cached per
// (components, build, device).
int max_cluster_blocks(int ns, int occ) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    dev = 0;
  }
  const std::pair<int, int> key{ns * 4 + occ, dev};
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  const int c = probe_cluster_blocks(ns, occ);
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = c;
  return c;
}

static int probe_cluster_blocks(int ns, int occ) {
  const void *fn = program_kernel_ptr(ns, 0, occ);
  if (allow_large_clusters(fn) != cudaSuccess) {
    (void)cudaGetLastError();
    return 8;
  }
  for (int c = 16; c >= 1; c >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(TPB);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess) {
      (void)cudaGetLastError();   // this cluster size is not possible: try the next smaller
      continue;
    }
    if (nclusters >= 1) return c;
  }
  return 1;
}

}  // namespace xcal
