// Launch of the persistent device program (xcal_kernel.cu instantiations):
// block, cluster or cooperative grid launch, and the occupancy queries the
// launch configuration uses.
#include <algorithm>

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

const void *program_kernel_ptr(int ns, int mixed, int occ) {
  if (ns == 1) return program_kernel_d1();
  if (ns == 2) {
    if (occ) return mixed ? program_kernel_f2o() : program_kernel_d2o();
    return mixed ? program_kernel_f2() : program_kernel_d2();
  }
  if (occ) return mixed ? program_kernel_f3o() : program_kernel_d3o();
  return mixed ? program_kernel_f3() : program_kernel_d3();
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
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
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

int max_cluster_blocks(int ns) {
  const void *fn = program_kernel_ptr(ns, 0, 0);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
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
