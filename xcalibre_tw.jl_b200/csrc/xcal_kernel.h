// Host-visible declarations of the persistent device program.
#pragma once
#include <cuda_runtime.h>

#include "xcal_device.cuh"

namespace xcal {
// occ selects the build: 0 = two resident CTAs per SM (128 registers),
// 1 = four (64 registers); the NS = 1 standalone-solve program has only the first.
cudaError_t launch_program(int ns, int mixed, int occ, int mode, int nblocks, const KParams *hparams, int prog,
                           int iters, cudaStream_t stream);
int max_coresident_blocks(int ns, int occ, int device);
int max_cluster_blocks(int ns, int occ = 0);
const void *program_kernel_ptr(int ns, int mixed, int occ);
void preload_programs();   // load every build on the current device
// the serving kernel (xcal_serve_kernel) of a dimension and precision, and the
// size of its launch on a device
const void *serve_kernel_ptr(int ns, int mixed);
int serve_grid(int ns, int mixed, int device);
}  // namespace xcal
