// Host-visible declarations of the persistent device program.
#pragma once
#include <cuda_runtime.h>

#include "xcal_device.cuh"

namespace xcal {
cudaError_t launch_program(int ns, int mixed, int mode, int nblocks, const KParams *hparams, int prog, int iters,
                           cudaStream_t stream);
int max_coresident_blocks(int ns, int device);
int max_cluster_blocks(int ns);
const void *program_kernel_ptr(int ns, int mixed);
}  // namespace xcal
