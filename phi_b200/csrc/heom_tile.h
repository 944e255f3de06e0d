// heom_tile.h -- tiled IndependentBath kernel (internal).
#pragma once

#include <cuda_runtime.h>

#include "heom_device.cuh"
#include "heom_kernels.h"

namespace phi {
// True when a compile-time-N tiled kernel exists for this problem.
bool tile_kernel_available(const HeomConsts &c);
cudaError_t launch_tile_stage(const StageLaunch &L, cudaStream_t stream);
// Node stride of complex64 buffers (N*N rounded up to even).
int mixed_node_stride(int N);
}  // namespace phi
