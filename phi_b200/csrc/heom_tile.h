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

// Schedule of the single-instance tile kernel: block-size variant (0 the
// shape's default, 1 the alternative), persistent CTAs per SM (0: as many as
// fit), with the measured apply times of the choice and of the default.
struct TileSchedule {
  int variant = 0;
  int cps = 0;
  int threads = 0;
  float ms = 0.f;
  float ms_default = 0.f;
};
int tile_block_threads(const HeomConsts &c, bool mixed, int variant);
// Times one Liouvillian apply (L's x -> out, apply mode) for every block-size
// variant and CTAs-per-SM cap and returns the fastest (about 30 launches).
cudaError_t tile_autotune(const StageLaunch &L, cudaStream_t stream, TileSchedule *out);

// ---- batched stages over many hierarchies (heom_tile_batch.cu) ----
// Tiles of one hierarchy in the given arithmetic (-1 when N has no tile kernel).
long long tile_count(const HeomConsts &c, bool mixed);
// Dynamic shared memory of one tile of stage launch L.
size_t tile_stage_smem(const StageLaunch &L);
// Size and host image of the per-instance tile parameters of stage launch L.
size_t tile_params_bytes();
void tile_params_host(const StageLaunch &L, void *out);

// One stage of many hierarchies in one persistent launch: CTAs walk the
// concatenated tile lists of all instances (work order = the order of the
// arrays); each tile runs the instantiation for its instance's (N, K+1).
struct TileBatchPlan {
  const void *params = nullptr;          // device: tile parameters per instance
  const long long *tile_start = nullptr; // device: count + 1 prefix sums of tile counts
  int count = 0;
  long long total_tiles = 0;
  size_t smem = 0;                       // max over instances
  bool mixed = false;
  int *err_flag = nullptr;               // set when a bounded wait gave up
};
// Resident CTAs per SM of the batch kernel at plan.smem.
int tile_batch_occupancy(const TileBatchPlan &plan);
cudaError_t launch_tile_batch(const TileBatchPlan &plan, int grid, cudaStream_t stream);
}  // namespace phi
