// heom_tile_batch.cu -- one RK stage of many independent IndependentBath
// hierarchies of uneven N, K and depth in ONE persistent launch.
//
// The instances' tile lists are concatenated (tile_start[i] = first tile of
// instance i); CTAs stride over the concatenated list, find the instance of a
// tile by binary search over tile_start, and run the tile with the
// instantiation of that instance's (N, K+1) -- the same tile_body as the
// single-instance kernel, so every instance gets the same arithmetic it gets
// alone.  Small hierarchies that would fill only a few CTAs of their own
// launch share the GPU with the large ones; one launch per stage serves them
// all, and the step loop replays from a CUDA graph.
//
// Each instantiation is a separate non-inlined device function, so one
// kernel carries all (N, K+1) pairs without the compile cost of inlining them
// into one body.  The two mbarriers are initialised once per CTA and their
// phase parity is tracked across the tiles it processes.
#include <cuda_runtime.h>

#include "heom_tile_body.cuh"

namespace phi {

using namespace tile_detail;

namespace {


template <int N, int KT, bool MIXED>
__device__ __noinline__ int run_tile(const TileParams &p, long long tile, unsigned char *smem, uint32_t par0,
                                     uint32_t par1) {
  return tile_body<N, KT, MIXED>(p, tile, smem, par0, par1);
}

template <int N, bool MIXED>
__device__ __forceinline__ int run_tile_k(int K1, const TileParams &p, long long tile, unsigned char *smem,
                                          uint32_t par0, uint32_t par1) {
  switch (K1) {
    case 1: return run_tile<N, 1, MIXED>(p, tile, smem, par0, par1);
    case 2: return run_tile<N, 2, MIXED>(p, tile, smem, par0, par1);
    default: return run_tile<N, 3, MIXED>(p, tile, smem, par0, par1);
  }
}

template <bool MIXED>
__device__ __forceinline__ int run_tile_any(const TileParams &p, long long tile, unsigned char *smem,
                                            uint32_t par0, uint32_t par1) {
  const int K1 = p.c.K1;
  switch (p.c.N) {
    case 2: return run_tile_k<2, MIXED>(K1, p, tile, smem, par0, par1);
    case 3: return run_tile_k<3, MIXED>(K1, p, tile, smem, par0, par1);
    case 4: return run_tile_k<4, MIXED>(K1, p, tile, smem, par0, par1);
    case 5: return run_tile_k<5, MIXED>(K1, p, tile, smem, par0, par1);
    case 6: return run_tile_k<6, MIXED>(K1, p, tile, smem, par0, par1);
    case 7: return run_tile_k<7, MIXED>(K1, p, tile, smem, par0, par1);
    case 8: return run_tile_k<8, MIXED>(K1, p, tile, smem, par0, par1);
    case 10: return run_tile_k<10, MIXED>(K1, p, tile, smem, par0, par1);
    case 12: return run_tile_k<12, MIXED>(K1, p, tile, smem, par0, par1);
    case 16: return run_tile_k<16, MIXED>(K1, p, tile, smem, par0, par1);
    default: return run_tile_k<24, MIXED>(K1, p, tile, smem, par0, par1);
  }
}

// Resident CTAs per SM the register budget is fitted to: 4 in mixed
// precision (64 registers), 3 in FP64 (timed on the 512-instance workload:
// mixed 152 -> 145 ms per RK4 step at 4; FP64 229 ms at 3, 281 at 4; both
// slower at 2).
template <bool MIXED>
struct BatchMinBlocks {
  static constexpr int value = (MIXED ? 32 : 24) / kTileWarps;
};

template <bool MIXED>
__global__ void __launch_bounds__(kTileThreads, BatchMinBlocks<MIXED>::value)
    heom_tile_batch_kernel(const TileParams *__restrict__ params, const long long *__restrict__ tile_start,
                           int count, long long total_tiles, int *err_flag) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int inst_s;
  tile_init_barriers(smem_raw);
  uint32_t par0 = 0, par1 = 0;
  for (long long w = blockIdx.x; w < total_tiles; w += gridDim.x) {
    if (threadIdx.x == 0) {
      int lo = 0, hi = count - 1;  // last instance with tile_start <= w
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_start[mid] <= w) lo = mid;
        else hi = mid - 1;
      }
      inst_s = lo;
    }
    __syncthreads();  // inst_s visible; the previous tile's shared memory is free
    const int inst = inst_s;
    const TileParams &p = params[inst];
    const int r = run_tile_any<MIXED>(p, w - tile_start[inst], smem_raw, par0, par1);
    if (r < 0) {
      if (threadIdx.x == 0 && err_flag) atomicOr(err_flag, 1);
      return;
    }
    if (r == 0) {  // both barriers completed one phase for this tile
      par0 ^= 1u;
      par1 ^= 1u;
    }
  }
}

}  // namespace

int tile_batch_occupancy(const TileBatchPlan &plan) {
  int blocks = 0;
  const void *fn = plan.mixed ? (const void *)heom_tile_batch_kernel<true> : (const void *)heom_tile_batch_kernel<false>;
  if (plan.smem > 48 * 1024 &&
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, kTileThreads, plan.smem) != cudaSuccess) return 0;
  return blocks;
}

cudaError_t launch_tile_batch(const TileBatchPlan &plan, int grid, cudaStream_t stream) {
  if (plan.count <= 0 || plan.total_tiles <= 0) return cudaSuccess;
  if (grid <= 0) return cudaErrorInvalidValue;
  const TileParams *params = static_cast<const TileParams *>(plan.params);
  if (plan.mixed) {
    if (plan.smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(heom_tile_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)plan.smem);
      if (e != cudaSuccess) return e;
    }
    heom_tile_batch_kernel<true><<<grid, kTileThreads, plan.smem, stream>>>(params, plan.tile_start, plan.count,
                                                                 plan.total_tiles, plan.err_flag);
  } else {
    if (plan.smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(heom_tile_batch_kernel<false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem);
      if (e != cudaSuccess) return e;
    }
    heom_tile_batch_kernel<false><<<grid, kTileThreads, plan.smem, stream>>>(params, plan.tile_start, plan.count,
                                                                  plan.total_tiles, plan.err_flag);
  }
  return cudaGetLastError();
}

}  // namespace phi
