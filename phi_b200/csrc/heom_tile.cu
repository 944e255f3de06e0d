// heom_tile.cu -- tiled Liouvillian-apply / RK-stage kernel for one
// IndependentBath hierarchy: one launch per stage over the hierarchy's tiles;
// the tile itself is tile_body in heom_tile_body.cuh.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "heom_tile_body.cuh"

namespace phi {

using namespace tile_detail;

namespace {

// Threads per CTA of the single-instance kernel: 320 for the 24-site mixed
// kernel (a node's 300 pairs in one pass, two nodes per tile: timed on B200,
// its RKF45 step 1.65 -> 1.56 ms), 256 otherwise (320 everywhere was slower
// on the 7-site and the batched workloads).  The batched kernel always runs
// 256, so its tile counts (tile_count) use that.
template <int N, bool MIXED>
struct TileBlock {
  static constexpr int threads = (MIXED && N == 24) ? 320 : kTileThreads;
};

template <int N, int KT, bool MIXED>
__global__ void __launch_bounds__(TileBlock<N, MIXED>::threads,
                                  TileMinBlocks<KT, MIXED, TileBlock<N, MIXED>::threads>::value)
    heom_tile_kernel(TileParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  tile_init_barriers(smem_raw);
  tile_body<N, KT, MIXED, TileBlock<N, MIXED>::threads>(p, blockIdx.x, smem_raw, 0u, 0u);
}

template <int N, int KT, bool MIXED>
cudaError_t launch_tile_nk(const TileParams &p, cudaStream_t stream) {
  constexpr int BT = TileBlock<N, MIXED>::threads;
  using S = TileShape<N, MIXED, KT, BT>;
  const int max_bytes[kMaxPre] = {16, 16, 16, 16, 16};
  const size_t smem_max = tile_smem<N, KT, MIXED, BT>(p.c.T, kMaxPre, max_bytes);
  auto kern = heom_tile_kernel<N, KT, MIXED>;
  static thread_local int configured[kSmemLimitDevices] = {};
  cudaError_t e = raise_smem_limit(kern, smem_max, configured);
  if (e != cudaSuccess) return e;
  const long long tiles = (p.c.M + S::NT - 1) / S::NT;
  kern<<<(unsigned)tiles, BT, tile_smem<N, KT, MIXED, BT>(p.c.T, p.npre, p.pre_bytes), stream>>>(p);
  return cudaGetLastError();
}

template <int N, bool MIXED>
cudaError_t launch_tile_n(const TileParams &p, cudaStream_t stream) {
  switch (p.c.K1) {
    case 1: return launch_tile_nk<N, 1, MIXED>(p, stream);
    case 2: return launch_tile_nk<N, 2, MIXED>(p, stream);
    case 3: return launch_tile_nk<N, 3, MIXED>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <bool MIXED>
cudaError_t launch_tile_dispatch(const TileParams &p, cudaStream_t stream) {
  switch (p.c.N) {
    case 2: return launch_tile_n<2, MIXED>(p, stream);
    case 3: return launch_tile_n<3, MIXED>(p, stream);
    case 4: return launch_tile_n<4, MIXED>(p, stream);
    case 5: return launch_tile_n<5, MIXED>(p, stream);
    case 6: return launch_tile_n<6, MIXED>(p, stream);
    case 7: return launch_tile_n<7, MIXED>(p, stream);
    case 8: return launch_tile_n<8, MIXED>(p, stream);
    case 10: return launch_tile_n<10, MIXED>(p, stream);
    case 12: return launch_tile_n<12, MIXED>(p, stream);
    case 16: return launch_tile_n<16, MIXED>(p, stream);
    case 24: return launch_tile_n<24, MIXED>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

bool tile_kernel_available(const HeomConsts &c) {
  // IndependentBath with PHI's identity site map and K + 1 <= 3.
  if (c.kind != kIndependent || !c.identity_sites || c.K1 < 1 || c.K1 > 3 || c.nb != c.N) return false;
  // neighbour offsets are 32-bit element indices of the stage input
  if ((long long)c.M * (c.N * c.N + 1) >= (1ll << 31)) return false;
  switch (c.N) {
    case 2: case 3: case 4: case 5: case 6: case 7: case 8:
    case 10: case 12: case 16: case 24:
      return true;
    default:
      return false;
  }
}

int mixed_node_stride(int N) { return N * N + ((N * N) & 1); }

namespace tile_detail {
TileParams tile_params_for(const StageLaunch &L) {
  TileParams p;
  p.c = L.c;
  p.mode = L.mode;
  p.stage = L.stage;
  p.x = L.xv;
  p.out = L.outv;
  p.y = L.y;
  p.acc = L.acc;
  p.y32 = L.y32;
  p.a_next = L.a_next;
  p.w_acc = L.w_acc;
  p.rk4 = L.rk4;
  p.traj = L.traj;
  for (int i = 0; i < 5; ++i) p.k[i] = L.kv[i];
  p.ybuf[0] = L.ybuf[0];
  p.ybuf[1] = L.ybuf[1];
  p.y32buf[0] = L.y32buf[0];
  p.y32buf[1] = L.y32buf[1];
  p.ctl = L.ctl;
  p.act[0] = L.act[0];
  p.act[1] = L.act[1];
  p.act_par = L.act_par;
  p.dot_w = (L.mode == kModeApply && !L.mixed) ? L.dot_w : nullptr;
  p.dot_part = p.dot_w ? L.dot_part : nullptr;
  const bool mixed = L.mixed;
  const int xb = mixed ? 8 : 16;
  // Epilogue operands of this (mode, stage), in the order the epilogue reads them.
  p.npre = 0;
  for (int b = 0; b < kMaxPre; ++b) {
    p.pre[b] = nullptr;
    p.pre_bytes[b] = 16;
  }
  if (L.mode == kModeRk4) {
    if (L.stage == 0 && mixed) {
      p.pre[0] = L.y;
      p.npre = 1;
    } else if (L.stage == 1 || L.stage == 2) {
      p.pre[0] = L.y;
      p.pre[1] = L.acc;
      p.npre = 2;
    } else if (L.stage == 3) {
      p.pre[0] = L.acc;
      p.npre = 1;
    }
  } else if (L.mode == kModeRkf45) {
    if (L.stage == 0) {
      p.npre = mixed ? 1 : 0;  // y (chosen on the device)
    } else if (L.stage <= 4) {
      p.npre = 1 + L.stage;    // y, k_0 .. k_{s-1}
      for (int r = 0; r < L.stage; ++r) {
        p.pre[1 + r] = L.kv[r];
        p.pre_bytes[1 + r] = xb;
      }
    } else {
      p.npre = 5;              // y, k0, k2, k3, k4
      const int ks[4] = {0, 2, 3, 4};
      for (int r = 0; r < 4; ++r) {
        p.pre[1 + r] = L.kv[ks[r]];
        p.pre_bytes[1 + r] = xb;
      }
    }
    // 24 sites: stages 3-5 read y from global (see tile_body).
    if (L.c.N == 24 && L.stage >= 3) p.pre_bytes[0] = 0;
  }
  return p;
}
}  // namespace tile_detail

cudaError_t launch_tile_stage(const StageLaunch &L, cudaStream_t stream) {
  const TileParams p = tile_params_for(L);
  return L.mixed ? launch_tile_dispatch<true>(p, stream) : launch_tile_dispatch<false>(p, stream);
}

namespace {
template <int N, int KT>
long long tiles_of_k(long long M, bool mixed) {
  const long long nt = mixed ? TileShape<N, true, KT>::NT : TileShape<N, false, KT>::NT;
  return (M + nt - 1) / nt;
}
template <int N>
long long tiles_of(long long M, bool mixed, int K1) {
  switch (K1) {
    case 1: return tiles_of_k<N, 1>(M, mixed);
    case 2: return tiles_of_k<N, 2>(M, mixed);
    case 3: return tiles_of_k<N, 3>(M, mixed);
    default: return -1;
  }
}
template <int N>
size_t stage_smem_n(const TileParams &p, bool mixed) {
  switch (p.c.K1) {
    case 1: return mixed ? tile_smem<N, 1, true>(p.c.T, p.npre, p.pre_bytes) : tile_smem<N, 1, false>(p.c.T, p.npre, p.pre_bytes);
    case 2: return mixed ? tile_smem<N, 2, true>(p.c.T, p.npre, p.pre_bytes) : tile_smem<N, 2, false>(p.c.T, p.npre, p.pre_bytes);
    case 3: return mixed ? tile_smem<N, 3, true>(p.c.T, p.npre, p.pre_bytes) : tile_smem<N, 3, false>(p.c.T, p.npre, p.pre_bytes);
    default: return 0;
  }
}
}  // namespace

long long tile_count(const HeomConsts &c, bool mixed) {
  switch (c.N) {
    case 2: return tiles_of<2>(c.M, mixed, c.K1);
    case 3: return tiles_of<3>(c.M, mixed, c.K1);
    case 4: return tiles_of<4>(c.M, mixed, c.K1);
    case 5: return tiles_of<5>(c.M, mixed, c.K1);
    case 6: return tiles_of<6>(c.M, mixed, c.K1);
    case 7: return tiles_of<7>(c.M, mixed, c.K1);
    case 8: return tiles_of<8>(c.M, mixed, c.K1);
    case 10: return tiles_of<10>(c.M, mixed, c.K1);
    case 12: return tiles_of<12>(c.M, mixed, c.K1);
    case 16: return tiles_of<16>(c.M, mixed, c.K1);
    case 24: return tiles_of<24>(c.M, mixed, c.K1);
    default: return -1;
  }
}

size_t tile_stage_smem(const StageLaunch &L) {
  const TileParams p = tile_params_for(L);
  switch (L.c.N) {
    case 2: return stage_smem_n<2>(p, L.mixed);
    case 3: return stage_smem_n<3>(p, L.mixed);
    case 4: return stage_smem_n<4>(p, L.mixed);
    case 5: return stage_smem_n<5>(p, L.mixed);
    case 6: return stage_smem_n<6>(p, L.mixed);
    case 7: return stage_smem_n<7>(p, L.mixed);
    case 8: return stage_smem_n<8>(p, L.mixed);
    case 10: return stage_smem_n<10>(p, L.mixed);
    case 12: return stage_smem_n<12>(p, L.mixed);
    case 16: return stage_smem_n<16>(p, L.mixed);
    case 24: return stage_smem_n<24>(p, L.mixed);
    default: return 0;
  }
}

size_t tile_params_bytes() { return sizeof(TileParams); }

void tile_params_host(const StageLaunch &L, void *out) {
  const TileParams p = tile_params_for(L);
  std::memcpy(out, &p, sizeof(p));
}


}  // namespace phi
