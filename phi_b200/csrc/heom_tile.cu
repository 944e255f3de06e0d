// heom_tile.cu -- tiled Liouvillian-apply / RK-stage kernel for one
// IndependentBath hierarchy: one persistent launch per stage whose CTAs walk
// the hierarchy's tiles; the pair loop and the epilogue of a tile are
// tile_pairs / tile_epilogue of heom_tile_body.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "heom_tile_body.cuh"
#include "heom_umma.cuh"

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
  // The autotuner's alternative block size (heom_tile.cu, tile_autotune).
  static constexpr int alt = threads == kTileThreads ? 320 : kTileThreads;
};

// ---- persistent pipelined kernel ----
//
// A CTA stays resident and walks the tiles blockIdx.x, blockIdx.x +
// gridDim.x, ...  While tile i computes, the stage input X and the neighbour
// records (next / prev ids and occupations, contiguous per tile) of tile i+1
// arrive in the other of two shared-memory slots by cp.async.bulk; the
// epilogue operands of tile i (y, accumulator, k_r) are issued when tile i
// starts and land while its pair loop runs.  H, the Matsubara factors, the
// pair list, c_t, the dephasing rates and the prefactor tables are staged
// once per CTA.  Three mbarriers: one per slot (phase parity (i >> 1) & 1 for
// the CTA's i-th tile) and one for the epilogue operands (parity i & 1).
// Tensor-core products (heom_umma.cuh) in the 24-site mixed kernel: with a
// real H the tile's A = H X is one TF32 GEMM per tile, rows (node, column j
// of X, re / im) x K = the row index i of X, against B = H (rows padded to
// kTcRowsB), split into hi and lo parts; the CUDA cores then only combine
// A_ij and A_ji per pair.  M = 128 rows (the tile's 2 x 24 x 2 = 96 rows and
// 32 rows that alias the operand after them and whose results are unused).
template <int N, bool MIXED>
struct TileTc {
  static constexpr bool on = MIXED && N == 24;
  static constexpr int kM = 128, kRowsB = 32;
};

template <int N, int KT, bool MIXED, int BT>
struct PipeLayout {
  using S = TileShape<N, MIXED, KT, BT>;
  static constexpr int T = N * KT;
  static constexpr int ES = MIXED ? S::EP : S::E;
  static constexpr int XB = MIXED ? 8 : 16;
  static constexpr int RB = MIXED ? 4 : 8;  // bytes of the arithmetic type
  static constexpr size_t r16(size_t b) { return (b + 15) / 16 * 16; }
  static constexpr size_t r128(size_t b) { return (b + 127) / 128 * 128; }
  // One slot: the tile's X, then its next ids, prev ids (int32),
  // occupations (uint8) and dephasing rates (double), each copied from the
  // 16-byte aligned window around the tile's records (up to 3 ids, 15
  // bytes or 1 rate of slack on either side).
  static constexpr size_t kSlotX = r128((size_t)S::NT * ES * XB);
  static constexpr size_t kSlotIds = r16(((size_t)S::NT * T + 8) * 4);
  static constexpr size_t kSlotMi = r16((size_t)S::NT * T + 32);
  static constexpr size_t kSlotDeph = r16(((size_t)S::NT + 2) * 8);  // per-node dephasing rates
  static constexpr size_t kSlot = r128(kSlotX + 2 * kSlotIds + kSlotMi + kSlotDeph);
  static constexpr size_t kSlots = 128;                       // after the 4 mbarriers and the TMEM slot
  // Tensor-core operands: A hi, A lo (the tile's rows), B hi, B lo (kRowsB
  // rows); rows past a region's end read the next region.
  static constexpr bool kTcOn = TileTc<N, MIXED>::on;
  static constexpr size_t kTcRowsA = (size_t)S::NT * 2 * N;
  static constexpr size_t kTcA = kTcOn ? kTcRowsA / 8 * (size_t)umma::kSbo<N> : 0;
  static constexpr size_t kTcB = kTcOn ? (size_t)TileTc<N, MIXED>::kRowsB / 8 * (size_t)umma::kSbo<N> : 0;
  static constexpr size_t kTc = kSlots + 2 * kSlot;
  static constexpr size_t kUs = kTc + r128(2 * kTcA + 2 * kTcB);  // derivative tile
  static constexpr size_t kPre = kUs + r128((size_t)S::NT * S::EU * XB);
};

template <int N, int KT, bool MIXED, int BT>
size_t pipe_smem(int T, int L, int npre, const int *pre_bytes) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = PipeLayout<N, KT, MIXED, BT>;
  size_t b = Lay::kPre;
  for (int i = 0; i < npre; ++i)
    b += ((size_t)S::NT * (pre_bytes[i] == 16 ? S::E : Lay::ES) * pre_bytes[i] + 127) / 128 * 128;
  const int W = L + 2;
  b += (size_t)S::E * Lay::XB;                                        // H
  b += (size_t)(36 + BT / 32) * sizeof(double);                       // coef (FP64, FP32), warp maxima
  b += (size_t)(2 * S::NT * T + 2 * T + S::E + 2 * T * W) * Lay::RB;  // cn, cp, c_t, mats, prefactor tables
  b += (size_t)(S::NT * 3 * T) * sizeof(int);                         // ids, occupations
  b += 2 * S::P + 16;
  return b;
}

template <int N, int KT, bool MIXED, int BT>
__global__ void __launch_bounds__(BT, TileMinBlocks<KT, MIXED, BT>::value) heom_tile_pipe_kernel(TileParams p) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = PipeLayout<N, KT, MIXED, BT>;
  using TX = typename TileArith<MIXED>::TX;
  using R = typename TileArith<MIXED>::R;
  constexpr int E = S::E, P = S::P, NT = S::NT, ES = Lay::ES, T = N * KT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const HeomConsts &c = p.c;
  const int tid = threadIdx.x;
  if (p.mode == kModeRkf45 && *(volatile int *)&p.ctl->done) return;  // uniform across the grid

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  TX *Us = reinterpret_cast<TX *>(smem_raw + Lay::kUs);
  unsigned char *PreBase = smem_raw + Lay::kPre;
  uint32_t pre_off[kMaxPre];
  size_t tail = Lay::kPre;
  {
    uint32_t acc_off = 0;
#pragma unroll
    for (int b = 0; b < kMaxPre; ++b) {
      pre_off[b] = acc_off;
      if (b < p.npre) acc_off += ((uint32_t)NT * (p.pre_bytes[b] == 16 ? E : ES) * p.pre_bytes[b] + 127) / 128 * 128;
    }
    tail += acc_off;
  }
  const int W = c.L + 2;
  TX *Hs = reinterpret_cast<TX *>(smem_raw + tail);                           // E
  double *coef = reinterpret_cast<double *>(Hs + E);                          // 24, then 24 floats
  unsigned long long *wmax = reinterpret_cast<unsigned long long *>(coef + 36);  // BT / 32
  R *cn = reinterpret_cast<R *>(wmax + BT / 32);                              // NT*T
  R *cp = cn + NT * T;                                                        // NT*T
  R *ccr = cp + NT * T;                                                       // 2T
  R *mats = ccr + 2 * T;                                                      // E
  R *sqn = mats + E;                                                          // T*W
  R *sqp = sqn + T * W;                                                       // T*W
  int *ids = reinterpret_cast<int *>(sqp + T * W);                            // NT*2T
  int *nts = ids + NT * 2 * T;                                                // NT*T
  unsigned char *pi = reinterpret_cast<unsigned char *>(nts + NT * T);
  unsigned char *pj = pi + P;

  constexpr bool TC = Lay::kTcOn;
  static_assert(!TC || Lay::kTcRowsA <= TileTc<N, MIXED>::kM, "tile rows fit one MMA");
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 4);
  unsigned char *TcAhi = smem_raw + Lay::kTc, *TcAlo = TcAhi + Lay::kTcA;
  unsigned char *TcBhi = TcAlo + Lay::kTcA, *TcBlo = TcBhi + Lay::kTcB;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
    mbar_init(&bars[3], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // The tensor-core path needs a real H (every in-scope 24-site workload).
  const bool tc = TC && c.h_real;
  if (tc) {
    if (tid < 32) umma::tmem_alloc(tmem_slot, 32);
    // B = H, row r = (H_r0 .. H_r,N-1), rows N .. kRowsB-1 zero, hi / lo.
    for (int q = tid; q < TileTc<N, MIXED>::kRowsB * N; q += BT) {
      const int r = q / N, k = q - r * N;
      const float v = r < N ? (float)__ldg(c.H + r + k * N).x : 0.0f;
      const float h = umma::tf32_hi(v);
      *reinterpret_cast<float *>(TcBhi + umma::core_offset<N>(r, k)) = h;
      *reinterpret_cast<float *>(TcBlo + umma::core_offset<N>(r, k)) = v - h;
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
  }
  int ycur = 0;
  if (p.mode == kModeRkf45) {
    ycur = p.ctl->ycur;
    if (tid < 24) {
      const double v = p.ctl->coef[tid];
      coef[tid] = v;
      reinterpret_cast<float *>(coef + 24)[tid] = (float)v;
    }
  }
  const bool hreal = c.h_real;
  R *Hr = reinterpret_cast<R *>(Hs);
  if (hreal) {
    for (int i = tid; i < E; i += BT) Hr[i] = (R)__ldg(c.H + i).x;
  } else {
    for (int i = tid; i < E; i += BT) Hs[i] = from_d2<TX>(__ldg(c.H + i));
  }
  for (int i = tid; i < E; i += BT) mats[i] = (R)__ldg(c.mats_elem + i);
  for (int i = tid; i < P; i += BT) {
    pi[i] = __ldg(c.pair_i + i);
    pj[i] = __ldg(c.pair_j + i);
  }
  for (int t = tid; t < T; t += BT) {
    const double2 ct = __ldg(c.corr + t);
    ccr[2 * t] = (R)ct.x;
    ccr[2 * t + 1] = (R)ct.y;
  }
  for (int q = tid; q < T * W; q += BT) {
    sqn[q] = (R)__ldg(c.sq_next + q);
    sqp[q] = (R)__ldg(c.sq_prev + q);
  }
  __syncthreads();  // barriers initialised, constants visible
  uint32_t tmem = 0;
  if (tc) {
    umma::fence_after_sync();
    tmem = *tmem_slot;
  }

  const long long ntiles = (c.M + NT - 1) / NT;
  const TX *xin;
  if (p.mode == kModeRkf45 && p.stage == 0)
    xin = MIXED ? static_cast<const TX *>(p.y32buf[ycur]) : reinterpret_cast<const TX *>(p.ybuf[ycur]);
  else
    xin = static_cast<const TX *>(p.x);
  // Filtering: an inactive neighbour contributes nothing (the DoNext /
  // DoPrevious overrides of IndependentBathAdaptiveTruncation,
  // hierarchy_updater.cc:256-303).
  const uint8_t *act_in = c.filtered ? p.act[p.mode == kModeRkf45 ? ycur : p.act_par] : nullptr;
  const long long polls0 = c.first_wait_polls == 0 ? kMaxPolls : (c.first_wait_polls < 0 ? 0 : c.first_wait_polls);

  // Thread 0: the X and neighbour records of `tile` into slot s.
  auto issue_slot = [&](long long tile, int s) {
    const long long n0 = tile * NT;
    const int nt = (int)((c.M - n0) < NT ? (c.M - n0) : NT);
    unsigned char *b = smem_raw + Lay::kSlots + (size_t)s * Lay::kSlot;
    const long long q0 = n0 * T, q1 = q0 + (long long)nt * T;
    const long long a4 = q0 & ~3ll, e4 = (q1 + 3) & ~3ll, a16 = q0 & ~15ll, e16 = (q1 + 15) & ~15ll;
    const long long a2 = n0 & ~1ll, e2 = (n0 + nt + 1) & ~1ll;
    const uint32_t xbytes = (uint32_t)(nt * ES * Lay::XB), idbytes = (uint32_t)((e4 - a4) * 4),
                   mibytes = (uint32_t)(e16 - a16), dbytes = (uint32_t)((e2 - a2) * 8);
    mbar_expect_tx(&bars[s], xbytes + 2 * idbytes + mibytes + dbytes);
    bulk_g2s(b, xin + n0 * ES, xbytes, &bars[s]);
    bulk_g2s(b + Lay::kSlotX, c.next + a4, idbytes, &bars[s]);
    bulk_g2s(b + Lay::kSlotX + Lay::kSlotIds, c.prev + a4, idbytes, &bars[s]);
    bulk_g2s(b + Lay::kSlotX + 2 * Lay::kSlotIds, c.mi + a16, mibytes, &bars[s]);
    bulk_g2s(b + Lay::kSlotX + 2 * Lay::kSlotIds + Lay::kSlotMi, c.deph_node + a2, dbytes, &bars[s]);
  };
  // Thread 0: the epilogue operands of `tile`.
  auto issue_pre = [&](long long tile) {
    const long long n0 = tile * NT;
    const int nt = (int)((c.M - n0) < NT ? (c.M - n0) : NT);
    uint32_t pbytes = 0;
#pragma unroll
    for (int b = 0; b < kMaxPre; ++b)
      if (b < p.npre) pbytes += (uint32_t)(nt * (p.pre_bytes[b] == 16 ? E : ES) * p.pre_bytes[b]);
    mbar_expect_tx(&bars[2], pbytes);
#pragma unroll
    for (int b = 0; b < kMaxPre; ++b) {
      if (b >= p.npre) break;
      if (p.pre_bytes[b] == 0) {
        // Read from global memory in the epilogue (the RKF45 state y): an
        // L2 prefetch of the tile's contiguous range now, so the epilogue's
        // loads do not wait for DRAM.
        if (b == 0 && p.mode == kModeRkf45)
          bulk_prefetch_l2(p.ybuf[ycur] + (size_t)n0 * E, (uint32_t)((size_t)nt * E * sizeof(double2)));
        continue;
      }
      const unsigned char *src = static_cast<const unsigned char *>(p.pre[b]);
      if (b == 0 && p.mode == kModeRkf45)
        src = static_cast<const unsigned char *>(p.pre_bytes[0] == 8 ? p.y32buf[ycur] : (const void *)p.ybuf[ycur]);
      const int stride = p.pre_bytes[b] == 16 ? E : ES;
      bulk_g2s(PreBase + pre_off[b], src + (size_t)n0 * stride * p.pre_bytes[b],
               (uint32_t)(nt * stride * p.pre_bytes[b]), &bars[2]);
    }
  };

  long long tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue_slot(tile, 0);
  double emax = 0.0;
  int i = 0;
  bool failed = false, next_issued = false, mma_inflight = false;
  for (; tile < ntiles; ++i, tile += gridDim.x) {
    const int s = i & 1;
    const long long n0 = tile * NT;
    const int nt_here = (int)((c.M - n0) < NT ? (c.M - n0) : NT);
    next_issued = tile + gridDim.x < ntiles;
    if (tid == 0) {
      if (next_issued) issue_slot(tile + gridDim.x, s ^ 1);
      if (p.npre > 0) issue_pre(tile);
    }
    if (!__syncthreads_and(mbar_wait_bounded(&bars[s], (uint32_t)(i >> 1) & 1u, polls0))) {
      failed = true;
      break;
    }
    // Per (node, term): neighbour element offsets (-1 when absent or
    // inactive), occupation and the prefactor magnitudes for it.
    const unsigned char *sb = smem_raw + Lay::kSlots + (size_t)s * Lay::kSlot;
    const TX *Xs = reinterpret_cast<const TX *>(sb);
    const int q0 = (int)((n0 * T) & 15);
    const int *nx_s = reinterpret_cast<const int *>(sb + Lay::kSlotX) + (q0 & 3);
    const int *pv_s = reinterpret_cast<const int *>(sb + Lay::kSlotX + Lay::kSlotIds) + (q0 & 3);
    const uint8_t *mi_s = sb + Lay::kSlotX + 2 * Lay::kSlotIds + q0;
    const double *deph =
        reinterpret_cast<const double *>(sb + Lay::kSlotX + 2 * Lay::kSlotIds + Lay::kSlotMi) + (n0 & 1);
    if (TC && tc) {
      // Tensor-core operand A: row (node, j, re / im) = nd * 2N + 2j + c,
      // K = i, element X_ij's component c, split into hi and lo.
      for (int e = tid; e < nt_here * 2 * E; e += BT) {
        const int row = e / N, ii = e - row * N;
        const int nd = row / (2 * N), rem = row - nd * 2 * N, j = rem >> 1;
        const TX x = Xs[nd * ES + ii + j * N];
        const float v = (rem & 1) ? (float)x.y : (float)x.x;
        const float h = umma::tf32_hi(v);
        *reinterpret_cast<float *>(TcAhi + umma::core_offset<N>(row, ii)) = h;
        *reinterpret_cast<float *>(TcAlo + umma::core_offset<N>(row, ii)) = v - h;
      }
      umma::fence_async_smem();
      __syncthreads();
      // D = A_hi B_hi^T + A_lo B_hi^T + A_hi B_lo^T in TMEM (lane = row,
      // column = r); it runs while the threads prepare the neighbour records.
      if (tid == 0) {
        umma::fence_after_sync();
        constexpr uint32_t idesc = umma::instr_desc_tf32(TileTc<N, MIXED>::kM, TileTc<N, MIXED>::kRowsB);
        int n = 0;
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
          const unsigned char *a = pass == 1 ? TcAlo : TcAhi, *b = pass == 2 ? TcBlo : TcBhi;
#pragma unroll
          for (int ks = 0; ks < N / 8; ++ks, ++n)
            umma::mma_tf32(tmem, umma::smem_desc<N>(a + ks * 2 * umma::kLbo), umma::smem_desc<N>(b + ks * 2 * umma::kLbo),
                           idesc, n > 0);
        }
        umma::commit(&bars[3]);
      }
      mma_inflight = true;
    }
    for (int q = tid; q < nt_here * T; q += BT) {
      const int nd = q / T, t = q - nd * T;
      const int nx = nx_s[q], pv = pv_s[q], nt = mi_s[q];
      const bool nx_on = nx >= 0 && (!act_in || __ldg(act_in + nx));
      const bool pv_on = pv >= 0 && (!act_in || __ldg(act_in + pv));
      ids[nd * 2 * T + t] = nx_on ? nx * ES : -1;
      ids[nd * 2 * T + T + t] = pv_on ? pv * ES : -1;
      nts[q] = nt;
      cn[q] = sqn[t * W + nt];
      cp[q] = sqp[t * W + nt];
    }
    __syncthreads();
    if (TC && tc) {
      // Each row's A = H X values from TMEM into the derivative tile.
      if (!__syncthreads_and(mbar_wait_bounded(&bars[3], (uint32_t)i & 1u))) {
        failed = true;
        break;
      }
      mma_inflight = false;
      umma::fence_after_sync();
      const int warp = tid >> 5;
      if (warp < (int)(Lay::kTcRowsA + 31) / 32) {
        const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16);
        uint32_t v16[16], v8[8];
        umma::ld_x16(base, v16);
        umma::ld_x8(base + 16, v8);
        umma::wait_ld();
        const int row = warp * 32 + (tid & 31);
        if (row < nt_here * 2 * N) {
          const int nd = row / (2 * N), rem = row - nd * 2 * N, j = rem >> 1, cc = rem & 1;
          float *u = reinterpret_cast<float *>(Us + nd * S::EU + j * S::NP) + cc;
#pragma unroll
          for (int r = 0; r < 16; ++r) u[2 * r] = __uint_as_float(v16[r]);
#pragma unroll
          for (int r = 0; r < 8; ++r) u[2 * (16 + r)] = __uint_as_float(v8[r]);
        }
      }
      umma::fence_before_sync();
      __syncthreads();
      tile_pairs<N, KT, MIXED, BT, true>(c, Xs, Us, Hs, mats, pi, pj, ids, cn, cp, ccr, deph, nts, xin, nt_here);
    } else {
      tile_pairs<N, KT, MIXED, BT>(c, Xs, Us, Hs, mats, pi, pj, ids, cn, cp, ccr, deph, nts, xin, nt_here);
    }
    if (!__syncthreads_and(p.npre == 0 || mbar_wait_bounded(&bars[2], (uint32_t)i & 1u))) {
      failed = true;
      break;
    }
    tile_epilogue<N, KT, MIXED, BT>(p, Xs, Us, PreBase, pre_off, coef, wmax, tile, n0, nt_here, ycur, emax);
    tile_flags<N, KT, MIXED, BT>(p, Us, n0, nt_here, ycur);
    __syncthreads();  // slot s, the operands, Us and the per-tile arrays are reused
  }
  if (failed) {
    // Record the failure and drain this CTA's copies in flight with the
    // built-in limit, so none is still writing into shared memory at exit.
    if (tid == 0) atomicOr(c.err_flag, 1);
    const int s = i & 1;
    mbar_wait_bounded(&bars[s], (uint32_t)(i >> 1) & 1u);
    if (next_issued) mbar_wait_bounded(&bars[s ^ 1], (uint32_t)((i + 1) >> 1) & 1u);
    if (p.npre > 0) mbar_wait_bounded(&bars[2], (uint32_t)i & 1u);
    if (TC && tc) {
      if (mma_inflight) mbar_wait_bounded(&bars[3], (uint32_t)i & 1u);
      umma::fence_before_sync();
      __syncthreads();
      if (tid < 32) umma::tmem_dealloc(tmem, 32);
    }
    return;
  }
  if (p.mode == kModeRkf45 && p.stage == 5) tile_error_max<MIXED, BT>(p, emax, wmax);
  if (TC && tc) {
    umma::fence_before_sync();
    __syncthreads();
    if (tid < 32) umma::tmem_dealloc(tmem, 32);
  }
}

// Resident CTAs per SM of a kernel at a dynamic shared-memory size and the
// SM count of the current device, cached per (kernel, size, device).
struct OccEntry {
  const void *fn;
  size_t smem;
  int dev;
  int grid;
};

int persistent_grid(const void *fn, int threads, size_t smem) {
  static thread_local OccEntry cache[64];
  static thread_local int used = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  for (int k = 0; k < used; ++k)
    if (cache[k].fn == fn && cache[k].smem == smem && cache[k].dev == dev) return cache[k].grid;
  int sms = 0, blocks = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, smem) != cudaSuccess) return 0;
  const int grid = sms * (blocks > 0 ? blocks : 1);
  if (used < 64) cache[used++] = OccEntry{fn, smem, dev, grid};
  return grid;
}

// The same for a kernel that allocates tensor memory, whose occupancy the
// runtime's calculator reports as one CTA per SM: resident CTAs from the
// SM's shared memory (with the per-CTA reservation), its thread slots, and
// the register budget the kernel was compiled for (at least min_blocks).
// Measured on B200 with the 24-site kernel: two such CTAs per SM run
// together (RKF45 step 2.31 ms with one per SM, 1.36 ms with two).
int persistent_grid_tmem(int threads, size_t smem, int min_blocks) {
  static thread_local int cached_dev = -1, sms = 0, smem_sm = 0, reserved = 0, threads_sm = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (dev != cached_dev) {
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
      return 0;
    cached_dev = dev;
  }
  int blocks = (int)((size_t)smem_sm / (smem + (size_t)reserved));
  blocks = std::min(blocks, threads_sm / threads);
  blocks = std::min(blocks, std::max(min_blocks, 1));
  return sms * std::max(blocks, 1);
}

// Launch of one block-size variant.  The grid is the resident-CTA count of
// this launch's shared-memory size (capped at tile_cps CTAs per SM when the
// schedule sets it) and never more than the tiles.  *per_sm (optional)
// receives the resident CTAs per SM before the cap.
template <int N, int KT, bool MIXED, int BT>
cudaError_t launch_tile_bt(const TileParams &p, cudaStream_t stream, int *per_sm = nullptr) {
  using S = TileShape<N, MIXED, KT, BT>;
  const long long tiles = (p.c.M + S::NT - 1) / S::NT;
  const int max_bytes[kMaxPre] = {16, 16, 16, 16, 16};
  const size_t smem_max = pipe_smem<N, KT, MIXED, BT>(p.c.T, p.c.L, kMaxPre, max_bytes);
  auto kern = heom_tile_pipe_kernel<N, KT, MIXED, BT>;
  static thread_local int configured[kSmemLimitDevices] = {};
  cudaError_t e = raise_smem_limit(kern, smem_max, configured);
  if (e != cudaSuccess) return e;
  const size_t smem = pipe_smem<N, KT, MIXED, BT>(p.c.T, p.c.L, p.npre, p.pre_bytes);
  int cap = TileTc<N, MIXED>::on ? persistent_grid_tmem(BT, smem, TileMinBlocks<KT, MIXED, BT>::value)
                                 : persistent_grid((const void *)kern, BT, smem);
  if (cap <= 0) return cudaErrorInvalidConfiguration;
  int sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return cudaErrorInvalidDevice;
  if (per_sm) *per_sm = cap / sms;
  if (p.c.tile_cps > 0 && p.c.tile_cps * sms < cap) cap = p.c.tile_cps * sms;
  const long long grid = tiles < cap ? tiles : cap;
  kern<<<(unsigned)grid, BT, smem, stream>>>(p);
  return cudaGetLastError();
}

template <int N, int KT, bool MIXED>
cudaError_t launch_tile_nk(const TileParams &p, cudaStream_t stream, int *per_sm = nullptr) {
  // The steady-state apply writes one partial inner product per tile into
  // an array sized by tile_count, i.e. by the default block's tiles.
  if (p.c.tile_variant == 1 && !p.dot_w)
    return launch_tile_bt<N, KT, MIXED, TileBlock<N, MIXED>::alt>(p, stream, per_sm);
  return launch_tile_bt<N, KT, MIXED, TileBlock<N, MIXED>::threads>(p, stream, per_sm);
}

template <int N, bool MIXED>
cudaError_t launch_tile_n(const TileParams &p, cudaStream_t stream, int *per_sm) {
  switch (p.c.K1) {
    case 1: return launch_tile_nk<N, 1, MIXED>(p, stream, per_sm);
    case 2: return launch_tile_nk<N, 2, MIXED>(p, stream, per_sm);
    case 3: return launch_tile_nk<N, 3, MIXED>(p, stream, per_sm);
    default: return cudaErrorInvalidValue;
  }
}

template <bool MIXED>
cudaError_t launch_tile_dispatch(const TileParams &p, cudaStream_t stream, int *per_sm = nullptr) {
  switch (p.c.N) {
    case 2: return launch_tile_n<2, MIXED>(p, stream, per_sm);
    case 3: return launch_tile_n<3, MIXED>(p, stream, per_sm);
    case 4: return launch_tile_n<4, MIXED>(p, stream, per_sm);
    case 5: return launch_tile_n<5, MIXED>(p, stream, per_sm);
    case 6: return launch_tile_n<6, MIXED>(p, stream, per_sm);
    case 7: return launch_tile_n<7, MIXED>(p, stream, per_sm);
    case 8: return launch_tile_n<8, MIXED>(p, stream, per_sm);
    case 10: return launch_tile_n<10, MIXED>(p, stream, per_sm);
    case 12: return launch_tile_n<12, MIXED>(p, stream, per_sm);
    case 16: return launch_tile_n<16, MIXED>(p, stream, per_sm);
    case 24: return launch_tile_n<24, MIXED>(p, stream, per_sm);
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
      // mixed: the complex64 copy y32 feeds the complex64 stage input
      p.pre[0] = mixed ? (const void *)L.y32 : (const void *)L.y;
      p.pre_bytes[0] = mixed ? 8 : 16;
      p.pre[1] = L.acc;
      p.npre = 2;
    } else if (L.stage == 3) {
      p.pre[0] = L.acc;
      p.npre = 1;
    }
  } else if (L.mode == kModeRkf45) {
    if (L.stage == 0) {
      p.npre = 0;              // y (or y32) is the stage input itself
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
    // Slot 0 (y, chosen on the device): complex64 y32 for the mixed stage
    // inputs of stages 1-4; read from global memory in mixed stage 5 and in
    // the 24-site FP64 stages 3-5 (see tile_epilogue).
    if (mixed && L.stage >= 1 && L.stage <= 4) p.pre_bytes[0] = 8;
    if ((mixed && L.stage == 5) || (!mixed && L.c.N == 24 && L.stage >= 3)) p.pre_bytes[0] = 0;
  }
  return p;
}
}  // namespace tile_detail

cudaError_t launch_tile_stage(const StageLaunch &L, cudaStream_t stream) {
  const TileParams p = tile_params_for(L);
  return L.mixed ? launch_tile_dispatch<true>(p, stream) : launch_tile_dispatch<false>(p, stream);
}

namespace {
template <bool MIXED>
int block_threads_n(int N, int variant) {
  switch (N) {
#define PHI_TB(n) \
  case n: return variant == 1 ? TileBlock<n, MIXED>::alt : TileBlock<n, MIXED>::threads;
    PHI_TB(2) PHI_TB(3) PHI_TB(4) PHI_TB(5) PHI_TB(6) PHI_TB(7) PHI_TB(8) PHI_TB(10) PHI_TB(12) PHI_TB(16) PHI_TB(24)
#undef PHI_TB
    default: return 0;
  }
}
}  // namespace

int tile_block_threads(const HeomConsts &c, bool mixed, int variant) {
  return mixed ? block_threads_n<true>(c.N, variant) : block_threads_n<false>(c.N, variant);
}

cudaError_t tile_autotune(const StageLaunch &L0, cudaStream_t stream, TileSchedule *out) {
  StageLaunch L = L0;
  L.mode = kModeApply;
  L.dot_w = nullptr;
  L.dot_part = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  TileSchedule best{};
  best.ms = 1e30f;
  float ms_default = 0.f;
  constexpr int kReps = 3;
  for (int variant = 0; variant < 2 && e == cudaSuccess; ++variant) {
    L.c.tile_variant = variant;
    L.c.tile_cps = 0;
    int per_sm = 0;
    TileParams p = tile_params_for(L);
    // warm-up launch (module load, smem attribute) and the occupancy
    e = L.mixed ? launch_tile_dispatch<true>(p, stream, &per_sm) : launch_tile_dispatch<false>(p, stream, &per_sm);
    for (int cps = per_sm; cps >= 1 && e == cudaSuccess; --cps) {
      p.c.tile_cps = cps == per_sm ? 0 : cps;
      e = cudaEventRecord(e0, stream);
      for (int r = 0; r < kReps && e == cudaSuccess; ++r)
        e = L.mixed ? launch_tile_dispatch<true>(p, stream) : launch_tile_dispatch<false>(p, stream);
      if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) break;
      ms /= kReps;
      if (variant == 0 && cps == per_sm) ms_default = ms;
      if (ms < best.ms) {
        best.ms = ms;
        best.variant = variant;
        best.cps = p.c.tile_cps;
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e != cudaSuccess) return e;
  best.ms_default = ms_default;
  best.threads = tile_block_threads(L.c, L.mixed, best.variant);
  *out = best;
  return cudaSuccess;
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
