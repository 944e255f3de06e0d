// heom_tile_body.cuh -- the tiled IndependentBath stage (one tile of one
// hierarchy) shared by the single-instance kernel (heom_tile.cu) and the
// batched persistent kernel (heom_tile_batch.cu).  Internal header.
//
// The stage serves the IndependentBath model (PHI's default;
// hierarchy_updater.cc:129-144, :216-254) with a compile-time system size N,
// in two arithmetics:
//
//   FP64   every buffer complex128 (the path PHI computes).
//   MIXED  stage inputs X_s and stage derivatives k_s stored as complex64 and
//          the Liouvillian evaluated in FP32; the state y, the RK4
//          accumulator, every stage combine (X_{s+1} = y + sum b k), the
//          fourth/fifth-order solutions, the RKF45 error norm and the step
//          control stay FP64.  A complex64 copy of y (y32) is the stage-0
//          input.  complex64 buffers pad every node to an even number of
//          elements so each node range is 16-byte aligned.
//
// A CTA of BT threads (kTileThreads = 256, or what the single-instance
// launch picks per (N, arithmetic)) owns a tile of NT consecutive nodes (one
// or two upper-triangle pairs of one node per thread).  Everything the tile reads of
// its own nodes is contiguous in HBM and arrives by TMA bulk copies issued at
// CTA start:
//
//   t = 0   one thread issues cp.async.bulk copies of the tile's stage input
//           X_s (barrier 0) and of every epilogue operand -- state y, RK4
//           accumulator, RKF45 k_r -- (barrier 1) into shared memory; all
//           threads load the tile's next/prev ids and occupations.
//   phase 2 (after barrier 0) work item = (node, upper-triangle pair i <= j):
//           A_ij, A_ji from shared memory (A = H X, [H, X] = A - A^+),
//           dephasing + Matsubara factor, and the neighbour terms: for each
//           term on site j (column part) or site i (row part), the one
//           element of the linked ADO this pair needs, loaded from L2 with
//           independent predicated loads (a Hermitian ADO's row m is the
//           conjugate of its column m).  dX_ij and dX_ji = conj(dX_ij) go to
//           shared memory.
//   phase 3 (after barrier 1) epilogue per tile element: plain store, RK4 or
//           RKF45 stage combine, RKF45 error max; operands from shared memory.
//
// Stores of the next stage input use the default cache policy (its neighbour
// gathers in the next stage should hit L2); k and accumulator stores stream.
// This kernel serves PHI's identity site map (bath m on |m><m|, terms of site
// m are m*(K+1) .. m*(K+1)+K) with K+1 <= 3; other maps use the generic
// kernel of heom_kernels.cu (FP64 only).
//
// Every mbarrier wait is bounded: after kMaxPolls polls the kernel records the
// failure in HeomConsts::err_flag, waits (bounded again) for its own copies,
// and returns; the host reports PHI_E_TIMEOUT.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "heom_device.cuh"
#include "heom_kernels.h"
#include "heom_tile.h"
#include "heom_tl_term.cuh"

namespace phi {
namespace tile_detail {

constexpr int kTileThreads = 256;             // threads per CTA
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kMaxPre = 5;  // epilogue operand buffers per launch
constexpr long long kMaxPolls = 1ll << 22;

struct TileParams {
  HeomConsts c;
  int mode;
  int stage;
  const void *x;        // stage input (TX)
  void *out;            // apply output / next stage input (TX)
  double2 *y;           // RK4 state
  double2 *acc;         // RK4 accumulator
  void *y32;            // MIXED RK4: complex64 copy of y (written at stage 3)
  double a_next;
  double w_acc;
  Rk4Ctl *rk4;
  double2 *traj;
  void *k[5];           // RKF45 k0..k4 (TX)
  double2 *ybuf[2];     // RKF45 state ping-pong
  void *y32buf[2];      // MIXED RKF45: complex64 copies of ybuf
  Rkf45Ctl *ctl;
  uint8_t *act[2];               // filtering: active flags (see StageLaunch)
  int act_par;
  const double2 *dot_w;          // FP64 apply: <dot_w, out> per tile (see StageLaunch)
  double *dot_part;
  int npre;                      // epilogue operands prefetched
  const void *pre[kMaxPre];      // sources; slot 0 of RKF45 is chosen on the device
  int pre_bytes[kMaxPre];        // 16 (complex128) or 8 (complex64)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// One contiguous global -> shared copy (sizes and addresses multiples of 16 B).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// A hint: the contiguous global range [src, src + bytes) is brought into L2
// (16-byte aligned address, size a multiple of 16 bytes); nothing waits on it.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity of `bar` to complete;
// false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  long long polls = kMaxPolls) {
  for (long long i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Initialises the two mbarriers at the start of dynamic shared memory (one
// thread) and makes them visible to the CTA.
__device__ __forceinline__ void tile_init_barriers(unsigned char *smem_raw) {
  if (threadIdx.x == 0) {
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// complex helpers over double2 / float2
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <class TX> __device__ __forceinline__ TX from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <class TX> __device__ __forceinline__ TX mk(double re, double im);
template <> __device__ __forceinline__ double2 mk<double2>(double re, double im) { return make_double2(re, im); }
template <> __device__ __forceinline__ float2 mk<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}
__device__ __forceinline__ double2 cfma(double2 acc, double2 b, double s) {
  return make_double2(fma(b.x, s, acc.x), fma(b.y, s, acc.y));
}
template <class TX> __device__ __forceinline__ void st_stream(TX *p, TX v) { __stcs(p, v); }

template <int N, bool MIXED, int KT, int BT = kTileThreads>
struct TileShape {
  static constexpr int E = N * N;
  static constexpr int EP = E + (E & 1);  // complex64 node stride (16-byte aligned nodes)
  static constexpr int P = N * (N + 1) / 2;
  // (node, pair) items per thread: two for N >= 12, whose nodes would
  // otherwise leave a tile of one node and idle threads, two in mixed
  // precision from N = 4 (timed on B200: the 7-site RKF45 step 0.245 ->
  // 0.238 ms, the batched workload +16 % throughput; from N = 2 it gains
  // less, three are slower in both arithmetics), and two in FP64 for
  // K+1 = 3 up to N = 6 (the 4-site steady solve -4.5 %; with K+1 <= 2 FP64
  // is slower with two: 9 % on the 7-site step, 5 % on the batched one);
  // one otherwise.
  static constexpr bool kTwo = N >= 12 || (MIXED && N >= 4) || (!MIXED && KT == 3 && N <= 6);
  static constexpr int NT0 = (kTwo ? 2 : 1) * BT / P;
  static constexpr int NT = NT0 < 1 ? 1 : (NT0 > 64 ? 64 : NT0);
  // Column stride of the derivative tile in shared memory: odd, so the
  // transposed (j, i) writes of one warp fall in distinct banks.
  static constexpr int NP = (N & 1) ? N : N + 1;
  static constexpr int EU = N * NP;
};

template <int N, bool MIXED, int KT, int BT = kTileThreads>
struct TileLayout {
  using S = TileShape<N, MIXED, KT, BT>;
  static constexpr int ES = MIXED ? S::EP : S::E;  // node stride of X / k buffers
  static constexpr int XB = MIXED ? 8 : 16;        // bytes per element of X / k
  // byte offsets in dynamic shared memory
  static constexpr size_t kBars = 0;
  static constexpr size_t kX = 128;
  static constexpr size_t kXBytes = ((size_t)S::NT * ES * XB + 127) / 128 * 128;
  static constexpr size_t kU = kX + kXBytes;
  static constexpr size_t kUBytes = ((size_t)S::NT * S::EU * XB + 127) / 128 * 128;
  static constexpr size_t kPre = kU + kUBytes;
};

// Resident warps per SM the register budget is fitted to (timed on B200).
// K+1 = 2 (7 sites): FP64 6 % faster at 4 CTAs than at 5 without spills;
// mixed, with its two items per thread, 1 % faster at 4 (64 registers) than
// at 5 and 4 % faster than at 3.  K+1 = 1 (24 sites): FP64 1.6 % faster at
// 4 CTAs than at 5; the 320-thread mixed kernel fastest at 4 CTAs (40
// warps).  More neighbour terms per site keep more gathered values live.
template <int KT, bool MIXED, int BT = kTileThreads>
struct TileMinBlocks {
  static constexpr int warps = KT == 1 ? (MIXED ? 40 : 32) : (KT == 2 ? 32 : 24);
  static constexpr int value = warps / (BT / 32);
};

// New filter flags of a tile's nodes from |y_new|^2 staged in the first 8
// bytes of each derivative-tile slot (slot bytes apart, column stride NP):
// one warp per node; below the tolerance -> inactive, above -> active, equal
// -> unchanged (hierarchy_integrator.cc:2827-2850, :2359-2384).  A NaN never
// wins the `>`, as in PHI's scan.  Kept out of line so its registers do not
// add to the tile body's.
static __device__ __noinline__ void tile_filter_flags(const unsigned char *us, int slot, int N, int NP, int nt_here,
                                               const uint8_t *act_in, uint8_t *act_out, double tol,
                                               int warps) {
  const int E = N * N, lane = threadIdx.x & 31;
  for (int nd = threadIdx.x >> 5; nd < nt_here; nd += warps) {
    double m = 0.0;
    for (int w = lane; w < E; w += 32) {
      const int col = w / N;
      const double v = *reinterpret_cast<const double *>(us + (size_t)(nd * N * NP + (w - col * N) + col * NP) * slot);
      m = v > m ? v : m;
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_xor_sync(0xffffffffu, m, off);
      m = o > m ? o : m;
    }
    if (lane == 0) {
      const double mx = sqrt(m);
      act_out[nd] = mx < tol ? (uint8_t)0 : (mx > tol ? (uint8_t)1 : act_in[nd]);
    }
  }
}

template <bool MIXED>
struct TileArith {
  using TX = typename std::conditional<MIXED, float2, double2>::type;
  using R = typename std::conditional<MIXED, float, double>::type;
};

// ---- the parts of one tile shared by the kernels ----
// Phase 2: the derivative of every (node, upper-triangle pair) of a tile into
// the derivative tile Us, from shared memory (the tile's stage input Xs, H,
// per-element Matsubara factors, pair lists, per-(node, term) neighbour
// offsets and prefactor magnitudes, dephasing rates) and, for the neighbour
// terms, from the stage input in HBM (xin).  HX_US: the products A = H X of
// the tile are already in Us (computed on the tensor cores); each item reads
// its two entries A_ij, A_ji there before it overwrites them with the
// derivative (no other item touches those two slots).
template <int N, int KT, bool MIXED, int BT, bool HX_US = false>
__device__ __forceinline__ void tile_pairs(const HeomConsts &c, const typename TileArith<MIXED>::TX *Xs,
                                           typename TileArith<MIXED>::TX *Us,
                                           const typename TileArith<MIXED>::TX *Hs,
                                           const typename TileArith<MIXED>::R *mats, const unsigned char *pi,
                                           const unsigned char *pj, const int *ids,
                                           const typename TileArith<MIXED>::R *cn,
                                           const typename TileArith<MIXED>::R *cp,
                                           const typename TileArith<MIXED>::R *ccr, const double *deph,
                                           const int *nts, const typename TileArith<MIXED>::TX *xin, int nt_here) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = TileLayout<N, MIXED, KT, BT>;
  using TX = typename TileArith<MIXED>::TX;
  using R = typename TileArith<MIXED>::R;
  constexpr int P = S::P, ES = Lay::ES, NP = S::NP, EU = S::EU;
  constexpr int T = N * KT;
  const int tid = threadIdx.x;
  const bool hreal = c.h_real;
  const R *Hr = reinterpret_cast<const R *>(Hs);
  const R ih = (R)c.inv_hbar;
  const int items = nt_here * P;
  for (int it = tid; it < items; it += BT) {
    const int nd = it / P, u = it - nd * P;
    const int i = pi[u], j = pj[u];
    const TX *X = Xs + nd * ES;
    // Every neighbour value this pair needs, as independent predicated loads.
    // In mixed precision they are issued before the products, whose work
    // then hides their latency (timed on B200: 7-site RKF45 step -1.5 %,
    // 24-site -1 %, batched RK4 -2.6 %); the FP64 kernels issue them after
    // the products, where the extra live registers do not spill (hoisted:
    // 7-site FP64 unchanged, 4-site steady solve 0.7 % slower).
    constexpr bool kHoist = MIXED;
    TX gn_c[KT], gp_c[KT], gn_r[KT], gp_r[KT];
    auto gather = [&]() {
      const int *nid = ids + nd * 2 * T;
      const int oij = i + j * N, oji = j + i * N;
      const TX zero = mk<TX>(0.0, 0.0);
      const bool on = !c.vacuum;
#pragma unroll
      for (int q = 0; q < KT; ++q) {
        const int tj = j * KT + q, ti = i * KT + q;
        const int nxj = nid[tj], pvj = nid[T + tj], nxi = nid[ti], pvi = nid[T + ti];
        gn_c[q] = (on && nxj >= 0 && i != j) ? __ldg(xin + nxj + oij) : zero;
        gp_c[q] = (on && pvj >= 0 && i != j) ? __ldg(xin + pvj + oij) : zero;
        gn_r[q] = (on && nxi >= 0 && i != j) ? __ldg(xin + nxi + oji) : zero;
        gp_r[q] = (on && pvi >= 0) ? __ldg(xin + pvi + oji) : zero;
      }
    };
    if constexpr (kHoist) gather();
    R ar = 0, ai = 0, br = 0, bi = 0;  // A_ij, A_ji
    if (HX_US) {
      const TX aij = Us[nd * EU + i + j * NP], aji = Us[nd * EU + j + i * NP];
      ar = aij.x;
      ai = aij.y;
      br = aji.x;
      bi = aji.y;
    } else if (hreal) {
#pragma unroll
      for (int k = 0; k < N; ++k) {
        // X_ki = conj(X_ik) (Hermitian ADO): lanes with consecutive i read
        // consecutive words instead of a stride of N.
        const R hik = Hr[i + k * N], hjk = Hr[j + k * N];
        const TX xkj = X[k + j * N], xik = X[i + k * N];
        ar = fma(hik, xkj.x, ar);
        ai = fma(hik, xkj.y, ai);
        br = fma(hjk, xik.x, br);
        bi = fma(-hjk, xik.y, bi);
      }
    } else {
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const TX hik = Hs[i + k * N], xkj = X[k + j * N];
        const TX hjk = Hs[j + k * N], xik = X[i + k * N];  // X_ki = conj(X_ik)
        ar = fma(hik.x, xkj.x, ar);
        ar = fma(-hik.y, xkj.y, ar);
        ai = fma(hik.x, xkj.y, ai);
        ai = fma(hik.y, xkj.x, ai);
        br = fma(hjk.x, xik.x, br);
        br = fma(hjk.y, xik.y, br);
        bi = fma(-hjk.x, xik.y, bi);
        bi = fma(hjk.y, xik.x, bi);
      }
    }
    // -i/hbar (A_ij - conj(A_ji))
    R vx = (ai + bi) * ih, vy = -(ar - br) * ih;
    const TX xij = X[i + j * N];
    if (!c.vacuum) {
      const R fac = (R)deph[nd] + mats[i + j * N];
      vx = fma(-fac, xij.x, vx);
      vy = fma(-fac, xij.y, vy);
      const R *ncn = cn + nd * T, *ncp = cp + nd * T;
      if constexpr (!kHoist) gather();
      if (i != j) {
#pragma unroll
        for (int q = 0; q < KT; ++q) {
          const int tj = j * KT + q, ti = i * KT + q;
          // column part: + p X+_ij (p = i s), + i conj(c) sp X-_ij
          const R sj = ncn[tj];
          vx = fma(-sj, gn_c[q].y, vx);
          vy = fma(sj, gn_c[q].x, vy);
          const R spj = ncp[tj];
          const R cjx = ccr[2 * tj], cjy = ccr[2 * tj + 1];
          const TX g = gp_c[q];
          const R re = cjx * g.x + cjy * g.y, im = cjx * g.y - cjy * g.x;
          vx = fma(-spj, im, vx);
          vy = fma(spj, re, vy);
          // row part: - p conj(X+_ji), - i c sp conj(X-_ji)
          const R si = ncn[ti];
          vx = fma(-si, gn_r[q].y, vx);
          vy = fma(-si, gn_r[q].x, vy);
          const R spi = ncp[ti];
          const R cix = ccr[2 * ti], ciy = ccr[2 * ti + 1];
          const TX h = gp_r[q];
          const R re2 = cix * h.x + ciy * h.y, im2 = ciy * h.x - cix * h.y;
          vx = fma(spi, im2, vx);
          vy = fma(-spi, re2, vy);
        }
      } else {
        // diagonal: next terms cancel; prev gives 2 sp Im(c) X-_mm
#pragma unroll
        for (int q = 0; q < KT; ++q) {
          const int ti = i * KT + q;
          const R spi = ncp[ti];
          const R ciy = ccr[2 * ti + 1];
          vx = fma((R)2 * spi * ciy, gp_r[q].x, vx);
        }
      }
    }
    TX v;
    v.x = vx;
    v.y = vy;
    if (i == j) {
      v.y = 0;
      Us[nd * EU + i + j * NP] = v;
    } else {
      Us[nd * EU + i + j * NP] = v;
      v.y = -v.y;
      Us[nd * EU + j + i * NP] = v;
    }
  }
  // Time-local truncation: the deepest tier's term, a pass of its own so the
  // pair loop above keeps its registers.  Item `it` maps to the thread that
  // wrote its two slots in the pair loop, so no barrier is needed before it.
  if (c.time_local) {
    for (int it = tid; it < items; it += BT) {
      const int nd = it / P, u = it - nd * P;
      const int i = pi[u], j = pj[u];
      if (i == j) continue;
      int tier = 0;  // deepest tier only (is_timelocal_truncated)
      for (int t = 0; t < T; ++t) tier += nts[nd * T + t];
      if (tier != c.L) continue;
      const TX tv = tl_pair_term<TX>(Xs + nd * ES, c.tl_q, N, i, j);
      TX a = Us[nd * EU + i + j * NP];
      a.x += tv.x;
      a.y += tv.y;
      Us[nd * EU + i + j * NP] = a;
      TX b = Us[nd * EU + j + i * NP];  // the Hermitian partner takes conj(tv)
      b.x += tv.x;
      b.y -= tv.y;
      Us[nd * EU + j + i * NP] = b;
    }
  }
}

// Phase 3: the epilogue over a tile's elements (plain store, RK4 or RKF45
// stage combine) from the derivative tile Us and the prefetched operands at
// PreBase + pre_off[b]; the RKF45 stage-5 error of this thread's elements is
// folded into emax (max of |y4 - y5|, or of its square in mixed precision).
// coef holds the 24 RKF45 coefficients in FP64 followed by the same 24 in
// FP32.
template <int N, int KT, bool MIXED, int BT>
__device__ __forceinline__ void tile_epilogue(const TileParams &p, const typename TileArith<MIXED>::TX *Xs,
                                              typename TileArith<MIXED>::TX *Us, const unsigned char *PreBase,
                                              const uint32_t (&pre_off)[kMaxPre], const double *coef,
                                              unsigned long long *wmax, long long tile, long long n0, int nt_here,
                                              int ycur, double &emax) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = TileLayout<N, MIXED, KT, BT>;
  using TX = typename TileArith<MIXED>::TX;
  constexpr int E = S::E, ES = Lay::ES, NP = S::NP, EU = S::EU;
  const HeomConsts &c = p.c;
  const int tid = threadIdx.x;
  const int tile_elems = nt_here * E;
  auto uix = [](int e) {
    if (NP == N) return e;
    const int nd = e / E, w = e - nd * E, cc = w / N;
    return nd * EU + (w - cc * N) + cc * NP;
  };
  auto flag_stage = [&]() {
    return c.filtered && ((p.mode == kModeRk4 && p.stage == 3) || (p.mode == kModeRkf45 && p.stage == 5));
  };
  // element e of the tile: node nd = e / E, offset w = e % E; complex128
  // buffers are indexed (n0 + nd) * E + w, X / k buffers (n0 + nd) * ES + w.
  auto preD = [&](int b) { return reinterpret_cast<const double2 *>(PreBase + pre_off[b]); };
  // RKF45 operand slot 0 is the state y: 16 bytes -> y staged in complex128;
  // 8 bytes (mixed stages 1-4) -> its complex64 copy y32, which is all the
  // complex64 stage input X_{s+1} = y + sum b k needs; 0 bytes -> y read from
  // global memory in the epilogue (mixed stage 5, and the 24-site FP64
  // kernels' stages 3-5: less shared memory per tile, more CTAs per SM).
  const int ybytes = p.npre > 0 ? p.pre_bytes[0] : 16;
  auto preX = [&](int b) { return reinterpret_cast<const TX *>(PreBase + pre_off[b]); };
  // Filtering: |y_new|^2 of element e goes to the first 8 bytes of its own
  // slot Us[uix(e)], which only this thread reads, and only before; the
  // per-node maxima are taken from there after the loop.
  auto fl_put = [&](int e, double2 v) {
    *reinterpret_cast<double *>(&Us[uix(e)]) = fma(v.x, v.x, v.y * v.y);
  };
  if (p.mode == kModeApply) {
    TX *out = static_cast<TX *>(p.out);
    bool dot = false;
    if constexpr (!MIXED) dot = p.dot_w != nullptr;
    if (!dot) {
      for (int e = tid; e < tile_elems; e += BT) {
        const int nd = e / E, w = e - nd * E;
        st_stream(out + (n0 + nd) * ES + w, Us[uix(e)]);
      }
    } else if constexpr (!MIXED) {
      // Steady-state solve: the output's element (0,0) of node 0 is the
      // eliminated unknown (zero), and the tile's share of <dot_w, out> (the
      // real inner product of Hermitian states) goes to dot_part[tile] --
      // the inner product the solver would otherwise read the vector for.
      double dsum = 0.0;
      for (int e = tid; e < tile_elems; e += BT) {
        const int nd = e / E, w = e - nd * E;
        const long long gx = (n0 + nd) * ES + w;
        TX v = Us[uix(e)];
        if (gx == 0) v = mk<TX>(0.0, 0.0);
        st_stream(out + gx, v);
        const double2 r = __ldg(p.dot_w + gx);
        dsum = fma(r.x, v.x, fma(r.y, v.y, dsum));
      }
      for (int off = 16; off > 0; off >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, off);
      double *wsum = reinterpret_cast<double *>(wmax);
      if ((tid & 31) == 0) wsum[tid >> 5] = dsum;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < BT / 32; ++w) t += wsum[w];
        p.dot_part[tile] = t;
      }
    }
  } else if (p.mode == kModeRk4) {
    const int s = p.stage;
    TX *out = static_cast<TX *>(p.out);
    long long row = -1;
    if (s == 3 && n0 == 0 && p.traj) {
      const Rk4Ctl *rc = p.rk4;
      if (rc->out_factor > 0 && rc->step % rc->out_factor == 0 && rc->nout < rc->capacity) row = rc->nout;
    }
    for (int e = tid; e < tile_elems; e += BT) {
      const int nd = e / E, w = e - nd * E;
      const long long gd = (n0 + nd) * E + w, gx = (n0 + nd) * ES + w;
      const double2 kv = to_d2(Us[uix(e)]);
      if (MIXED && s < 3) {
        // Mixed: the complex64 stage input y32 + a k in FP32 (stage 0: y32
        // is the input; stages 1-2: pre = {y32, acc}); the accumulator in
        // FP64 (stage 0: pre = {y}).
        const float af = (float)p.a_next;
        const TX kx = Us[uix(e)];
        const TX ys = s == 0 ? Xs[nd * ES + w] : preX(0)[nd * ES + w];
        out[gx] = mk<TX>(fmaf((float)kx.x, af, (float)ys.x), fmaf((float)kx.y, af, (float)ys.y));
        st_stream(p.acc + gd, cfma((s == 0 ? preD(0) : preD(1))[e], kv, p.w_acc));
      } else if (s == 0) {  // FP64: pre = {} (y is the input)
        const double2 ys = to_d2(Xs[nd * ES + w]);
        out[gx] = from_d2<TX>(cfma(ys, kv, p.a_next));
        st_stream(p.acc + gd, cfma(ys, kv, p.w_acc));
      } else if (s < 3) {  // pre = {y, acc}
        out[gx] = from_d2<TX>(cfma(preD(0)[e], kv, p.a_next));
        st_stream(p.acc + gd, cfma(preD(1)[e], kv, p.w_acc));
      } else {             // pre = {acc}
        const double2 yn = cfma(preD(0)[e], kv, p.w_acc);
        p.y[gd] = yn;
        if (MIXED) static_cast<TX *>(p.y32)[gx] = from_d2<TX>(yn);
        if (row >= 0 && e < E) p.traj[row * E + e] = yn;
        if (flag_stage()) fl_put(e, yn);
      }
    }
    if (s == 3 && n0 == 0 && p.traj) {
      __syncthreads();
      if (tid == 0) {
        Rk4Ctl *rc = p.rk4;
        if (row >= 0) rc->nout = rc->nout + 1;
        rc->step = rc->step + 1;
      }
    }
  } else {
    const int s = p.stage;
    const double *cf = coef;
    TX *out = static_cast<TX *>(p.out);
    for (int e = tid; e < tile_elems; e += BT) {
      const int nd = e / E, w = e - nd * E;
      const long long gd = (n0 + nd) * E + w, gx = (n0 + nd) * ES + w;
      const TX kx = Us[uix(e)];
      const double2 kv = to_d2(kx);
      if (MIXED && s < 5) {
        // Mixed stages 0-4: the complex64 stage input X_{s+1} = y32 + sum b k
        // in FP32 throughout (it is stored in complex64; an FP64 combine
        // rounded to it differs by an ulp of complex64).  pre = {y32, k_0 ..
        // k_{s-1}}; stage 0: y32 is the input.
        const float *cff = reinterpret_cast<const float *>(coef + 24);
        const TX ys = s == 0 ? Xs[nd * ES + w] : preX(0)[nd * ES + w];
        st_stream(static_cast<TX *>(p.k[s]) + gx, kx);
        const int row = s * (s + 1) / 2;
        float xr = ys.x, xi = ys.y;
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (r < s) {
            const TX kr = preX(1 + r)[nd * ES + w];
            xr = fmaf((float)kr.x, cff[row + r], xr);
            xi = fmaf((float)kr.y, cff[row + r], xi);
          }
        xr = fmaf((float)kx.x, cff[row + s], xr);
        xi = fmaf((float)kx.y, cff[row + s], xi);
        out[gx] = mk<TX>(xr, xi);
      } else if (s < 5) {  // pre = {y, k_0 .. k_{s-1}}; stage 0: y is the input
        const double2 ys = s == 0 ? to_d2(Xs[nd * ES + w])
                           : (ybytes == 0 ? __ldg(p.ybuf[ycur] + gd)
                                          : (ybytes == 8 ? to_d2(preX(0)[nd * ES + w]) : preD(0)[e]));
        st_stream(static_cast<TX *>(p.k[s]) + gx, kx);
        const int row = s * (s + 1) / 2;
        double2 xv = ys;
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (r < s) xv = cfma(xv, to_d2(preX(1 + r)[nd * ES + w]), cf[row + r]);
        xv = cfma(xv, kv, cf[row + s]);
        out[gx] = from_d2<TX>(xv);
      } else {      // pre = {y, k0, k2, k3, k4}
        const double2 ys = ybytes == 0 ? __ldg(p.ybuf[ycur] + gd) : preD(0)[e];
        const double2 k0 = to_d2(preX(1)[nd * ES + w]), k2 = to_d2(preX(2)[nd * ES + w]);
        const double2 k3 = to_d2(preX(3)[nd * ES + w]), k4 = to_d2(preX(4)[nd * ES + w]);
        double2 y4 = cfma(ys, k0, cf[15]);
        y4 = cfma(y4, k2, cf[16]);
        y4 = cfma(y4, k3, cf[17]);
        y4 = cfma(y4, k4, cf[18]);
        double2 y5 = cfma(ys, k0, cf[19]);
        y5 = cfma(y5, k2, cf[20]);
        y5 = cfma(y5, k3, cf[21]);
        y5 = cfma(y5, k4, cf[22]);
        y5 = cfma(y5, kv, cf[23]);
        st_stream(p.ybuf[ycur ^ 1] + gd, y5);
        if (MIXED) st_stream(static_cast<TX *>(p.y32buf[ycur ^ 1]) + gx, from_d2<TX>(y5));
        if (flag_stage()) fl_put(e, y5);
        const double dx = y4.x - y5.x, dy = y4.y - y5.y;
        if (MIXED) {
          // max of |y4 - y5|^2; one square root per thread below
          const double e2 = fma(dx, dx, dy * dy);
          emax = (e2 > emax || e2 != e2) ? e2 : emax;
        } else {
          // |z| as PHI computes it (std::abs of the complex difference)
          const double err = hypot(dx, dy);
          emax = (err > emax || err != err) ? err : emax;
        }
      }
    }
  }
}

// The RKF45 stage-5 error of a CTA: the maximum over its threads' emax, one
// atomicMax on the bit pattern of the control block's error word.
template <bool MIXED, int BT>
__device__ __forceinline__ void tile_error_max(const TileParams &p, double emax, unsigned long long *wmax) {
  const int tid = threadIdx.x;
  if (MIXED) emax = sqrt(emax);
    unsigned long long bits = (unsigned long long)__double_as_longlong(emax);
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
      bits = o > bits ? o : bits;
    }
    // One atomic per CTA: a single error word takes every CTA's maximum,
    // so per-warp atomics would serialise tens of thousands of updates.
    if ((tid & 31) == 0) wmax[tid >> 5] = bits;
    __syncthreads();
    if (tid == 0) {
      unsigned long long m = wmax[0];
#pragma unroll
      for (int w = 1; w < (BT / 32); ++w) m = wmax[w] > m ? wmax[w] : m;
      if (m) atomicMax(&p.ctl->err_bits, m);
    }
}

// New filter flags of a tile's nodes after the stage that writes the new
// state (RK4 stage 3, RKF45 stage 5).
template <int N, int KT, bool MIXED, int BT>
__device__ __forceinline__ void tile_flags(const TileParams &p, const typename TileArith<MIXED>::TX *Us, long long n0,
                                           int nt_here, int ycur) {
  using S = TileShape<N, MIXED, KT, BT>;
  using TX = typename TileArith<MIXED>::TX;
  const HeomConsts &c = p.c;
  if (!(c.filtered && ((p.mode == kModeRk4 && p.stage == 3) || (p.mode == kModeRkf45 && p.stage == 5)))) return;
  // Below the tolerance -> inactive, above -> active, equal -> unchanged
  // (hierarchy_integrator.cc:2827-2850, :2359-2384).
  __syncthreads();
  const int ap = p.mode == kModeRkf45 ? ycur : p.act_par;
  tile_filter_flags(reinterpret_cast<const unsigned char *>(Us), (int)sizeof(TX), N, S::NP, nt_here,
                    p.act[ap] + n0, p.act[ap ^ 1] + n0, c.filter_tol, BT / 32);
}


// KT = terms per site (K + 1) under PHI's identity site map.
// One tile (NT consecutive nodes of one hierarchy) of one stage.  The caller
// has initialised the two mbarriers at the start of shared memory and passes
// the phase parity each is at.  Returns 1 when the tile was skipped before
// any copy was issued (RKF45 run finished), 0 when both barriers completed a
// phase (barrier 1 with 0 bytes when p.npre == 0), -1 after a bounded wait gave up
// (err_flag set; the caller must stop).
template <int N, int KT, bool MIXED, int BT = kTileThreads>
__device__ __forceinline__ int tile_body(const TileParams &p, long long tile, unsigned char *smem_raw,
                                         uint32_t par0, uint32_t par1) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = TileLayout<N, MIXED, KT, BT>;
  using TX = typename std::conditional<MIXED, float2, double2>::type;
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr int E = S::E, P = S::P, NT = S::NT, ES = Lay::ES;
  const HeomConsts &c = p.c;
  constexpr int T = N * KT;  // PHI's identity site map: K+1 terms per site
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + Lay::kBars);
  TX *Xs = reinterpret_cast<TX *>(smem_raw + Lay::kX);   // NT*ES
  TX *Us = reinterpret_cast<TX *>(smem_raw + Lay::kU);   // NT*EU (column stride NP)
  unsigned char *PreBase = smem_raw + Lay::kPre;
  // Byte offsets of the prefetched epilogue operands.  Every loop over them
  // is unrolled so the offsets stay in registers.
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
  TX *Hs = reinterpret_cast<TX *>(smem_raw + tail);                 // E
  double *deph = reinterpret_cast<double *>(Hs + E);                // NT (8-aligned: E*8 or E*16)
  double *coef = deph + NT;                                         // 24, then 24 floats
  unsigned long long *wmax = reinterpret_cast<unsigned long long *>(coef + 36);  // per-warp maxima
  R *cn = reinterpret_cast<R *>(wmax + (BT / 32));                          // NT*T |next prefactor|
  R *cp = cn + NT * T;                                              // NT*T prev scale
  R *ccr = cp + NT * T;                                             // 2T   c_t (re, im)
  R *mats = ccr + 2 * T;                                            // E    Matsubara factor per element
  int *ids = reinterpret_cast<int *>(mats + E);                     // NT*2T element offsets
  int *nts = ids + NT * 2 * T;                                      // NT*T
  unsigned char *pi = reinterpret_cast<unsigned char *>(nts + NT * T);
  unsigned char *pj = pi + P;

  const int tid = threadIdx.x;
  int ycur = 0;
  if (p.mode == kModeRkf45) {
    if (*(volatile int *)&p.ctl->done) return 1;  // uniform across the grid
    ycur = p.ctl->ycur;
    if (tid < 24) {
      const double v = p.ctl->coef[tid];
      coef[tid] = v;
      reinterpret_cast<float *>(coef + 24)[tid] = (float)v;
    }
  }
  const long long n0 = tile * NT;
  if (n0 >= c.M) return 1;
  // Filtering: the flags of the current state are p.act[ap], ap = ycur
  // (RKF45) or p.act_par; the launch that writes the new state (RK4 stage 3,
  // RKF45 stage 5 -- the candidate, kept on accept) writes its flags to
  // p.act[ap ^ 1].  Both are recomputed from the parameters where used, so
  // nothing of it stays live across the tile.
  auto act_idx = [&]() { return p.mode == kModeRkf45 ? ycur : p.act_par; };
  const int nt_here = (int)((c.M - n0) < NT ? (c.M - n0) : NT);
  const TX *xin;
  if (p.mode == kModeRkf45 && p.stage == 0)
    xin = MIXED ? static_cast<const TX *>(p.y32buf[ycur]) : reinterpret_cast<const TX *>(p.ybuf[ycur]);
  else
    xin = static_cast<const TX *>(p.x);

  // ---- t = 0: bulk prefetch of the tile's contiguous ranges ----
  if (tid == 0) {
    const uint32_t xbytes = (uint32_t)(nt_here * ES * Lay::XB);
    mbar_expect_tx(&bars[0], xbytes);
    bulk_g2s(Xs, xin + n0 * ES, xbytes, &bars[0]);
    uint32_t pbytes = 0;
#pragma unroll
    for (int b = 0; b < kMaxPre; ++b)
      if (b < p.npre) pbytes += (uint32_t)(nt_here * (p.pre_bytes[b] == 16 ? E : ES) * p.pre_bytes[b]);
    // Arrives on barrier 1 in every tile (with 0 bytes when nothing is
    // prefetched), so its phase advances once per tile like barrier 0's.
    mbar_expect_tx(&bars[1], pbytes);
#pragma unroll
    for (int b = 0; b < kMaxPre; ++b) {
      if (b >= p.npre) break;
      if (p.pre_bytes[b] == 0) continue;  // read from global in the epilogue
      const unsigned char *src = static_cast<const unsigned char *>(p.pre[b]);
      if (b == 0 && p.mode == kModeRkf45)
        src = static_cast<const unsigned char *>(p.pre_bytes[0] == 8 ? p.y32buf[ycur] : (const void *)p.ybuf[ycur]);
      const int stride = p.pre_bytes[b] == 16 ? E : ES;
      const uint32_t bytes = (uint32_t)(nt_here * stride * p.pre_bytes[b]);
      bulk_g2s(PreBase + pre_off[b], src + (size_t)n0 * stride * p.pre_bytes[b], bytes, &bars[1]);
    }
  }
  // A real Hamiltonian (every in-scope workload) is kept as E reals in the
  // same buffer, halving the products of A = H X.
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
  const int W = c.L + 2;
  const int tile_terms = nt_here * T;
  // Per (node, term): neighbour ids scaled to element offsets of the stage
  // input (-1 when absent), occupation, and the prefactor magnitudes for that
  // occupation, so the pair loop reads shared memory only.
  const uint8_t *act_in = c.filtered ? p.act[act_idx()] : nullptr;
  for (int q = tid; q < tile_terms; q += BT) {
    const int nd = q / T, t = q - nd * T;
    const int nx = __ldg(c.next + n0 * T + q), pv = __ldg(c.prev + n0 * T + q);
    const int nt = __ldg(c.mi + n0 * T + q);
    // An inactive neighbour contributes nothing (the DoNext / DoPrevious
    // overrides of IndependentBathAdaptiveTruncation, hierarchy_updater.cc:256-303).
    const bool nx_on = nx >= 0 && (!act_in || __ldg(act_in + nx));
    const bool pv_on = pv >= 0 && (!act_in || __ldg(act_in + pv));
    ids[nd * 2 * T + t] = nx_on ? nx * ES : -1;
    ids[nd * 2 * T + T + t] = pv_on ? pv * ES : -1;
    nts[q] = nt;
    cn[q] = (R)__ldg(c.sq_next + t * W + nt);
    cp[q] = (R)__ldg(c.sq_prev + t * W + nt);
  }
  for (int t = tid; t < T; t += BT) {
    const double2 ct = __ldg(c.corr + t);
    ccr[2 * t] = (R)ct.x;
    ccr[2 * t + 1] = (R)ct.y;
  }
  __syncthreads();  // barrier init and metadata visible
  if (tid < nt_here) {
    double d = 0.0;
    for (int t = 0; t < T; ++t) d = fma((double)nts[tid * T + t], __ldg(c.nu + t), d);
    deph[tid] = d;
  }
  const long long polls0 = c.first_wait_polls == 0 ? kMaxPolls : (c.first_wait_polls < 0 ? 0 : c.first_wait_polls);
  bool ok = mbar_wait_bounded(&bars[0], par0, polls0);
  __syncthreads();  // deph visible
  if (!__syncthreads_and(ok)) {
    if (tid == 0) atomicOr(c.err_flag, 1);
    // Drain this tile's own copies with the built-in limit, so no copy is
    // still writing into shared memory when the CTA stops.
    mbar_wait_bounded(&bars[0], par0);
    if (p.npre > 0) mbar_wait_bounded(&bars[1], par1);
    return -1;
  }

  tile_pairs<N, KT, MIXED, BT>(c, Xs, Us, Hs, mats, pi, pj, ids, cn, cp, ccr, deph, nts, xin, nt_here);
  ok = p.npre == 0 || mbar_wait_bounded(&bars[1], par1);
  if (!__syncthreads_and(ok)) {
    if (tid == 0) atomicOr(c.err_flag, 1);
    return -1;
  }
  double emax = 0.0;
  tile_epilogue<N, KT, MIXED, BT>(p, Xs, Us, PreBase, pre_off, coef, wmax, tile, n0, nt_here, ycur, emax);
  if (p.mode == kModeRkf45 && p.stage == 5) tile_error_max<MIXED, BT>(p, emax, wmax);
  tile_flags<N, KT, MIXED, BT>(p, Us, n0, nt_here, ycur);
  return 0;
}

template <int N, int KT, bool MIXED, int BT = kTileThreads>
inline size_t tile_smem(int T, int npre, const int *pre_bytes) {
  using S = TileShape<N, MIXED, KT, BT>;
  using Lay = TileLayout<N, MIXED, KT, BT>;
  size_t b = Lay::kPre;
  for (int i = 0; i < npre; ++i)
    b += ((size_t)S::NT * (pre_bytes[i] == 16 ? S::E : Lay::ES) * pre_bytes[i] + 127) / 128 * 128;
  b += (size_t)S::E * Lay::XB;
  b += (size_t)(S::NT + 36 + BT / 32) * sizeof(double);  // deph, coef (FP64 and FP32), warp maxima
  b += (size_t)(2 * S::NT * T + 2 * T + S::E) * Lay::XB / 2;  // cn, cp, ccr, mats in the arithmetic type
  b += (size_t)(S::NT * 3 * T) * sizeof(int);
  b += 2 * S::P + 16;
  return b;
}

// The tile parameters of one stage launch (host; heom_tile.cu).
TileParams tile_params_for(const StageLaunch &L);

}  // namespace tile_detail
}  // namespace phi
