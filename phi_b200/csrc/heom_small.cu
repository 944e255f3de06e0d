// heom_small.cu -- the whole RK4 run of a small hierarchy in one CTA.
//
// A hierarchy of a few hundred elements (PHI's spin-boson configuration has
// 11 nodes of 2 x 2) gives each stage kernel a handful of warps of work, so
// a run of four launches per step is bound by launch and memory latency,
// not by the SMs.  Here one CTA keeps the state y, the RK4 accumulator, the
// stage input and the stage derivative in shared memory and loops over every
// step of the run on the device: a stage is one pass over the hierarchy's
// upper-triangle (node, pair) items and one element-wise combine, separated
// by block barriers.  The arithmetic is that of the generic group kernel
// (heom_kernels.cu) for IndependentBath and DiagonalBath couplings:
// HierarchyUpdater::Get (hierarchy_updater.h:36-75, hierarchy_updater.cc
// :84-127, :216-254) and the RK4 combines of Rk4Integrate
// (hierarchy_integrator.cc:2705-2826); every derivative ADO is evaluated on
// its upper triangle and mirrored.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "heom_device.cuh"
#include "heom_kernels.h"
#include "heom_tile.h"

namespace phi {
namespace {

constexpr int kSmallThreads = 256;  // at most; register rows need one thread per item

__device__ __forceinline__ double2 s_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 s_axpy(double2 a, double2 b, double s) {
  return make_double2(fma(b.x, s, a.x), fma(b.y, s, a.y));
}

struct SmallRk4Params {
  HeomConsts c;
  double2 *y;     // hierarchy state (global), read at the start, written at the end
  double dt;
  long long steps;
  Rk4Ctl *rk4;    // step / output bookkeeping, as the stage kernels keep it
  double2 *traj;  // rho_0 rows (may be null)
};

// The derivative of node n's ADO at an upper-triangle pair (i, j) is a
// fixed linear combination of stage-input elements (every stage input is
// exactly Hermitian).  Each item's combination -- element offsets and complex
// coefficients -- is built once per launch into shared memory, so a stage
// is R complex multiply-adds from shared memory per item:
//   -i/hbar [H, X]_ij = sum_k (-i/hbar) H_ik X_kj + (i/hbar) conj(H_jk) X_ik
//   -(dephasing_n + Matsubara_ij) X_ij
//   IndependentBath (hierarchy_updater.cc:216-254), site m = j: +i p X+_ij,
//     +i sp conj(c) X-_ij; site m = i: -i p X+_ij, -i sp c X-_ij; i = j = m:
//     2 sp Im(c) X-_mm (the next terms cancel);
//   DiagonalBath (:105-127): -i (V_i - V_j) X+_ij, -i n (c V_i - c* V_j) X-_ij.
struct RowBuilder {
  int *idx;
  double2 *coef;
  int n = 0;
  __device__ void add(long long e, double2 cf) {
    idx[n] = (int)e;
    coef[n] = cf;
    ++n;
  }
};

template <int KIND>
__device__ int build_row(const HeomConsts &c, const double2 *Hs, long long n, int i, int j, int *idx,
                         double2 *coef) {
  const int N = c.N, E = N * N, T = c.T, L2 = c.L + 2;
  const double ih = c.inv_hbar;
  RowBuilder r{idx, coef};
  const long long base = n * E;
  for (int k = 0; k < N; ++k) {
    const double2 h1 = Hs[i + k * N], h2 = Hs[j + k * N];
    r.add(base + k + j * N, make_double2(h1.y * ih, -h1.x * ih));   // -i ih H_ik
    r.add(base + i + k * N, make_double2(h2.y * ih, h2.x * ih));    // +i ih conj(H_jk)
  }
  if (c.vacuum) return r.n;
  double deph = 0.0;  // sum_t n_t nu_t in term order
  for (int t = 0; t < T; ++t) deph += __ldg(c.mi + n * T + t) * __ldg(c.nu + t);
  r.add(base + i + j * N, make_double2(-(deph + __ldg(c.mats_elem + i + j * N)), 0.0));
  if (KIND == kIndependent) {
    for (int side = 0; side < 2; ++side) {
      const int site = side == 0 ? j : i;
      for (int q = __ldg(c.site_ptr + site); q < __ldg(c.site_ptr + site + 1); ++q) {
        const int t = __ldg(c.site_terms + q);
        const int nt = __ldg(c.mi + n * T + t);
        const int nx = __ldg(c.next + n * T + t), pv = __ldg(c.prev + n * T + t);
        const double sn = __ldg(c.sq_next + t * L2 + nt), sp = __ldg(c.sq_prev + t * L2 + nt);
        const double2 ct = __ldg(c.corr + t);
        const long long off = (long long)i + (long long)j * N;
        if (i == j) {
          if (side == 1 && pv >= 0) r.add((long long)pv * E + off, make_double2(2.0 * sp * ct.y, 0.0));
          continue;
        }
        if (side == 0) {
          if (nx >= 0) r.add((long long)nx * E + off, make_double2(0.0, sn));
          if (pv >= 0) r.add((long long)pv * E + off, make_double2(sp * ct.y, sp * ct.x));   // i sp conj(c)
        } else {
          if (nx >= 0) r.add((long long)nx * E + off, make_double2(0.0, -sn));
          if (pv >= 0) r.add((long long)pv * E + off, make_double2(sp * ct.y, -sp * ct.x));  // -i sp c
        }
      }
    }
  } else {
    for (int s2 = 0; s2 < 2 * T; ++s2) {
      const bool is_next = s2 < T;
      const int t = is_next ? s2 : s2 - T;
      const int id = is_next ? __ldg(c.next + n * T + t) : __ldg(c.prev + n * T + t);
      if (id < 0) continue;
      const double *V = c.bath_V + (size_t)__ldg(c.term_site + t) * N;
      const double vi = __ldg(V + i), vj = __ldg(V + j);
      double2 f;
      if (is_next) {
        f = make_double2(0.0, -(vi - vj));
      } else {
        const double2 ct = __ldg(c.corr + t);
        const int nt = __ldg(c.mi + n * T + t);
        const double re = ct.x * vi - ct.x * vj;
        const double im = ct.y * vi + ct.y * vj;
        f = make_double2(im * nt, -re * nt);
      }
      r.add((long long)id * E + i + (long long)j * N, f);
    }
  }
  return r.n;
}

// Entries of one item's row, an upper bound: the commutator (2N), the decay,
// and the neighbour terms (IndependentBath: next and prev of the terms of
// sites i and j; DiagonalBath: next and prev of every term).
__host__ __device__ inline int small_row_max(const HeomConsts &c) {
  return 2 * c.N + 1 + (c.kind == kIndependent ? 4 * c.T : 2 * c.T);
}

// RM > 0: every thread owns at most one item and keeps its row (at most RM
// entries, padded with zero coefficients) in registers for the whole run;
// RM = 0: rows stay in shared memory and threads loop over items.
template <int KIND, int RM>
__global__ void __launch_bounds__(kSmallThreads, 1) heom_small_rk4_kernel(SmallRk4Params p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HeomConsts &c = p.c;
  const int N = c.N, E = N * N, P = N * (N + 1) / 2;
  const long long M = c.M, ME = M * E, items = M * P;
  const int R = small_row_max(c);
  const int tid = threadIdx.x, nth = blockDim.x;
  double2 *Hs = reinterpret_cast<double2 *>(smem_raw);
  double2 *Y = Hs + E;
  double2 *ACC = Y + ME;
  double2 *X = ACC + ME;
  double2 *K = X + ME;
  double2 *coef = K + ME;                                 // items * R
  int *idx = reinterpret_cast<int *>(coef + items * R);   // items * R
  int *cnt = idx + items * R;                             // items
  for (int e = tid; e < E; e += nth) Hs[e] = c.H[e];
  for (long long e = tid; e < ME; e += nth) Y[e] = p.y[e];
  __syncthreads();
  for (long long u = tid; u < items; u += nth) {
    const long long n = u / P;
    const int q = (int)(u - n * P);
    cnt[u] = build_row<KIND>(c, Hs, n, __ldg(c.pair_i + q), __ldg(c.pair_j + q), idx + u * R, coef + u * R);
  }
  __syncthreads();
  // Register-resident row of this thread's item (RM > 0).
  int r_idx[RM > 0 ? RM : 1];
  double2 r_cf[RM > 0 ? RM : 1];
  int my_out0 = -1, my_out1 = -1;  // K offsets of the item and its mirror (-1: none)
  if (RM > 0) {
    const long long u = tid;
    const int nr = u < items ? cnt[u] : 0;
#pragma unroll
    for (int r = 0; r < RM; ++r) {
      r_idx[r] = r < nr ? idx[u * R + r] : 0;
      r_cf[r] = r < nr ? coef[u * R + r] : make_double2(0.0, 0.0);
    }
    if (u < items) {
      const long long n = u / P;
      const int q = (int)(u - n * P);
      const int i = __ldg(c.pair_i + q), j = __ldg(c.pair_j + q);
      my_out0 = (int)(n * E + i + j * N);
      my_out1 = i == j ? -1 : (int)(n * E + j + i * N);
    }
  }
  const double dt = p.dt;
  Rk4Ctl *rc = p.rk4;
  long long step = rc->step, nout = rc->nout;
  const long long out_factor = rc->out_factor, capacity = rc->capacity;
  for (long long it = 0; it < p.steps; ++it) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const double a = s == 2 ? dt : dt / 2;
      const double w = (s == 0 || s == 3) ? dt / 6 : dt / 3;
      if (RM > 0) {
        // One item per thread: the thread combines its own two elements
        // right away, and the stage inputs alternate between X and K (K
        // holds X_2), so a stage needs one barrier:
        //   stage 0: Y -> X,  1: X -> K,  2: K -> X,  3: X -> Y.
        const double2 *in = s == 0 ? Y : (s == 2 ? K : X);
        double2 *outb = s == 1 ? K : X;
        if (my_out0 >= 0) {
          double2 xv[RM > 0 ? RM : 1];
#pragma unroll
          for (int r = 0; r < RM; ++r) xv[r] = in[r_idx[r]];
          double2 v = make_double2(0.0, 0.0);
#pragma unroll
          for (int r = 0; r < RM; ++r) {
            v.x = fma(r_cf[r].x, xv[r].x, v.x);
            v.x = fma(-r_cf[r].y, xv[r].y, v.x);
            v.y = fma(r_cf[r].x, xv[r].y, v.y);
            v.y = fma(r_cf[r].y, xv[r].x, v.y);
          }
          if (my_out1 < 0) v.y = 0.0;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int e = h == 0 ? my_out0 : my_out1;
            if (e < 0) continue;
            const double2 kv = h == 0 ? v : s_conj(v);
            if (s == 0) {
              const double2 ys = Y[e];
              outb[e] = s_axpy(ys, kv, a);
              ACC[e] = s_axpy(ys, kv, w);
            } else if (s < 3) {
              outb[e] = s_axpy(Y[e], kv, a);
              ACC[e] = s_axpy(ACC[e], kv, w);
            } else {
              Y[e] = s_axpy(ACC[e], kv, w);
            }
          }
        }
        __syncthreads();
        continue;
      }
      const double2 *in = s == 0 ? Y : X;
      for (long long u = tid; u < items; u += nth) {
        const int *ri = idx + u * R;
        const double2 *rcf = coef + u * R;
        double2 v = make_double2(0.0, 0.0);
        for (int r = 0; r < cnt[u]; ++r) {
          const double2 cf = rcf[r], x = in[ri[r]];
          v.x = fma(cf.x, x.x, v.x);
          v.x = fma(-cf.y, x.y, v.x);
          v.y = fma(cf.x, x.y, v.y);
          v.y = fma(cf.y, x.x, v.y);
        }
        const long long n = u / P;
        const int q = (int)(u - n * P);
        const int i = __ldg(c.pair_i + q), j = __ldg(c.pair_j + q);
        if (i == j) {
          v.y = 0.0;
          K[n * E + i + j * N] = v;
        } else {
          K[n * E + i + j * N] = v;
          K[n * E + j + i * N] = s_conj(v);
        }
      }
      __syncthreads();
      for (long long e = tid; e < ME; e += nth) {
        const double2 kv = K[e];
        if (s == 0) {
          const double2 ys = Y[e];
          X[e] = s_axpy(ys, kv, a);
          ACC[e] = s_axpy(ys, kv, w);
        } else if (s < 3) {
          X[e] = s_axpy(Y[e], kv, a);
          ACC[e] = s_axpy(ACC[e], kv, w);
        } else {
          Y[e] = s_axpy(ACC[e], kv, w);
        }
      }
      __syncthreads();
    }
    // rho_0 row after step `step` when step % out_factor == 0 (:2858).
    if (out_factor > 0 && step % out_factor == 0) {
      if (p.traj && nout < capacity)
        for (int e = tid; e < E; e += nth) p.traj[nout * E + e] = Y[e];
      ++nout;
    }
    ++step;
  }
  for (long long e = tid; e < ME; e += nth) p.y[e] = Y[e];
  if (tid == 0) {
    rc->step = step;
    rc->nout = nout;
  }
}

size_t small_smem(const HeomConsts &c) {
  const size_t E = (size_t)c.N * c.N, items = (size_t)c.M * (c.N * (c.N + 1) / 2);
  const size_t R = (size_t)small_row_max(c);
  return (E + 4 * (size_t)c.M * E) * sizeof(double2) + items * R * (sizeof(double2) + sizeof(int)) +
         items * sizeof(int);
}

// Threads of the launch: enough for the larger of the item and element
// loops, in whole warps, at most kSmallThreads (fewer warps make the two
// barriers of a stage cheaper).
int small_threads(const HeomConsts &c) {
  const long long work = std::max<long long>(c.M * (c.N * (c.N + 1) / 2), c.M * c.N * c.N);
  const long long w = (work + 31) / 32 * 32;
  return (int)std::min<long long>(kSmallThreads, std::max<long long>(32, w));
}

// Register rows: the bound on a row's length, in buckets of 8 / 16
// entries, when every item has its own thread (0 otherwise).
int small_register_row(const HeomConsts &c) {
  const long long items = c.M * (c.N * (c.N + 1) / 2);
  const int r = small_row_max(c);
  if (items > kSmallThreads) return 0;
  return r <= 8 ? 8 : (r <= 16 ? 16 : 0);
}

template <int KIND, int RM>
cudaError_t launch_small_variant(const SmallRk4Params &p, size_t smem, int threads, cudaStream_t stream) {
  static int configured[kSmemLimitDevices] = {};
  cudaError_t e = raise_smem_limit(heom_small_rk4_kernel<KIND, RM>, smem, configured);
  if (e != cudaSuccess) return e;
  heom_small_rk4_kernel<KIND, RM><<<1, threads, smem, stream>>>(p);
  return cudaGetLastError();
}

template <int KIND>
cudaError_t launch_small_kind(const SmallRk4Params &p, size_t smem, cudaStream_t stream) {
  const HeomConsts &c = p.c;
  const int rm = small_register_row(c);
  if (rm > 0) {
    const int threads = small_threads(c);  // >= items: one item per thread
    if (rm == 8) return launch_small_variant<KIND, 8>(p, smem, threads, stream);
    return launch_small_variant<KIND, 16>(p, smem, threads, stream);
  }
  return launch_small_variant<KIND, 0>(p, smem, small_threads(c), stream);
}

}  // namespace

bool small_rk4_eligible(const HeomConsts &c) {
  if (c.kind != kIndependent && c.kind != kDiagonal) return false;
  // Problems the tiled kernel takes stay on it: a batch of such instances
  // is then bit-identical to each instance run alone.
  if (tile_kernel_available(c)) return false;
  if (c.filtered || c.time_local) return false;
  return (size_t)c.M * c.N * c.N <= kSmallMaxElements && small_smem(c) <= kSmallMaxSmem;
}

cudaError_t launch_small_rk4(const HeomConsts &c, double2 *y, double dt, long long steps, Rk4Ctl *rk4,
                             double2 *traj, cudaStream_t stream) {
  if (!small_rk4_eligible(c) || steps <= 0) return cudaErrorInvalidValue;
  SmallRk4Params p;
  p.c = c;
  p.y = y;
  p.dt = dt;
  p.steps = steps;
  p.rk4 = rk4;
  p.traj = traj;
  const size_t smem = small_smem(c);
  return c.kind == kIndependent ? launch_small_kind<kIndependent>(p, smem, stream)
                                : launch_small_kind<kDiagonal>(p, smem, stream);
}

}  // namespace phi
