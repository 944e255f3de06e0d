// heom_kernels.cu -- the per-node Liouvillian and the fused RK stage kernels.
//
// One "group" of GROUP threads owns one hierarchy node at a time; a 256-thread
// CTA holds 256/GROUP groups and walks the node range grid-stride.  Per node:
//
//   1. metadata: next/prev ids for every term, the multi-index n_t;
//   2. own ADO X_n -> shared memory (coalesced, node-major contiguous);
//      IndependentBath: column m = site(t) of every linked ADO -> shared memory
//      (a Hermitian ADO's row m is the conjugate of its column m, so the
//      neighbour terms of PHI's DoNext/DoPrevious, which touch row m and
//      column m, read only contiguous columns);
//   3. A = H X_n (the one complex N x N product of the node);
//   4. upper-triangle pairs (i <= j):
//        dX_ij = -i/hbar (A_ij - conj(A_ji))         (= -i/hbar [H, X]_ij)
//                - (dephasing_n + matsubara_ij) X_ij
//                + neighbour terms
//      and dX_ji = conj(dX_ij), so every output ADO is exactly Hermitian;
//   5. an epilogue that is the RK stage combine (RK4 / RKF45) or a plain store.
//
// Reference: HierarchyUpdater::Get and the IndependentBath / DiagonalBath /
// FullBath / Vacuum terms (hierarchy_updater.h:36-75,
// hierarchy_updater.cc:10-144, :216-254), the RK4 stage combines
// (hierarchy_integrator.cc:2705-2826) and the RKF45 combines, error and
// control (:2010-2482).
#include <cuda_runtime.h>

#include <cstdint>

#include "heom_device.cuh"
#include "heom_kernels.h"
#include "heom_tile.h"
#include "heom_tl_term.cuh"

namespace phi {
namespace {

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a + b * s for real s.
__device__ __forceinline__ double2 c_axpy(double2 a, double2 b, double s) {
  return make_double2(fma(b.x, s, a.x), fma(b.y, s, a.y));
}
// acc + i * s * b
__device__ __forceinline__ double2 c_add_i(double2 acc, double2 b, double s) {
  return make_double2(acc.x - s * b.y, acc.y + s * b.x);
}

template <int GROUP>
__device__ __forceinline__ void group_sync(int g) {
  if (GROUP == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(GROUP) : "memory");
  }
}

// Shared-memory plan (doubles of complex = 16 B units).
struct SmemPlan {
  int E;         // N*N
  int gcols;     // 2*T*N (independent) or 2*N*N (diagonal/full scratch)
  int per_group; // complex slots per group
  int ints_per_group;
};

__host__ __device__ inline SmemPlan smem_plan(int N, int T, int kind) {
  SmemPlan p;
  p.E = N * N;
  p.gcols = kind == kIndependent ? 2 * T * N : 2 * N * N;
  p.per_group = 3 * p.E + p.gcols;
  // ids[2T], nts[T], then three 8-byte slots at an even int offset (the
  // node's dephasing rate, its max |y|^2 when filtering, and whether it is
  // in the deepest tier, for time-local truncation).
  p.ints_per_group = ((3 * T + 1) & ~1) + 6;
  return p;
}

struct StageParams {
  HeomConsts c;
  int mode;          // StageMode
  int stage;         // RK stage index
  const double2 *x;  // stage input (node-major)
  double2 *out;      // apply output / next stage input
  // RK4
  double2 *y;
  double2 *acc;
  double a_next;     // X_{s+1} = y + a_next * k
  double w_acc;      // accumulator weight
  Rk4Ctl *rk4;
  double2 *traj;
  // RKF45
  double2 *k[5];
  double2 *ybuf[2];
  Rkf45Ctl *ctl;
  // filtering (see StageLaunch)
  uint8_t *act[2];
  int act_par;
  // apply mode, gridDim.y > 1: block row y applies to x + y * x_bstride and
  // writes out + y * out_bstride (many inputs of one operator per launch)
  long long x_bstride, out_bstride;
};

template <int GROUP, int KIND>
__global__ void __launch_bounds__(256) heom_stage_kernel(StageParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HeomConsts &c = p.c;
  const int N = c.N, E = N * N, T = c.T;
  constexpr int NG = 256 / GROUP;
  const int g = threadIdx.x / GROUP, lane = threadIdx.x % GROUP;

  const SmemPlan plan = smem_plan(N, T, KIND);
  double2 *Hs = reinterpret_cast<double2 *>(smem_raw);
  double2 *Xs = Hs + E + (size_t)g * plan.per_group;
  double2 *As = Xs + E;
  double2 *Us = As + E;
  double2 *Gs = Us + E;
  double *coef_s = reinterpret_cast<double *>(Hs + E + (size_t)NG * plan.per_group);
  int *ids = reinterpret_cast<int *>(coef_s + 32) + (size_t)g * plan.ints_per_group;
  int *nts = ids + 2 * T;
  double *deph_s = reinterpret_cast<double *>(ids + ((3 * T + 1) & ~1));  // 8-byte aligned
  unsigned long long *nmax_s = reinterpret_cast<unsigned long long *>(deph_s + 1);
  int *tlf_s = reinterpret_cast<int *>(nmax_s + 1);

  int ycur = 0;
  if (p.mode == kModeRkf45) {
    if (*(volatile int *)&p.ctl->done) return;  // uniform for the whole grid
    ycur = p.ctl->ycur;
    for (int i = threadIdx.x; i < 24; i += blockDim.x) coef_s[i] = p.ctl->coef[i];
  }
  for (int i = threadIdx.x; i < E; i += blockDim.x) Hs[i] = c.H[i];
  __syncthreads();

  const double ih = c.inv_hbar;
  double emax = 0.0;
  // RKF45 stage 0 reads the current state, whose buffer only the device knows.
  if (gridDim.y > 1) {
    p.x += blockIdx.y * p.x_bstride;
    p.out += blockIdx.y * p.out_bstride;
  }
  const double2 *xin = (p.mode == kModeRkf45 && p.stage == 0) ? p.ybuf[ycur] : p.x;
  const double2 *yin = p.mode == kModeRkf45 ? p.ybuf[ycur] : p.y;
  // Filtering: flags of the current state, and of the state this launch
  // writes (RK4 stage 3, RKF45 stage 5 -- the candidate, kept on accept).
  const uint8_t *act_in = nullptr;
  uint8_t *act_out = nullptr;
  if (c.filtered) {
    const int ap = p.mode == kModeRkf45 ? ycur : p.act_par;
    act_in = p.act[ap];
    act_out = p.act[ap ^ 1];
  }
  const bool flag_stage = act_in && act_out &&
                          ((p.mode == kModeRk4 && p.stage == 3) || (p.mode == kModeRkf45 && p.stage == 5));

  for (long long n = (long long)blockIdx.x * NG + g; n < c.M; n += (long long)gridDim.x * NG) {
    // 1. metadata
    for (int s = lane; s < 2 * T; s += GROUP) {
      const int id = s < T ? __ldg(c.next + n * T + s) : __ldg(c.prev + n * T + (s - T));
      // an inactive neighbour contributes nothing (hierarchy_updater.cc:256-303)
      ids[s] = (id >= 0 && act_in && !__ldg(act_in + id)) ? -1 : id;
    }
    for (int t = lane; t < T; t += GROUP) nts[t] = __ldg(c.mi + n * T + t);
    // 2. own ADO
    const double2 *xn = xin + n * E;
    for (int e = lane; e < E; e += GROUP) Xs[e] = __ldg(xn + e);
    group_sync<GROUP>(g);
    if (lane == 0) {
      double d = 0.0;
      for (int t = 0; t < T; ++t) d += nts[t] * __ldg(c.nu + t);
      deph_s[0] = d;
      nmax_s[0] = 0ull;
      int tier = 0;
      for (int t = 0; t < T; ++t) tier += nts[t];
      tlf_s[0] = c.time_local && tier == c.L;
    }
    if (KIND == kIndependent && !c.vacuum) {
      for (int idx = lane; idx < 2 * T * N; idx += GROUP) {
        const int s = idx / N, k = idx - s * N;
        const int id = ids[s];
        if (id >= 0) {
          const int t = s < T ? s : s - T;
          const int m = __ldg(c.term_site + t);
          Gs[idx] = __ldg(xin + (long long)id * E + k + m * N);
        }
      }
    }
    // 3. A = H X
    for (int e = lane; e < E; e += GROUP) {
      const int i = e % N, j = e / N;
      double2 a = make_double2(0.0, 0.0);
      for (int k = 0; k < N; ++k) {
        const double2 h = Hs[i + k * N], x = Xs[k + j * N];
        a.x = fma(h.x, x.x, a.x);
        a.x = fma(-h.y, x.y, a.x);
        a.y = fma(h.x, x.y, a.y);
        a.y = fma(h.y, x.x, a.y);
      }
      As[e] = a;
    }
    if (KIND != kIndependent) {
      // Neighbour (and, for FullBath, Matsubara) terms into Gs[0..E) per element.
      double2 *NB = Gs;
      double2 *W = Gs + E;  // work matrix
      for (int e = lane; e < E; e += GROUP) NB[e] = make_double2(0.0, 0.0);
      group_sync<GROUP>(g);
      if (!c.vacuum) {
        if (KIND == kFull) {
          // -Delta_b [V_b, [V_b, X]]  (FullBath::DoMatsubara, hierarchy_updater.cc:10-25)
          for (int b = 0; b < c.nb; ++b) {
            const double *V = c.bath_V + (size_t)b * E;
            for (int e = lane; e < E; e += GROUP) {
              const int i = e % N, j = e / N;
              double2 w = make_double2(0.0, 0.0);
              for (int k = 0; k < N; ++k) {
                w = c_axpy(w, Xs[k + j * N], __ldg(V + i + k * N));
                w = c_axpy(w, Xs[i + k * N], -__ldg(V + k + j * N));
              }
              W[e] = w;
            }
            group_sync<GROUP>(g);
            const double dlt = __ldg(c.mats_bath + b);
            for (int e = lane; e < E; e += GROUP) {
              const int i = e % N, j = e / N;
              double2 w = make_double2(0.0, 0.0);
              for (int k = 0; k < N; ++k) {
                w = c_axpy(w, W[k + j * N], __ldg(V + i + k * N));
                w = c_axpy(w, W[i + k * N], -__ldg(V + k + j * N));
              }
              NB[e] = c_axpy(NB[e], w, -dlt);
            }
            group_sync<GROUP>(g);
          }
        }
        for (int s = 0; s < 2 * T; ++s) {
          const int id = ids[s];
          if (id < 0) continue;
          const bool is_next = s < T;
          const int t = is_next ? s : s - T;
          const int b = __ldg(c.term_site + t);
          const int nt = nts[t];
          const double2 *xo = xin + (long long)id * E;
          if (KIND == kDiagonal) {
            // DiagonalBath::DoNext / DoPrevious (hierarchy_updater.cc:105-127):
            // next: -i (V_i - V_j) X+_ij ; prev: n_t (-i)(c V_i - c^* V_j) X-_ij
            const double *V = c.bath_V + (size_t)b * N;
            const double2 ct = __ldg(c.corr + t);
            for (int e = lane; e < E; e += GROUP) {
              const int i = e % N, j = e / N;
              const double2 xv = __ldg(xo + e);
              const double vi = __ldg(V + i), vj = __ldg(V + j);
              double2 f;
              if (is_next) {
                f = make_double2(0.0, -(vi - vj));
              } else {
                // -i (c vi - conj(c) vj) * n_t
                const double re = ct.x * vi - ct.x * vj;
                const double im = ct.y * vi + ct.y * vj;
                f = make_double2(im * nt, -re * nt);
              }
              NB[e] = c_add(NB[e], c_mul(f, xv));
            }
          } else {
            // FullBath::DoNext: -p V X+ + p X+ V, p = i s;
            // FullBath::DoPrevious: -pr V X- - pc X- V (hierarchy_updater.cc:46-82)
            const double *V = c.bath_V + (size_t)b * E;
            for (int e = lane; e < E; e += GROUP) W[e] = __ldg(xo + e);
            group_sync<GROUP>(g);
            double2 pl, pr;
            if (is_next) {
              const double sn = __ldg(c.sq_next + t * (c.L + 2) + nt);
              pl = make_double2(0.0, -sn);  // -p
              pr = make_double2(0.0, sn);   // +p
            } else {
              const double sp = __ldg(c.sq_prev + t * (c.L + 2) + nt);
              const double2 ct = __ldg(c.corr + t);
              pl = make_double2(ct.y * sp, -ct.x * sp);   // -pr = -i c sp
              pr = make_double2(ct.y * sp, ct.x * sp);    // -pc = i conj(c) sp
            }
            for (int e = lane; e < E; e += GROUP) {
              const int i = e % N, j = e / N;
              double2 vx = make_double2(0.0, 0.0), xv = make_double2(0.0, 0.0);
              for (int k = 0; k < N; ++k) {
                vx = c_axpy(vx, W[k + j * N], __ldg(V + i + k * N));
                xv = c_axpy(xv, W[i + k * N], __ldg(V + k + j * N));
              }
              NB[e] = c_add(NB[e], c_add(c_mul(pl, vx), c_mul(pr, xv)));
            }
            group_sync<GROUP>(g);
          }
        }
        if (tlf_s[0]) {
          // Time-local truncation on the deepest tier, DiagonalBath /
          // FullBath::DoTimelocal (hierarchy_updater.cc:28-44, :93-104):
          // W = Q_b X - X Q_b^+, then -[V_b, W] for every bath b.
          for (int b = 0; b < c.nb; ++b) {
            const double2 *Q = c.tl_q + (size_t)b * E;
            group_sync<GROUP>(g);  // W is reused
            for (int e = lane; e < E; e += GROUP) {
              const int i = e % N, j = e / N;
              double2 w = make_double2(0.0, 0.0);
              for (int k = 0; k < N; ++k) {
                w = c_add(w, c_mul(__ldg(Q + i + k * N), Xs[k + j * N]));
                w = c_sub(w, c_mul(Xs[i + k * N], c_conj(__ldg(Q + j + k * N))));
              }
              W[e] = w;
            }
            group_sync<GROUP>(g);
            if (KIND == kDiagonal) {
              const double *V = c.bath_V + (size_t)b * N;
              for (int e = lane; e < E; e += GROUP) {
                const int i = e % N, j = e / N;
                NB[e] = c_axpy(NB[e], W[e], -(__ldg(V + i) - __ldg(V + j)));
              }
            } else {
              const double *V = c.bath_V + (size_t)b * E;
              for (int e = lane; e < E; e += GROUP) {
                const int i = e % N, j = e / N;
                double2 vw = make_double2(0.0, 0.0);
                for (int k = 0; k < N; ++k) {
                  vw = c_axpy(vw, W[k + j * N], __ldg(V + i + k * N));
                  vw = c_axpy(vw, W[i + k * N], -__ldg(V + k + j * N));
                }
                NB[e] = c_sub(NB[e], vw);
              }
            }
          }
        }
      }
    }
    group_sync<GROUP>(g);

    // 4. upper-triangle pairs
    const double deph = deph_s[0];
    const bool tl_node = tlf_s[0] != 0;
    const int npairs = N * (N + 1) / 2;
    for (int u = lane; u < npairs; u += GROUP) {
      const int i = __ldg(c.pair_i + u), j = __ldg(c.pair_j + u);
      const double2 aij = As[i + j * N], aji = As[j + i * N];
      double2 v = make_double2((aij.y + aji.y) * ih, -(aij.x - aji.x) * ih);
      const double2 xij = Xs[i + j * N];
      if (!c.vacuum) {
        const double fac = deph + __ldg(c.mats_elem + i + j * N);
        v = c_axpy(v, xij, -fac);
        if (KIND == kIndependent && tl_node && i != j) v = c_add(v, tl_pair_term<double2>(Xs, c.tl_q, N, i, j));
        if (KIND == kIndependent) {
          if (i != j) {
            for (int q = __ldg(c.site_ptr + j); q < __ldg(c.site_ptr + j + 1); ++q) {
              const int t = __ldg(c.site_terms + q);
              const int nt = nts[t];
              if (ids[t] >= 0) {  // + p X+_ij, p = i sqrt((n+1)|c|)
                v = c_add_i(v, Gs[t * N + i], __ldg(c.sq_next + t * (c.L + 2) + nt));
              }
              if (ids[T + t] >= 0) {  // - pc X-_ij = i conj(c) sp X-_ij
                const double sp = __ldg(c.sq_prev + t * (c.L + 2) + nt);
                const double2 ct = __ldg(c.corr + t);
                v = c_add_i(v, c_mul(c_conj(ct), Gs[(T + t) * N + i]), sp);
              }
            }
            for (int q = __ldg(c.site_ptr + i); q < __ldg(c.site_ptr + i + 1); ++q) {
              const int t = __ldg(c.site_terms + q);
              const int nt = nts[t];
              if (ids[t] >= 0) {  // - p X+_ij, X+_ij = conj(X+_ji)
                v = c_add_i(v, c_conj(Gs[t * N + j]), -__ldg(c.sq_next + t * (c.L + 2) + nt));
              }
              if (ids[T + t] >= 0) {  // - pr X-_ij = -i c sp X-_ij
                const double sp = __ldg(c.sq_prev + t * (c.L + 2) + nt);
                const double2 ct = __ldg(c.corr + t);
                v = c_add_i(v, c_mul(ct, c_conj(Gs[(T + t) * N + j])), -sp);
              }
            }
          } else {
            // diagonal (m, m): next terms cancel; prev gives -(pc + pr) X-_mm
            //   = 2 sp Im(c) X-_mm
            for (int q = __ldg(c.site_ptr + i); q < __ldg(c.site_ptr + i + 1); ++q) {
              const int t = __ldg(c.site_terms + q);
              if (ids[T + t] >= 0) {
                const double sp = __ldg(c.sq_prev + t * (c.L + 2) + nts[t]);
                const double2 ct = __ldg(c.corr + t);
                v.x = fma(2.0 * sp * ct.y, Gs[(T + t) * N + i].x, v.x);
              }
            }
          }
        } else {
          v = c_add(v, Gs[i + j * N]);
        }
      }
      if (i == j) {
        v.y = 0.0;
        Us[i + j * N] = v;
      } else {
        Us[i + j * N] = v;
        Us[j + i * N] = c_conj(v);
      }
    }
    group_sync<GROUP>(g);

    // 5. epilogue
    const long long base = n * E;
    double fl_m = 0.0;  // filtering: max |y_new|^2 of this lane's elements
    if (p.mode == kModeApply) {
      for (int e = lane; e < E; e += GROUP) p.out[base + e] = Us[e];
    } else if (p.mode == kModeRk4) {
      const int s = p.stage;
      for (int e = lane; e < E; e += GROUP) {
        const double2 kv = Us[e];
        if (s == 0) {
          const double2 ys = Xs[e];
          p.out[base + e] = c_axpy(ys, kv, p.a_next);
          p.acc[base + e] = c_axpy(ys, kv, p.w_acc);
        } else if (s < 3) {
          const double2 ys = __ldg(p.y + base + e);
          p.out[base + e] = c_axpy(ys, kv, p.a_next);
          p.acc[base + e] = c_axpy(p.acc[base + e], kv, p.w_acc);
        } else {
          const double2 yn = c_axpy(p.acc[base + e], kv, p.w_acc);
          p.y[base + e] = yn;
          const double m2 = fma(yn.x, yn.x, yn.y * yn.y);
          fl_m = m2 > fl_m ? m2 : fl_m;
          if (n == 0 && p.traj) Xs[e] = yn;
        }
      }
      if (n == 0 && p.stage == 3 && p.traj) {
        group_sync<GROUP>(g);
        Rk4Ctl *rc = p.rk4;
        const long long step = rc->step;
        if (rc->out_factor > 0 && step % rc->out_factor == 0) {
          const long long row = rc->nout;
          if (row < rc->capacity)
            for (int e = lane; e < E; e += GROUP) p.traj[row * E + e] = Xs[e];
        }
        group_sync<GROUP>(g);
        if (lane == 0) {
          if (rc->out_factor > 0 && step % rc->out_factor == 0) rc->nout = rc->nout + 1;
          rc->step = step + 1;
        }
      }
    } else {  // RKF45
      const int s = p.stage;
      const double *cf = coef_s;
      for (int e = lane; e < E; e += GROUP) {
        const double2 kv = Us[e];
        const double2 ys = s == 0 ? Xs[e] : __ldg(yin + base + e);
        if (s < 5) {
          if (s < 5) p.k[s][base + e] = kv;
          // X_{s+1} = y + sum_{r<=s} b_{s+1,r} k_r  (left to right, as :2015-2200)
          const int row = s * (s + 1) / 2;
          double2 xv = ys;
          for (int r = 0; r < s; ++r) xv = c_axpy(xv, __ldg(p.k[r] + base + e), cf[row + r]);
          xv = c_axpy(xv, kv, cf[row + s]);
          p.out[base + e] = xv;
        } else {
          const double2 k0 = __ldg(p.k[0] + base + e), k2 = __ldg(p.k[2] + base + e);
          const double2 k3 = __ldg(p.k[3] + base + e), k4 = __ldg(p.k[4] + base + e);
          double2 y4 = c_axpy(ys, k0, cf[15]);
          y4 = c_axpy(y4, k2, cf[16]);
          y4 = c_axpy(y4, k3, cf[17]);
          y4 = c_axpy(y4, k4, cf[18]);
          double2 y5 = c_axpy(ys, k0, cf[19]);
          y5 = c_axpy(y5, k2, cf[20]);
          y5 = c_axpy(y5, k3, cf[21]);
          y5 = c_axpy(y5, k4, cf[22]);
          y5 = c_axpy(y5, kv, cf[23]);
          p.ybuf[ycur ^ 1][base + e] = y5;
          const double m2 = fma(y5.x, y5.x, y5.y * y5.y);
          fl_m = m2 > fl_m ? m2 : fl_m;
          const double err = hypot(y4.x - y5.x, y4.y - y5.y);
          emax = (err > emax || err != err) ? err : emax;
        }
      }
    }
    if (flag_stage) {
      // New flags of the state just written (hierarchy_integrator.cc:2827-2850,
      // :2359-2384): below the tolerance -> inactive, above -> active, equal
      // -> unchanged.  A NaN never wins the `>` above, as in PHI's scan.
      if (fl_m > 0.0) atomicMax(nmax_s, (unsigned long long)__double_as_longlong(fl_m));
      group_sync<GROUP>(g);
      if (lane == 0) {
        const double mx = sqrt(__longlong_as_double((long long)nmax_s[0]));
        const uint8_t old = act_in[n];
        act_out[n] = mx < c.filter_tol ? (uint8_t)0 : (mx > c.filter_tol ? (uint8_t)1 : old);
      }
    }
    group_sync<GROUP>(g);
  }

  if (p.mode == kModeRkf45 && p.stage == 5) {
    // max-reduce |y4 - y5| (hierarchy_integrator.cc:2317-2351); the bit
    // pattern of a non-negative double orders like the value (NaN above inf).
    unsigned long long bits = (unsigned long long)__double_as_longlong(emax);
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
      bits = o > bits ? o : bits;
    }
    // one atomic per CTA (every CTA updates the same error word)
    __shared__ unsigned long long wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = bits;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long m = wmax[0];
      for (int w = 1; w < 8; ++w) m = wmax[w] > m ? wmax[w] : m;
      if (m) atomicMax(&p.ctl->err_bits, m);
    }
  }
}

// Accept/reject and step-size control of Rkf45Integrate
// (hierarchy_integrator.cc:2355-2482), one thread.  The accept test uses the
// step size the attempt was made with.
__global__ void rkf45_control_kernel(Rkf45Ctl *ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) {
    ctl->tl_pending = 0;
    return;
  }
  ctl->tl_pending = 0;
  const double err = __longlong_as_double((long long)ctl->err_bits);
  ctl->err_bits = 0ull;
  const long long attempt = ctl->steps;
  if (ctl->err_trace && attempt < ctl->trace_cap) ctl->err_trace[attempt] = err;
  ctl->steps += 1;
  if (!(err == err) || err > 1.0e300) {
    ctl->nonfinite = 1;
    ctl->done = 1;
    ctl->status = 2;
    return;
  }
  bool accept = err < ctl->tol || ctl->dt * ctl->dtdn < ctl->min_dt;
  bool grow = err < ctl->tol / 10;
  if (ctl->forced && attempt < ctl->forced_len) {
    accept = ctl->forced[attempt] != 0;
    grow = ctl->forced[attempt] == 2;
  }
  if (accept) {
    // Time-local matrices advance by the rest of this attempt (dt - a5).
    ctl->tl_h_accept = ctl->dt - ctl->a[4];
    ctl->tl_pending = 1;
    ctl->ycur ^= 1;
    ctl->time += ctl->dt;
    ctl->accepted += 1;
    if (err > ctl->max_error) ctl->max_error = err;
    bool update = grow;
    if (ctl->time + ctl->dt > ctl->end_time) {
      update = true;
      ctl->dtup = (ctl->end_time - ctl->time) / ctl->dt;
    }
    if (update) {
      ctl->dt *= ctl->dtup;
      for (int q = 0; q < 24; ++q) ctl->coef[q] *= ctl->dtup;
      for (int q = 0; q < 5; ++q) ctl->a[q] *= ctl->dtup;
    }
  } else {
    ctl->dt *= ctl->dtdn;
    for (int q = 0; q < 24; ++q) ctl->coef[q] *= ctl->dtdn;
    for (int q = 0; q < 5; ++q) ctl->a[q] *= ctl->dtdn;
    ctl->tl_pending = 2;
  }
  if (!(ctl->time < ctl->end_time)) ctl->done = 1;
  if (!ctl->done && ctl->steps >= ctl->max_steps) {
    ctl->done = 1;
    ctl->status = 1;
  }
}

template <int GROUP, int KIND>
cudaError_t launch_group(const StageParams &p, size_t smem, int grid, int batch, cudaStream_t stream) {
  auto kern = heom_stage_kernel<GROUP, KIND>;
  static thread_local int configured[kSmemLimitDevices] = {};
  cudaError_t e = raise_smem_limit(kern, smem, configured);
  if (e != cudaSuccess) return e;
  kern<<<dim3(grid, batch), 256, smem, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace

int choose_group(int N) {
  if (N <= 11) return 32;
  if (N <= 22) return 128;
  return 256;
}

size_t stage_smem_bytes(int N, int T, int kind) {
  const SmemPlan plan = smem_plan(N, T, kind);
  const int NG = 256 / choose_group(N);
  size_t bytes = (size_t)(plan.E + (size_t)NG * plan.per_group) * sizeof(double2);
  bytes += 32 * sizeof(double);
  bytes += (size_t)NG * plan.ints_per_group * sizeof(int);
  return bytes + 16;
}

int stage_grid(const HeomConsts &c, int num_sms) {
  const int NG = 256 / choose_group(c.N);
  long long need = (c.M + NG - 1) / NG;
  const size_t smem = stage_smem_bytes(c.N, c.T, c.kind);
  int per_sm = (int)((200 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 8) per_sm = 8;
  long long cap = (long long)num_sms * per_sm;
  if (need > cap) need = cap;
  if (need < 1) need = 1;
  return (int)need;
}

cudaError_t launch_stage(const StageLaunch &L, cudaStream_t stream) {
  if (!L.generic && tile_kernel_available(L.c)) {
    if (L.xv || L.outv || L.mixed) return launch_tile_stage(L, stream);
    StageLaunch T = L;  // complex128 caller: the typed pointers are the storage
    T.xv = L.x;
    T.outv = L.out;
    for (int i = 0; i < 5; ++i) T.kv[i] = L.k[i];
    return launch_tile_stage(T, stream);
  }
  if (L.mixed) return cudaErrorInvalidValue;  // mixed precision needs the tiled kernel
  StageParams p;
  p.c = L.c;
  p.mode = L.mode;
  p.stage = L.stage;
  p.x = L.x;
  p.out = L.out;
  p.y = L.y;
  p.acc = L.acc;
  p.a_next = L.a_next;
  p.w_acc = L.w_acc;
  p.rk4 = L.rk4;
  p.traj = L.traj;
  for (int i = 0; i < 5; ++i) p.k[i] = L.k[i];
  p.ybuf[0] = L.ybuf[0];
  p.ybuf[1] = L.ybuf[1];
  p.ctl = L.ctl;
  p.act[0] = L.act[0];
  p.act[1] = L.act[1];
  p.act_par = L.act_par;
  p.x_bstride = L.x_bstride;
  p.out_bstride = L.out_bstride;
  const int batch = L.batch;
  if (batch < 1 || batch > 65535 || (batch > 1 && L.mode != kModeApply)) return cudaErrorInvalidValue;
  const size_t smem = stage_smem_bytes(L.c.N, L.c.T, L.c.kind);
  const int grid = L.grid;
  const int group = choose_group(L.c.N);
#define PHI_DISPATCH(G)                                                      \
  switch (L.c.kind) {                                                        \
    case kIndependent: return launch_group<G, kIndependent>(p, smem, grid, batch, stream); \
    case kDiagonal: return launch_group<G, kDiagonal>(p, smem, grid, batch, stream); \
    default: return launch_group<G, kFull>(p, smem, grid, batch, stream); \
  }
  if (group == 32) {
    PHI_DISPATCH(32)
  } else if (group == 128) {
    PHI_DISPATCH(128)
  } else {
    PHI_DISPATCH(256)
  }
#undef PHI_DISPATCH
}

namespace {
__global__ void to_c64_kernel(const double2 *in, float2 *out, long long M, int E, int EP) {
  const long long total = M * EP;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / EP;
    const int w = (int)(i - n * EP);
    const double2 v = w < E ? in[n * E + w] : make_double2(0.0, 0.0);
    out[i] = make_float2((float)v.x, (float)v.y);
  }
}
__global__ void to_c128_kernel(const float2 *in, double2 *out, long long M, int E, int EP) {
  const long long total = M * E;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / E;
    const int w = (int)(i - n * E);
    const float2 v = in[n * EP + w];
    out[i] = make_double2(v.x, v.y);
  }
}
int conv_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}
}  // namespace

cudaError_t launch_to_c64(const double2 *in, float2 *out, long long M, int E, int padded, cudaStream_t s) {
  to_c64_kernel<<<conv_blocks(M * padded), 256, 0, s>>>(in, out, M, E, padded);
  return cudaGetLastError();
}

cudaError_t launch_to_c128(const float2 *in, double2 *out, long long M, int E, int padded, cudaStream_t s) {
  to_c128_kernel<<<conv_blocks(M * E), 256, 0, s>>>(in, out, M, E, padded);
  return cudaGetLastError();
}

cudaError_t launch_rkf45_control(Rkf45Ctl *ctl, cudaStream_t stream) {
  rkf45_control_kernel<<<1, 32, 0, stream>>>(ctl);
  return cudaGetLastError();
}

}  // namespace phi
