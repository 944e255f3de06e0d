// heom_timelocal.cu -- the time-local truncation matrices on the device.
//
// PHI's time-local truncation (use_time_local_truncation) keeps, for every
// bath m and correlation term k, an N x N matrix Q_{m,k}, and their sums
// Q_m = sum_k Q_{m,k}, which the deepest tier of the hierarchy reads
// (IndependentBath::DoTimelocal, hierarchy_updater.cc:171-190).  The
// integrator advances them along its stage times
// (UpdateTimeLocalTruncation, hierarchy_integrator.cc:1675-1693): for a step
// of h, with PHI's first-order propagator U = I - i H h (FillPropagator,
// hierarchy.cc:229-237; the Hamiltonian as stored, without 1/hbar),
//
//   Q_{m,k} <- d_k U^+ (Q_{m,k} + h c_{m,k} |m><m|) U,
//   d_0 = exp(-gamma_m h), d_k = exp(-nu k h)   (hierarchy.cc:264-341),
//
// skipped when h < 1e-9.  RKF45 also keeps stored copies, restored before
// its last stage and after a rejected step and refreshed after an accepted
// one (:1695-1733, :2246-2247, :2388-2389, :2479).
//
// One CTA per bath: H, Q_{m,k} and the intermediate product sit in shared
// memory (3 N^2 complex, at most 192 KiB for N = 64); every element is
// written by the thread that reads it in the next product only after a
// barrier.  The work is O(nb K N^3) per update, microseconds beside a stage.
#include <cuda_runtime.h>

#include "heom_timelocal.h"

namespace phi {
namespace {

constexpr int kTlThreads = 256;
constexpr double kTlMinStep = 1e-9;  // UpdateTimeLocalTruncation skips smaller steps

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(kTlThreads) tl_kernel(TlLaunch p) {
  extern __shared__ __align__(16) double2 tl_smem[];
  const HeomConsts &c = p.c;
  const int N = c.N, E = N * N, K1 = c.K1, m = blockIdx.x, tid = threadIdx.x;
  double h = p.h;
  bool restore = false, store = false;
  if (p.op == kTlRkf45Stage) {
    const Rkf45Ctl *ctl = p.ctl;
    if (*(volatile const int *)&ctl->done) return;  // uniform for the grid
    const double *a = ctl->a;
    switch (p.stage) {
      case 1: h = a[0]; break;
      case 2: h = a[1] - a[0]; break;
      case 3: h = a[2] - a[1]; break;
      case 4: h = a[3] - a[2]; break;
      default: h = a[4]; restore = true; break;  // stage 5 restarts from the stored copy
    }
  } else if (p.op == kTlRkf45Post) {
    const int pend = *(volatile const int *)&p.ctl->tl_pending;
    if (pend == 0) return;
    if (pend == 2) {
      restore = true;
      h = 0.0;
    } else {
      h = p.ctl->tl_h_accept;
      store = true;
    }
  }
  double2 *qk = p.qk + (size_t)m * K1 * E;
  double2 *qk_st = p.qk_st + (size_t)m * K1 * E;
  double2 *q = p.q + (size_t)m * E;
  double2 *q_st = p.q_st + (size_t)m * E;
  if (restore) {
    for (int e = tid; e < K1 * E; e += kTlThreads) qk[e] = qk_st[e];
    for (int e = tid; e < E; e += kTlThreads) q[e] = q_st[e];
    __syncthreads();  // the advance reads these elements from other threads
  }
  if (h >= kTlMinStep) {
    double2 *Hs = tl_smem, *Qs = Hs + E, *Ts = Qs + E;
    for (int e = tid; e < E; e += kTlThreads) Hs[e] = c.H[e];
    for (int k = 0; k < K1; ++k) {
      const int t = m * K1 + k;
      for (int e = tid; e < E; e += kTlThreads) Qs[e] = qk[(size_t)k * E + e];
      __syncthreads();
      // + h c_{m,k} times the bath operator: |m><m| for independent baths,
      // diag(V_m) for diagonal ones, V_m for full ones (AddIndependent /
      // AddDiagonal / AddFullBathOperator, hierarchy.cc:218-233, :289-300).
      const double2 ct = c.corr[t];
      if (c.kind == kDiagonal) {
        for (int d = tid; d < N; d += kTlThreads) {
          const double v = c.bath_V[(size_t)m * N + d];
          Qs[d + d * N].x += h * ct.x * v;
          Qs[d + d * N].y += h * ct.y * v;
        }
      } else if (c.kind == kFull) {
        for (int e = tid; e < E; e += kTlThreads) {
          const double v = c.bath_V[(size_t)m * E + e];
          Qs[e].x = fma(h * ct.x, v, Qs[e].x);
          Qs[e].y = fma(h * ct.y, v, Qs[e].y);
        }
      } else if (tid == 0) {
        Qs[m + m * N].x += h * ct.x;
        Qs[m + m * N].y += h * ct.y;
      }
      __syncthreads();
      const double damp = exp(-c.nu[t] * h);
      // T = d U^+ Q with U^+[i][n] = conj(U[n][i]) = delta + i h conj(H[n][i]).
      for (int e = tid; e < E; e += kTlThreads) {
        const int i = e % N, j = e / N;
        double2 acc = make_double2(0.0, 0.0);
        for (int n = 0; n < N; ++n) {
          const double2 hn = Hs[n + i * N];
          const double2 ua = make_double2((n == i ? 1.0 : 0.0) + h * hn.y, h * hn.x);
          const double2 pr = cmul(ua, Qs[n + j * N]);
          acc.x += pr.x;
          acc.y += pr.y;
        }
        Ts[e] = make_double2(damp * acc.x, damp * acc.y);
      }
      __syncthreads();
      // Q = T U with U[n][j] = delta - i h H[n][j]; Q_m accumulates over k.
      for (int e = tid; e < E; e += kTlThreads) {
        const int i = e % N, j = e / N;
        double2 acc = make_double2(0.0, 0.0);
        for (int n = 0; n < N; ++n) {
          const double2 hn = Hs[n + j * N];
          const double2 u = make_double2((n == j ? 1.0 : 0.0) + h * hn.y, -h * hn.x);
          const double2 pr = cmul(Ts[i + n * N], u);
          acc.x += pr.x;
          acc.y += pr.y;
        }
        qk[(size_t)k * E + e] = acc;
        if (k == 0) {
          q[e] = acc;
        } else {
          const double2 s = q[e];  // written by this thread at k - 1
          q[e] = make_double2(s.x + acc.x, s.y + acc.y);
        }
      }
      __syncthreads();  // Qs / Ts are reused by the next term
    }
  }
  if (store) {
    for (int e = tid; e < K1 * E; e += kTlThreads) qk_st[e] = qk[e];
    for (int e = tid; e < E; e += kTlThreads) q_st[e] = q[e];
  }
}

}  // namespace

size_t tl_smem_bytes(int N) { return (size_t)3 * N * N * sizeof(double2); }

cudaError_t launch_tl(const TlLaunch &p, cudaStream_t stream) {
  const size_t smem = tl_smem_bytes(p.c.N);
  static thread_local int configured[kSmemLimitDevices] = {};
  cudaError_t e = raise_smem_limit(tl_kernel, smem, configured);
  if (e != cudaSuccess) return e;
  tl_kernel<<<p.c.nb, kTlThreads, smem, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace phi
