// heom_bicgstab.cu -- steady state of the hierarchy by BiCGSTAB(ell) on the
// device.
//
// The reference solves L x = 0 for the whole hierarchy with the system
// element rho_0[0,0] eliminated (PrepForSteadyState, BicgstabLSteadyState,
// BicgstabSteadyState; hierarchy_integrator.cc:1471-1613, :3112-3441,
// :3495-3783): x_0[0,0] is fixed to 1, the equation of element (0,0) of node 0
// is dropped (trace conservation implies it), the right-hand side is minus the
// column of L that multiplies x_0[0,0], and the result is divided by
// tr rho_0.  Here that system is
//
//   A x = L(x)  with output element (0,0) of node 0 set to zero,
//   b   = -L(E00) with element (0,0) of node 0 set to zero,
//
// and every Krylov vector keeps element (0,0) of node 0 at zero.  Every ADO
// of PHI's hierarchy is Hermitian and A maps Hermitian states to Hermitian
// states, so the inner products sum_ij conj(a_ij) b_ij are real: the method
// runs on the real vector space of Hermitian hierarchies with real scalars.
//
// Method: BiCGSTAB(ell) (Sleijpen and Fokkema, ETNA 1, 1993), the reference's
// default; ell = 1 is BiCGSTAB.  Each outer iteration takes ell BiCG steps
// (two operator applies each) and then one minimal-residual step over
// r_1..r_ell, solved from the normal equations of the ell x ell Gram matrix
// (Cholesky in FP64, falling back to the one-term step if it is singular).
// HEOM Liouvillians have eigenvalues with large imaginary parts, where
// BiCGSTAB's one-term real minimal-residual step stagnates; the degree-ell
// polynomial of BiCGSTAB(ell) has complex roots and does not.
//
// Inner products are FP64 block partial sums reduced by the last block to
// finish, in block order (deterministic); the scalar recurrences run in that
// block.  Kernels return at once when the solve is done, so a captured graph
// of several outer iterations is replayed until the host sees the done flag.
#include <cuda_runtime.h>

#include <cstdint>

#include "heom_bicgstab.h"

namespace phi {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ double cdot_re(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ bool finite(double v) { return v == v && v - v == 0.0; }

// Block reduction of K doubles; thread 0 gets the totals.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
  __shared__ double sh[K][kBlock / 32];
  __syncthreads();  // sh may still be read by an earlier call
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[k][warp] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) s += sh[k][w];
      v[k] = s;
    }
  }
}

// Reduces the block's K partial sums, publishes them and returns true in
// every thread of the one block that finishes last; that block then holds the
// grid totals in thread 0's tot[] (summed in block order) and has reset the
// arrival counter for the next kernel.
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double (&tot)[K], double *partials, unsigned int *counter) {
  __shared__ bool last;
  block_sum<K>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double w[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    w[k] = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += kBlock)
      w[k] += ((volatile const double *)partials)[k * gridDim.x + b];
  }
  block_sum<K>(w);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = w[k];
    *counter = 0u;
  }
  return true;
}

#define GRID_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < (n); i += (long long)gridDim.x * kBlock)

__device__ __forceinline__ bool solve_done(const BicgScalars *sc) { return *(volatile const int *)&sc->done; }

__device__ __forceinline__ void fail(BicgScalars *sc, int code) {
  sc->breakdown = code;
  sc->done = 1;
}

// r_0 = b - A x_0 (A x_0 in r_1), rhat = r_0, u_0 = 0; rr = <r_0, r_0>, bb.
// The first BiCG step's rho and beta follow: rho0 = -omega rho0 = -1 with
// the initial omega = 1, rho1 = <rhat, r_0> = rr, beta = alpha rho1 / rho0 = 0.
__global__ void init_kernel(BicgVectors V, long long n, BicgScalars *sc) {
  double acc[2] = {0.0, 0.0}, tot[2];
  GRID_LOOP(i, n) {
    const double2 b = V.b[i], t = V.r[1][i];
    const double2 r = i == 0 ? make_double2(0.0, 0.0) : make_double2(b.x - t.x, b.y - t.y);
    V.r[0][i] = r;
    V.rhat[i] = r;
    V.u[0][i] = make_double2(0.0, 0.0);
    acc[0] += cdot_re(r, r);
    acc[1] += cdot_re(b, b);
  }
  if (grid_sum<2>(acc, tot, sc->partials, &sc->counter) && threadIdx.x == 0) {
    sc->rr = tot[0];
    sc->bb = tot[1];
    // tol_mode 0: ||r|| <= tol ||b||; 1: ||r|| <= tol; 2: ||r||^2 <= tol.
    sc->tol2 = sc->tol_mode == 2 ? sc->tol
               : sc->tol_mode == 1 ? sc->tol * sc->tol
                                   : sc->tol * sc->tol * (tot[1] > 0 ? tot[1] : 1.0);
    sc->alpha = 0.0;
    sc->omega = 1.0;
    sc->beta = 0.0;
    sc->rho0 = tot[0];
    sc->steps = 0;
    sc->done = 0;
    sc->converged = 0;
    sc->breakdown = kBicgOk;
    sc->restart = 0;
    if (!finite(tot[0]) || !finite(tot[1])) {
      fail(sc, kBicgNonFinite);
    } else if (tot[0] <= sc->tol2) {
      sc->done = 1;
      sc->converged = 1;
    } else if (tot[0] == 0.0) {
      fail(sc, kBicgRhoZero);
    }
  }
}

// BiCG step j >= 1: rho1 = <rhat, r_j>, beta = alpha rho1 / rho0, rho0 = rho1.
// Also drops element 0 of r_j = A r_{j-1}.
__global__ void rho_kernel(BicgVectors V, long long n, BicgScalars *sc, int j) {
  if (solve_done(sc)) return;
  double2 *rj = V.r[j];
  double acc[1] = {0.0}, tot[1];
  GRID_LOOP(i, n) {
    if (i == 0) {
      rj[0] = make_double2(0.0, 0.0);
      continue;
    }
    acc[0] += cdot_re(V.rhat[i], rj[i]);
  }
  if (grid_sum<1>(acc, tot, sc->partials, &sc->counter) && threadIdx.x == 0) {
    if (!finite(tot[0])) {
      fail(sc, kBicgNonFinite);
    } else if (sc->rho0 == 0.0 || tot[0] == 0.0) {
      fail(sc, kBicgRhoZero);
    } else {
      sc->beta = sc->alpha * tot[0] / sc->rho0;
      sc->rho0 = tot[0];
    }
  }
}

// u_i = r_i - beta u_i for i = 0..j.
__global__ void u_update_kernel(BicgVectors V, long long n, const BicgScalars *sc, int j) {
  if (solve_done(sc)) return;
  const double beta = sc->beta;
  GRID_LOOP(e, n) {
    for (int i = 0; i <= j; ++i) {
      const double2 r = V.r[i][e], u = V.u[i][e];
      V.u[i][e] = make_double2(r.x - beta * u.x, r.y - beta * u.y);
    }
  }
}

// alpha = rho0 / <rhat, u_{j+1}>; drops element 0 of u_{j+1} = A u_j.
__global__ void gamma_kernel(BicgVectors V, long long n, BicgScalars *sc, int j) {
  if (solve_done(sc)) return;
  double2 *uj = V.u[j + 1];
  double acc[1] = {0.0}, tot[1];
  GRID_LOOP(i, n) {
    if (i == 0) {
      uj[0] = make_double2(0.0, 0.0);
      continue;
    }
    acc[0] += cdot_re(V.rhat[i], uj[i]);
  }
  if (grid_sum<1>(acc, tot, sc->partials, &sc->counter) && threadIdx.x == 0) {
    if (!finite(tot[0])) fail(sc, kBicgNonFinite);
    else if (tot[0] == 0.0) fail(sc, kBicgGammaZero);
    else sc->alpha = sc->rho0 / tot[0];
  }
}

// rho_kernel / gamma_kernel's scalar steps from per-tile partial sums of
// <rhat, .> (the apply zeroed element 0 and summed them); one block, summed
// in tile order (deterministic).
__global__ void dot_finish_kernel(const double *parts, long long nparts, BicgScalars *sc, int which) {
  if (solve_done(sc)) return;
  double v[1] = {0.0};
  for (long long b = threadIdx.x; b < nparts; b += kBlock) v[0] += parts[b];
  block_sum<1>(v);
  if (threadIdx.x != 0) return;
  bicg_dot_step(sc, v[0], which);
}

// r_i -= alpha u_{i+1} for i = 0..j; x += alpha u_0.
__global__ void r_update_kernel(BicgVectors V, long long n, const BicgScalars *sc, int j) {
  if (solve_done(sc)) return;
  const double a = sc->alpha;
  GRID_LOOP(e, n) {
    for (int i = 0; i <= j; ++i) {
      const double2 r = V.r[i][e], u = V.u[i + 1][e];
      V.r[i][e] = make_double2(r.x - a * u.x, r.y - a * u.y);
    }
    const double2 x = V.x[e], u0 = V.u[0][e];
    V.x[e] = make_double2(x.x + a * u0.x, x.y + a * u0.y);
  }
}

// Dot index of <r_i, r_k>, 1 <= i <= k <= ell; the <r_0, r_k> follow them.
__host__ __device__ constexpr int gram_index(int i, int k) { return (k - 1) * k / 2 + (i - 1); }

// Minimal residual over r_1..r_ell: gamma = argmin ||r_0 - sum_j gamma_j r_j||
// from G gamma = c, G_ik = <r_i, r_k>, c_k = <r_0, r_k>.  Drops element 0 of
// r_ell = A r_{ell-1}.
template <int ELL>
__global__ void gram_kernel(BicgVectors V, long long n, BicgScalars *sc) {
  if (solve_done(sc)) return;
  constexpr int NG = ELL * (ELL + 1) / 2;
  constexpr int ND = NG + ELL;
  double acc[ND], tot[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) acc[k] = 0.0;
  GRID_LOOP(e, n) {
    if (e == 0) {
      V.r[ELL][0] = make_double2(0.0, 0.0);
      continue;
    }
    double2 r[ELL + 1];
#pragma unroll
    for (int i = 0; i <= ELL; ++i) r[i] = V.r[i][e];
#pragma unroll
    for (int k = 1; k <= ELL; ++k) {
#pragma unroll
      for (int i = 1; i <= k; ++i) acc[gram_index(i, k)] += cdot_re(r[i], r[k]);
      acc[NG + k - 1] += cdot_re(r[0], r[k]);
    }
  }
  if (grid_sum<ND>(acc, tot, sc->partials, &sc->counter) && threadIdx.x == 0) {
    double G[ELL][ELL], c[ELL];
    bool ok = true;
    for (int k = 1; k <= ELL; ++k) {
      for (int i = 1; i <= k; ++i) G[i - 1][k - 1] = G[k - 1][i - 1] = tot[gram_index(i, k)];
      c[k - 1] = tot[NG + k - 1];
    }
    for (int k = 0; k < ND; ++k) ok = ok && finite(tot[k]);
    if (!ok) {
      fail(sc, kBicgNonFinite);
      return;
    }
    // Cholesky G = L L^T; a pivot that is not clearly positive means
    // r_1..r_ell are numerically dependent.
    double L[ELL][ELL];
    for (int a = 0; a < ELL; ++a)
      for (int b = 0; b < ELL; ++b) L[a][b] = G[a][b];
    bool chol = true;
    for (int k = 0; k < ELL && chol; ++k) {
      double d = L[k][k];
      for (int m = 0; m < k; ++m) d -= L[k][m] * L[k][m];
      if (!(d > 1e-14 * G[k][k])) {
        chol = false;
        break;
      }
      d = sqrt(d);
      L[k][k] = d;
      for (int a = k + 1; a < ELL; ++a) {
        double s = L[a][k];
        for (int m = 0; m < k; ++m) s -= L[a][m] * L[k][m];
        L[a][k] = s / d;
      }
    }
    double g[ELL];
    if (chol) {
      double y[ELL];
      for (int a = 0; a < ELL; ++a) {
        double s = c[a];
        for (int m = 0; m < a; ++m) s -= L[a][m] * y[m];
        y[a] = s / L[a][a];
      }
      for (int a = ELL - 1; a >= 0; --a) {
        double s = y[a];
        for (int m = a + 1; m < ELL; ++m) s -= L[m][a] * g[m];
        g[a] = s / L[a][a];
      }
    } else if (G[0][0] > 0.0) {
      // One-term minimal residual over r_1 only.  The residual polynomial
      // then lacks its degree-ell term, so the BiCG recurrence restarts
      // from the updated residual (u_0 = 0, beta = 0).
      for (int a = 0; a < ELL; ++a) g[a] = 0.0;
      g[0] = c[0] / G[0][0];
      sc->restart = 1;
    } else {
      fail(sc, kBicgGramSingular);
      return;
    }
    for (int a = 0; a < ELL; ++a) sc->gamma[a + 1] = g[a];
    // omega scales the next outer iteration's rho0 (rho0 = -omega rho0): the
    // leading coefficient of the residual polynomial's new factor.
    sc->omega = g[ELL - 1];
  }
}

// x += sum_j gamma_j r_{j-1}; r_0 -= sum_j gamma_j r_j; u_0 -= sum_j gamma_j u_j;
// then rr = <r_0, r_0>, the stopping test, and the first BiCG step of the
// next outer iteration (rho0 = -omega rho0; rho1 = <rhat, r_0>;
// beta = alpha rho1 / rho0; rho0 = rho1).
template <int ELL>
__global__ void mr_update_kernel(BicgVectors V, long long n, BicgScalars *sc) {
  if (solve_done(sc)) return;
  double g[ELL + 1];
#pragma unroll
  for (int j = 1; j <= ELL; ++j) g[j] = sc->gamma[j];
  const bool restart = sc->restart;
  double acc[2] = {0.0, 0.0}, tot[2];
  GRID_LOOP(e, n) {
    double2 x = V.x[e], r0 = V.r[0][e], u0 = V.u[0][e];
#pragma unroll
    for (int j = 1; j <= ELL; ++j) {
      const double2 rp = V.r[j - 1][e], rj = V.r[j][e], uj = V.u[j][e];
      x.x += g[j] * rp.x;
      x.y += g[j] * rp.y;
      r0.x -= g[j] * rj.x;
      r0.y -= g[j] * rj.y;
      u0.x -= g[j] * uj.x;
      u0.y -= g[j] * uj.y;
    }
    V.x[e] = x;
    V.r[0][e] = r0;
    V.u[0][e] = restart ? make_double2(0.0, 0.0) : u0;
    acc[0] += cdot_re(r0, r0);
    acc[1] += cdot_re(V.rhat[e], r0);
  }
  if (grid_sum<2>(acc, tot, sc->partials, &sc->counter) && threadIdx.x == 0) {
    sc->rr = tot[0];
    sc->steps += ELL;
    if (!finite(tot[0]) || !finite(tot[1])) {
      fail(sc, kBicgNonFinite);
    } else if (tot[0] <= sc->tol2) {
      sc->done = 1;
      sc->converged = 1;
    } else if (sc->steps >= sc->max_steps) {
      sc->done = 1;
    } else if (restart) {
      sc->restart = 0;
      sc->alpha = 0.0;
      sc->beta = 0.0;
      sc->rho0 = tot[1];
      if (tot[1] == 0.0) fail(sc, kBicgRhoZero);
    } else {
      const double rho0 = -sc->omega * sc->rho0;
      if (rho0 == 0.0 || tot[1] == 0.0) {
        fail(sc, kBicgRhoZero);
      } else {
        sc->beta = sc->alpha * tot[1] / rho0;
        sc->rho0 = tot[1];
      }
    }
  }
}

// 1 / tr rho_0 of the solution with x_0[0,0] = 1 (one thread).
__global__ void trace_kernel(const double2 *x, int N, BicgScalars *sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double tr = 1.0;
  for (int i = 1; i < N; ++i) tr += x[(long long)i * (N + 1)].x;
  sc->inv_trace = 1.0 / tr;
}

// out = x with x_0[0,0] = 1, divided by tr rho_0 (the reference renormalises
// rho_0 by its trace, hierarchy_integrator.cc:3755-3760; here every node is
// scaled so the hierarchy stays one consistent state).
__global__ void finalize_kernel(const double2 *x, double2 *out, long long n, const BicgScalars *sc) {
  const double s = sc->inv_trace;
  GRID_LOOP(i, n) {
    const double2 v = i == 0 ? make_double2(1.0, 0.0) : x[i];
    out[i] = make_double2(v.x * s, v.y * s);
  }
}

// b = -L(E00) with element 0 zeroed (in place on the apply output).
__global__ void rhs_kernel(double2 *b, long long n) {
  GRID_LOOP(i, n) b[i] = i == 0 ? make_double2(0.0, 0.0) : make_double2(-b[i].x, -b[i].y);
}

// Initial guess scaled so that element (0,0) of node 0 is 1.  Every block
// reads element 0; guess_clear_kernel clears it afterwards.
__global__ void guess_scale_kernel(double2 *x, long long n) {
  const double x00 = x[0].x;
  const double s = (x00 != 0.0 && finite(x00)) ? 1.0 / x00 : 1.0;
  GRID_LOOP(i, n) {
    if (i != 0) x[i] = make_double2(x[i].x * s, x[i].y * s);
  }
}
__global__ void guess_clear_kernel(double2 *x) { x[0] = make_double2(0.0, 0.0); }

template <int ELL>
cudaError_t launch_gram_t(const BicgVectors &V, long long n, BicgScalars *sc, int grid, cudaStream_t s) {
  gram_kernel<ELL><<<grid, kBlock, 0, s>>>(V, n, sc);
  return cudaGetLastError();
}
template <int ELL>
cudaError_t launch_mr_t(const BicgVectors &V, long long n, BicgScalars *sc, int grid, cudaStream_t s) {
  mr_update_kernel<ELL><<<grid, kBlock, 0, s>>>(V, n, sc);
  return cudaGetLastError();
}

}  // namespace

int bicg_grid(int num_sms) { return num_sms * 4 > kMaxBicgBlocks ? kMaxBicgBlocks : num_sms * 4; }

cudaError_t bicg_launch_rhs(double2 *b, long long n, int grid, cudaStream_t s) {
  rhs_kernel<<<grid, kBlock, 0, s>>>(b, n);
  return cudaGetLastError();
}
cudaError_t bicg_launch_guess(double2 *x, long long n, int grid, cudaStream_t s) {
  guess_scale_kernel<<<grid, kBlock, 0, s>>>(x, n);
  guess_clear_kernel<<<1, 1, 0, s>>>(x);
  return cudaGetLastError();
}
cudaError_t bicg_launch_init(const BicgVectors &V, long long n, BicgScalars *sc, int grid, cudaStream_t s) {
  init_kernel<<<grid, kBlock, 0, s>>>(V, n, sc);
  return cudaGetLastError();
}
cudaError_t bicg_launch_rho(const BicgVectors &V, long long n, BicgScalars *sc, int j, int grid, cudaStream_t s) {
  rho_kernel<<<grid, kBlock, 0, s>>>(V, n, sc, j);
  return cudaGetLastError();
}
cudaError_t bicg_launch_dot_finish(const double *parts, long long nparts, BicgScalars *sc, int which,
                                   cudaStream_t s) {
  dot_finish_kernel<<<1, kBlock, 0, s>>>(parts, nparts, sc, which);
  return cudaGetLastError();
}
cudaError_t bicg_launch_u_update(const BicgVectors &V, long long n, const BicgScalars *sc, int j, int grid,
                                 cudaStream_t s) {
  u_update_kernel<<<grid, kBlock, 0, s>>>(V, n, sc, j);
  return cudaGetLastError();
}
cudaError_t bicg_launch_gamma(const BicgVectors &V, long long n, BicgScalars *sc, int j, int grid, cudaStream_t s) {
  gamma_kernel<<<grid, kBlock, 0, s>>>(V, n, sc, j);
  return cudaGetLastError();
}
cudaError_t bicg_launch_r_update(const BicgVectors &V, long long n, const BicgScalars *sc, int j, int grid,
                                 cudaStream_t s) {
  r_update_kernel<<<grid, kBlock, 0, s>>>(V, n, sc, j);
  return cudaGetLastError();
}
cudaError_t bicg_launch_gram(const BicgVectors &V, long long n, BicgScalars *sc, int ell, int grid, cudaStream_t s) {
  switch (ell) {
    case 1: return launch_gram_t<1>(V, n, sc, grid, s);
    case 2: return launch_gram_t<2>(V, n, sc, grid, s);
    case 3: return launch_gram_t<3>(V, n, sc, grid, s);
    case 4: return launch_gram_t<4>(V, n, sc, grid, s);
    case 5: return launch_gram_t<5>(V, n, sc, grid, s);
    case 6: return launch_gram_t<6>(V, n, sc, grid, s);
    case 7: return launch_gram_t<7>(V, n, sc, grid, s);
    case 8: return launch_gram_t<8>(V, n, sc, grid, s);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t bicg_launch_mr_update(const BicgVectors &V, long long n, BicgScalars *sc, int ell, int grid,
                                  cudaStream_t s) {
  switch (ell) {
    case 1: return launch_mr_t<1>(V, n, sc, grid, s);
    case 2: return launch_mr_t<2>(V, n, sc, grid, s);
    case 3: return launch_mr_t<3>(V, n, sc, grid, s);
    case 4: return launch_mr_t<4>(V, n, sc, grid, s);
    case 5: return launch_mr_t<5>(V, n, sc, grid, s);
    case 6: return launch_mr_t<6>(V, n, sc, grid, s);
    case 7: return launch_mr_t<7>(V, n, sc, grid, s);
    case 8: return launch_mr_t<8>(V, n, sc, grid, s);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t bicg_launch_finalize(const double2 *x, double2 *out, long long n, int N, BicgScalars *sc, int grid,
                                 cudaStream_t s) {
  trace_kernel<<<1, 32, 0, s>>>(x, N, sc);
  finalize_kernel<<<grid, kBlock, 0, s>>>(x, out, n, sc);
  return cudaGetLastError();
}

}  // namespace phi
