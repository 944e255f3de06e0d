// heom_bicgstab.h -- device BiCGSTAB(ell) for the steady state (internal).
#pragma once

#include <cuda_runtime.h>

namespace phi {

constexpr int kMaxBicgBlocks = 1024;
constexpr int kMaxEll = 8;
// Inner products of the minimal-residual step: <r_i, r_k> for 1 <= i <= k <= ell
// and <r_0, r_k> for 1 <= k <= ell.
constexpr int kMaxGramDots = kMaxEll * (kMaxEll + 1) / 2 + kMaxEll;

// Krylov vectors, each M*N*N complex128 in the state's node-major layout.
struct BicgVectors {
  double2 *x, *rhat, *b;
  double2 *r[kMaxEll + 1];
  double2 *u[kMaxEll + 1];
};

enum BicgBreakdown {
  kBicgOk = 0,
  kBicgRhoZero = 1,     // <rhat, r_j> = 0 (BiCG breakdown)
  kBicgGammaZero = 2,   // <rhat, A u_j> = 0
  kBicgGramSingular = 3,
  kBicgNonFinite = 4,
};

// Device-resident solver state; every scalar recurrence runs on the device.
struct BicgScalars {
  double rho0, alpha, omega, beta;
  double rr, bb, tol, tol2;
  double gamma[kMaxEll + 1];  // minimal-residual coefficients gamma_1..gamma_ell
  double inv_trace;
  int ell, steps, max_steps, done, converged, breakdown, tol_mode;
  int restart;  // the minimal-residual step fell back to one term: restart the BiCG recurrence
  unsigned int counter;
  double partials[kMaxGramDots * kMaxBicgBlocks];
};

#ifdef __CUDACC__
// The scalar step once <rhat, .> is summed (one thread): which = 0, rho --
// beta = alpha rho_new / rho_old and the new rho, a breakdown if either
// vanishes; which = 1, gamma -- alpha = rho / gamma.  A non-finite sum stops
// the solve.
__device__ inline void bicg_dot_step(BicgScalars *sc, double tot, int which) {
  int code = kBicgOk;
  if (!(tot == tot && tot - tot == 0.0)) {
    code = kBicgNonFinite;
  } else if (which == 0) {
    if (sc->rho0 == 0.0 || tot == 0.0) {
      code = kBicgRhoZero;
    } else {
      sc->beta = sc->alpha * tot / sc->rho0;
      sc->rho0 = tot;
    }
  } else if (tot == 0.0) {
    code = kBicgGammaZero;
  } else {
    sc->alpha = sc->rho0 / tot;
  }
  if (code != kBicgOk) {
    sc->breakdown = code;
    sc->done = 1;
  }
}
#endif

int bicg_grid(int num_sms);
// b = -b with element (0,0) of node 0 zeroed (b holds L(E00) on entry).
cudaError_t bicg_launch_rhs(double2 *b, long long n, int grid, cudaStream_t s);
// x /= x[0] (the guess scaled to x_0[0,0] = 1), then x[0] = 0.
cudaError_t bicg_launch_guess(double2 *x, long long n, int grid, cudaStream_t s);
// r_0 = b - r_1 (r_1 holds A x_0 on entry), rhat = r_0, u_0 = 0; scalars.
cudaError_t bicg_launch_init(const BicgVectors &V, long long n, BicgScalars *sc, int grid, cudaStream_t s);
// BiCG step j of an outer iteration, around the two operator applies.
cudaError_t bicg_launch_rho(const BicgVectors &V, long long n, BicgScalars *sc, int j, int grid, cudaStream_t s);
cudaError_t bicg_launch_u_update(const BicgVectors &V, long long n, const BicgScalars *sc, int j, int grid,
                                 cudaStream_t s);
cudaError_t bicg_launch_gamma(const BicgVectors &V, long long n, BicgScalars *sc, int j, int grid, cudaStream_t s);
cudaError_t bicg_launch_r_update(const BicgVectors &V, long long n, const BicgScalars *sc, int j, int grid,
                                 cudaStream_t s);
// The same two inner products when the apply that produced the vector
// already summed <rhat, .> per tile (the tiled kernel, dot_part of a stage
// launch): one block adds the nparts partials in order and runs the scalar
// step of rho (which = 0) or gamma (which = 1).
cudaError_t bicg_launch_dot_finish(const double *parts, long long nparts, BicgScalars *sc, int which,
                                   cudaStream_t s);
// Minimal-residual step over r_1..r_ell and the end-of-iteration control.
cudaError_t bicg_launch_gram(const BicgVectors &V, long long n, BicgScalars *sc, int ell, int grid, cudaStream_t s);
cudaError_t bicg_launch_mr_update(const BicgVectors &V, long long n, BicgScalars *sc, int ell, int grid,
                                  cudaStream_t s);
// out = x with x_0[0,0] = 1, divided by tr rho_0.
cudaError_t bicg_launch_finalize(const double2 *x, double2 *out, long long n, int N, BicgScalars *sc, int grid,
                                 cudaStream_t s);

}  // namespace phi
