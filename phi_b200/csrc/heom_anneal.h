// heom_anneal.h -- annealing Hamiltonian updates on the device (internal).
#pragma once

#include <cuda_runtime.h>

#include "heom_device.cuh"

namespace phi {

// PHI's CubicSpline (cubic_spline.cc): knots x_i = i / (n - 1), coefficients
// a, b, c, d per interval; device pointers.
struct AnnealSpline {
  const double *x = nullptr, *a = nullptr, *b = nullptr, *c = nullptr, *d = nullptr;
  int n = 0;
};

// The state UpdateTimeDependentHamiltonian keeps between calls: the last
// applied field values and each spline's interval search position.
struct AnnealState {
  double old_fx, old_fz;
  int last_x, last_z;
};

enum AnnealOp : int {
  kAnnealRk4 = 0,    // which: 0 -> t, 1 -> t + dt/2, 2 -> t + dt (and the step's time advances)
  kAnnealRkf45 = 1,  // which: stage 0..5 -> t, t + a1 .. t + a5 from the control block
};

// Hilbert-space truncation of the annealing Hamiltonian (F > k): at every
// update the full H is re-diagonalised, the lowest k eigenvectors become the
// basis, H is truncated into it, the full bath operators are rotated, and
// the rotation R(j, i) = <old_i | new_j> is left for anneal_rotate_kernel.
// Device pointers; F = 0 without truncation.
struct AnnealTrunc {
  int F = 0;
  int k = 0;
  const double *hx = nullptr, *hz = nullptr;  // F*F real, column-major
  double *V = nullptr;       // F*k: the current basis, column-major
  double *R = nullptr;       // k*k: the rotation of the last update
  int *rotate = nullptr;     // 1 when the last update changed the basis
  double *bath = nullptr;    // nb*k*k full bath operators, rotated in place (null: none)
  int nb = 0;
};
constexpr int kAnnealMaxFull = 32;  // largest F of a truncated annealing run

struct AnnealLaunch {
  int op = kAnnealRk4;
  int which = 0;
  double dt = 0.0;
  Rk4Ctl *rk4 = nullptr;
  Rkf45Ctl *ctl = nullptr;
  AnnealSpline sx, sz;
  AnnealState *st = nullptr;
  const double2 *hx = nullptr, *hz = nullptr;
  double2 *H = nullptr;  // the Hamiltonian the stage kernels read (HeomConsts::H)
  int E = 0;
  double integration_time = 1.0;
  double min_field_change = 0.01;
  AnnealTrunc tr;
};

// The live ADO arrays a truncated annealing update rotates
// (hierarchy_integrator.cc:1988-2263, :2688-2801): each node's k x k matrix
// X <- R herm(X) R^T, herm(X) completed from its upper triangle with a real
// diagonal (BLAS zhemm, hilbert_space_truncator.cc:63-74).  With ctl set,
// ybuf[ctl->ycur] is rotated too (the RKF45 state).
constexpr int kAnnealMaxRotate = 7;
struct AnnealRotate {
  const int *rotate = nullptr;
  const double *R = nullptr;
  int k = 0;
  long long M = 0;
  double2 *buf[kAnnealMaxRotate] = {};
  int nbuf = 0;
  double2 *ybuf[2] = {};
  const Rkf45Ctl *ctl = nullptr;
};

// Host: PHI's spline coefficients for n >= 2 samples y (x, a, b, c, d, each
// n doubles, written to out[0..5n)).
void anneal_spline_host(const double *y, int n, double *out);
cudaError_t launch_anneal(const AnnealLaunch &p, cudaStream_t stream);
cudaError_t launch_anneal_rotate(const AnnealRotate &p, int num_sms, cudaStream_t stream);

}  // namespace phi
