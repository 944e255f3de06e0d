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
};

// Host: PHI's spline coefficients for n >= 2 samples y (x, a, b, c, d, each
// n doubles, written to out[0..5n)).
void anneal_spline_host(const double *y, int n, double *out);
cudaError_t launch_anneal(const AnnealLaunch &p, cudaStream_t stream);

}  // namespace phi
