// heom_anneal.cu -- the annealing Hamiltonian on the device.
//
// With no static Hamiltonian PHI anneals: before every RK4 / RKF45 stage at
// time t it evaluates two cubic splines at alpha = t / T and sets
// H = f_x H_X + f_z H_Z, but only when either field moved by at least the
// minimum relative change since the last update
// (UpdateTimeDependentHamiltonian, hierarchy_integrator.cc:1618-1673; the
// stage times :1988-2252 and :2688-2792).  One CTA does it: thread 0 walks
// the splines (keeping their interval search positions, as CubicSpline does)
// and decides, the block writes H.  The stage kernels read H from the same
// buffer.  The stage time comes from the device control block, so captured
// step graphs need no host round trip.
#include <cuda_runtime.h>

#include <vector>

#include "heom_anneal.h"

namespace phi {
namespace {

constexpr int kAnnealThreads = 256;

// CubicSpline::Get with Locate (cubic_spline.cc:33-81).
__device__ double spline_get(const AnnealSpline &s, double x, int *last) {
  if (x > s.x[s.n - 1]) return s.a[s.n - 1];
  if (x < s.x[0]) return s.a[0];
  int i = *last;
  if (!(x > s.x[i] && x < s.x[i + 1])) {
    while (x > s.x[i + 1]) ++i;
    while (x < s.x[i]) --i;
    *last = i;
  }
  const double t = (x - s.x[i]) / (s.x[i + 1] - s.x[i]);
  // a + b t + c t t + d t t t, evaluated left to right without contraction
  double v = __dadd_rn(s.a[i], __dmul_rn(s.b[i], t));
  v = __dadd_rn(v, __dmul_rn(__dmul_rn(s.c[i], t), t));
  return __dadd_rn(v, __dmul_rn(__dmul_rn(__dmul_rn(s.d[i], t), t), t));
}

__global__ void __launch_bounds__(kAnnealThreads) anneal_kernel(AnnealLaunch p) {
  __shared__ int update;
  __shared__ double sfx, sfz;
  if (threadIdx.x == 0) {
    update = 0;
    bool skip = false;
    double t = 0.0;
    if (p.op == kAnnealRk4) {
      const double t0 = p.rk4->time;
      t = p.which == 0 ? t0 : (p.which == 1 ? t0 + p.dt / 2 : t0 + p.dt);
      if (p.which == 2) p.rk4->time = t;  // time_now += dt at the end of the step (:2856)
    } else {
      skip = *(volatile const int *)&p.ctl->done != 0;
      if (!skip) t = p.which == 0 ? p.ctl->time : p.ctl->time + p.ctl->a[p.which - 1];
    }
    if (!skip) {
      AnnealState *st = p.st;
      const double alpha = t / p.integration_time;
      const double fx = spline_get(p.sx, alpha, &st->last_x);
      const double fz = spline_get(p.sz, alpha, &st->last_z);
      const double chx = fabs(fx / st->old_fx - 1.0), chz = fabs(fz / st->old_fz - 1.0);
      if (!(chx < p.min_field_change && chz < p.min_field_change)) {
        st->old_fx = fx;
        st->old_fz = fz;
        sfx = fx;
        sfz = fz;
        update = 1;
      }
    }
  }
  __syncthreads();
  if (!update) return;
  const double fx = sfx, fz = sfz;
  for (int e = threadIdx.x; e < p.E; e += kAnnealThreads) {
    const double2 a = p.hx[e], b = p.hz[e];
    // (f + 0i)(a) + (g + 0i)(b), as PHI's complex products and sum
    p.H[e] = make_double2(__dadd_rn(__dsub_rn(__dmul_rn(fx, a.x), __dmul_rn(0.0, a.y)),
                                    __dsub_rn(__dmul_rn(fz, b.x), __dmul_rn(0.0, b.y))),
                          __dadd_rn(__dadd_rn(__dmul_rn(fx, a.y), __dmul_rn(0.0, a.x)),
                                    __dadd_rn(__dmul_rn(fz, b.y), __dmul_rn(0.0, b.x))));
  }
}

}  // namespace

// PHI's CubicSpline::Initialize and SolveTridiagonal (cubic_spline.cc:45-120)
// as written: b_0 = 3 (y_1 - y_0), b_{n-1} = 3 (y_{n-1} - y_{n-2}),
// b_i = 3 (y_{i+1} - y_i), solved against the tridiagonal (2, 4, ..., 4, 2 | 1)
// by an L D L^T factorisation and forward / backward substitution.
void anneal_spline_host(const double *y, int n, double *out) {
  double *x = out, *a = out + n, *b = out + 2 * n, *c = out + 3 * n, *d = out + 4 * n;
  const double ds = 1. / (n - 1);
  for (int i = 0; i < n; ++i) x[i] = i * ds;
  for (int i = 0; i < n; ++i) a[i] = y[i];
  b[0] = 3. * (y[1] - y[0]);
  b[n - 1] = 3. * (y[n - 1] - y[n - 2]);
  for (int i = 1; i < n - 1; ++i) b[i] = 3. * (y[i + 1] - y[i]);
  std::vector<double> dg(n), e(n);
  dg[0] = dg[n - 1] = 2.;
  for (int i = 1; i < n - 1; ++i) dg[i] = 4.;
  for (int i = 0; i < n - 1; ++i) e[i] = 1.;
  for (int i = 0; i < n - 1; ++i) {
    const double ei = e[i];
    e[i] = ei / dg[i];
    dg[i + 1] = dg[i + 1] - e[i] * ei;
  }
  for (int i = 1; i < n; ++i) b[i] = b[i] - b[i - 1] * e[i - 1];
  b[n - 1] = b[n - 1] / dg[n - 1];
  for (int i = n - 2; i >= 0; --i) b[i] = b[i] / dg[i] - b[i + 1] * e[i];
  for (int i = 0; i < n - 1; ++i) {
    c[i] = 3. * (a[i + 1] - a[i]) - 2. * b[i] - b[i + 1];
    d[i] = 2. * (a[i] - a[i + 1]) + b[i] + b[i + 1];
  }
  c[n - 1] = d[n - 1] = 0.0;  // never read: the last knot answers with a[n - 1]
}

cudaError_t launch_anneal(const AnnealLaunch &p, cudaStream_t stream) {
  anneal_kernel<<<1, kAnnealThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace phi
