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

#include <algorithm>
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

// ---------------------------------------------------------------------------
// Hilbert-space truncation (AnnealTrunc).

__device__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Cyclic Jacobi eigenvalue iteration (Jacobi 1846; rotations as in
// Rutishauser's formulation) of the real symmetric n x n matrix a (shared,
// column-major, n <= 32), run by one warp: lane r updates row / column r of
// each rotation.  On return the diagonal of a holds the eigenvalues and the
// columns of z the eigenvectors.  Every lane computes the rotation from the
// same shared values, so the branch on a vanishing element is warp-uniform.
__device__ void warp_jacobi(int n, double *a, double *z, int lane) {
  for (int e = lane; e < n * n; e += 32) z[e] = 0.0;
  __syncwarp();
  if (lane < n) z[lane + lane * n] = 1.0;
  double sc = 0.0;
  for (int e = lane; e < n * n; e += 32) sc = fmax(sc, fabs(a[e]));
  sc = warp_max(sc);
  for (int sweep = 0; sweep < 100 && sc > 0.0; ++sweep) {
    __syncwarp();
    double off = 0.0;
    for (int e = lane; e < n * n; e += 32)
      if (e % n < e / n) off += a[e] * a[e];
    // Lane 0's sum decides for the warp (the butterfly sums of the other
    // lanes may round differently).
    off = __shfl_sync(0xffffffffu, warp_sum(off), 0);
    if (sqrt(off) <= 1e-16 * sc) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        __syncwarp();
        const double apq = a[p + q * n];
        if (fabs(apq) <= 1e-300) continue;
        const double th = (a[q + q * n] - a[p + p * n]) / (2.0 * apq);
        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
        __syncwarp();
        if (lane < n) {  // columns p, q
          const double x = a[lane + p * n], y = a[lane + q * n];
          a[lane + p * n] = cs * x - sn * y;
          a[lane + q * n] = sn * x + cs * y;
        }
        __syncwarp();
        if (lane < n) {  // rows p, q
          const double x = a[p + lane * n], y = a[q + lane * n];
          a[p + lane * n] = cs * x - sn * y;
          a[q + lane * n] = sn * x + cs * y;
        }
        __syncwarp();
        if (lane == 0) a[p + q * n] = a[q + p * n] = 0.0;
        if (lane < n) {
          const double x = z[lane + p * n], y = z[lane + q * n];
          z[lane + p * n] = cs * x - sn * y;
          z[lane + q * n] = sn * x + cs * y;
        }
      }
  }
  __syncwarp();
}

// The truncated part of one applied Hamiltonian update (the block of
// anneal_kernel, after the fields fx, fz were accepted):
// HilbertSpaceTruncator::UpdateWith (hilbert_space_truncator.cc:101-113),
// Truncate (:34-58) of H and Rotate (:63-74) of the full bath operators
// (hierarchy_integrator.cc:1646-1668).
__device__ void truncated_update(const AnnealLaunch &p, double fx, double fz) {
  constexpr int F2 = kAnnealMaxFull * kAnnealMaxFull;
  __shared__ double hf[F2], a[F2], z[F2], vn[F2], w[F2];
  __shared__ int order[kAnnealMaxFull];
  __shared__ double sgn[kAnnealMaxFull];
  const AnnealTrunc &tr = p.tr;
  const int F = tr.F, k = tr.k, tid = threadIdx.x;
  // H = f_x H_X + f_z H_Z (real: truncation is built for real H_X, H_Z).
  for (int e = tid; e < F * F; e += kAnnealThreads) {
    const double h = __dadd_rn(__dmul_rn(fx, tr.hx[e]), __dmul_rn(fz, tr.hz[e]));
    hf[e] = h;
    a[e] = h;
  }
  __syncthreads();
  if (tid < 32) warp_jacobi(F, a, z, tid);
  __syncthreads();
  if (tid == 0) {
    // Ascending eigenvalues: selection sort with swaps of (value, index).
    double ev[kAnnealMaxFull];
    for (int i = 0; i < F; ++i) {
      ev[i] = a[i + i * F];
      order[i] = i;
    }
    for (int i = 0; i < F; ++i) {
      int best = i;
      for (int j = i + 1; j < F; ++j)
        if (ev[j] < ev[best]) best = j;
      if (best != i) {
        const double tv = ev[i];
        ev[i] = ev[best];
        ev[best] = tv;
        const int to = order[i];
        order[i] = order[best];
        order[best] = to;
      }
    }
  }
  __syncthreads();
  // Each kept vector takes the sign whose overlap with the previous vector
  // of the same index is non-negative (LAPACK's signs are arbitrary).
  if (tid < k) {
    double d = 0.0;
    for (int r = 0; r < F; ++r) d += tr.V[r + tid * F] * z[r + order[tid] * F];
    sgn[tid] = d < 0 ? -1.0 : 1.0;
  }
  __syncthreads();
  for (int e = tid; e < F * k; e += kAnnealThreads) {
    const int r = e % F, j = e / F;
    vn[e] = sgn[j] * z[r + order[j] * F];
  }
  __syncthreads();
  // R(j, i) = <old_i | new_j>, then the new basis replaces the old.
  for (int e = tid; e < k * k; e += kAnnealThreads) {
    const int j = e % k, i = e / k;
    double d = 0.0;
    for (int r = 0; r < F; ++r) d += tr.V[r + i * F] * vn[r + j * F];
    tr.R[e] = d;
    w[e] = d;  // R, kept in shared for the bath rotation
  }
  __syncthreads();
  for (int e = tid; e < F * k; e += kAnnealThreads) tr.V[e] = vn[e];
  // Truncate: work_i = H v_i (a = H V, F x k), H_k(j, i) = v_j^T work_i for
  // j <= i and its mirror.
  for (int e = tid; e < F * k; e += kAnnealThreads) {
    const int r = e % F, i = e / F;
    double acc = 0.0;
    for (int l = 0; l < F; ++l) acc += hf[r + l * F] * vn[l + i * F];
    a[e] = acc;
  }
  __syncthreads();
  for (int e = tid; e < k * k; e += kAnnealThreads) {
    const int j = e % k, i = e / k;
    if (j > i) continue;
    double acc = 0.0;
    for (int r = 0; r < F; ++r) acc += vn[r + j * F] * a[r + i * F];
    p.H[j + i * k] = make_double2(acc, 0.0);
    p.H[i + j * k] = make_double2(acc, 0.0);
  }
  // Rotate each full bath operator: B <- R herm(B) R^T (z = herm(B) R^T).
  for (int m = 0; m < tr.nb && tr.bath; ++m) {
    double *B = tr.bath + (size_t)m * k * k;
    __syncthreads();
    for (int e = tid; e < k * k; e += kAnnealThreads) {
      const int i = e % k, j = e / k;
      double acc = 0.0;
      for (int b = 0; b < k; ++b) {
        const double hb = i <= b ? B[i + b * k] : B[b + i * k];
        acc += hb * w[j + b * k];
      }
      z[e] = acc;
    }
    __syncthreads();
    for (int e = tid; e < k * k; e += kAnnealThreads) {
      const int i = e % k, j = e / k;
      double acc = 0.0;
      for (int c = 0; c < k; ++c) acc += w[i + c * k] * z[c + j * k];
      B[e] = acc;
    }
  }
  if (tid == 0) *tr.rotate = 1;
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
  if (!update) {
    if (p.tr.F > 0 && threadIdx.x == 0) *p.tr.rotate = 0;
    return;
  }
  const double fx = sfx, fz = sfz;
  if (p.tr.F > 0) {
    truncated_update(p, fx, fz);
    return;
  }
  for (int e = threadIdx.x; e < p.E; e += kAnnealThreads) {
    const double2 a = p.hx[e], b = p.hz[e];
    // (f + 0i)(a) + (g + 0i)(b), as PHI's complex products and sum
    p.H[e] = make_double2(__dadd_rn(__dsub_rn(__dmul_rn(fx, a.x), __dmul_rn(0.0, a.y)),
                                    __dsub_rn(__dmul_rn(fz, b.x), __dmul_rn(0.0, b.y))),
                          __dadd_rn(__dadd_rn(__dmul_rn(fx, a.y), __dmul_rn(0.0, a.x)),
                                    __dadd_rn(__dmul_rn(fz, b.y), __dmul_rn(0.0, b.x))));
  }
}

constexpr int kRotateThreads = 128;

// X <- R herm(X) R^T for every node of every listed buffer, one (node,
// buffer) unit per CTA iteration; a no-op unless the preceding update
// rotated the basis.
__global__ void __launch_bounds__(kRotateThreads) anneal_rotate_kernel(AnnealRotate p) {
  constexpr int K2 = (kAnnealMaxFull - 1) * (kAnnealMaxFull - 1);
  __shared__ double r[K2];
  __shared__ double2 x[K2], w[K2];
  if (*(volatile const int *)p.rotate == 0) return;
  const int k = p.k, E = k * k, tid = threadIdx.x;
  double2 *bufs[kAnnealMaxRotate + 1];
  int nb = 0;
  for (int b = 0; b < p.nbuf; ++b) bufs[nb++] = p.buf[b];
  if (p.ctl) bufs[nb++] = p.ybuf[p.ctl->ycur];
  for (int e = tid; e < E; e += kRotateThreads) r[e] = p.R[e];
  const long long units = p.M * nb;
  for (long long u = blockIdx.x; u < units; u += gridDim.x) {
    double2 *X = bufs[u / p.M] + (size_t)(u % p.M) * E;
    __syncthreads();
    for (int e = tid; e < E; e += kRotateThreads) {  // herm(X): upper triangle, real diagonal
      const int i = e % k, j = e / k;
      if (i < j) x[e] = X[e];
      else if (i > j) { const double2 v = X[j + i * k]; x[e] = make_double2(v.x, -v.y); }
      else x[e] = make_double2(X[e].x, 0.0);
    }
    __syncthreads();
    for (int e = tid; e < E; e += kRotateThreads) {  // w = herm(X) R^T
      const int i = e % k, j = e / k;
      double re = 0.0, im = 0.0;
      for (int b = 0; b < k; ++b) {
        const double rb = r[j + b * k];
        re += x[i + b * k].x * rb;
        im += x[i + b * k].y * rb;
      }
      w[e] = make_double2(re, im);
    }
    __syncthreads();
    for (int e = tid; e < E; e += kRotateThreads) {  // X = R w
      const int i = e % k, j = e / k;
      double re = 0.0, im = 0.0;
      for (int c = 0; c < k; ++c) {
        const double rc = r[i + c * k];
        re += rc * w[c + j * k].x;
        im += rc * w[c + j * k].y;
      }
      X[e] = make_double2(re, im);
    }
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
  if (p.tr.F > kAnnealMaxFull || (p.tr.F > 0 && (p.tr.k < 1 || p.tr.k >= p.tr.F))) return cudaErrorInvalidValue;
  anneal_kernel<<<1, kAnnealThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_anneal_rotate(const AnnealRotate &p, int num_sms, cudaStream_t stream) {
  if (p.k < 1 || p.k >= kAnnealMaxFull || p.nbuf > kAnnealMaxRotate) return cudaErrorInvalidValue;
  const long long units = p.M * (p.nbuf + (p.ctl ? 1 : 0));
  if (units == 0) return cudaSuccess;
  const int grid = (int)std::min<long long>(units, (long long)num_sms * 8);
  anneal_rotate_kernel<<<grid, kRotateThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace phi
