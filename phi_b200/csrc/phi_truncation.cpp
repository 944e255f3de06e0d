// phi_truncation.cpp -- Hilbert-space truncation of a problem (host).
//
// PHI's HilbertSpaceTruncator (hilbert_space_truncator.cc:34-134) keeps the
// lowest k eigenvectors V (F x k) of the full F x F Hamiltonian (LAPACK
// zheevr, range 'I', il = 1 .. iu = k, lapack_wrapper.h:71-96) and runs the
// hierarchy in that basis:
//   Truncate(A)   = V^+ A V        (the Hamiltonian, hierarchy_integrator.cc
//                                   :915-918; the initial density matrix,
//                                   :1073-1075; full bath operators, :1179-1186)
//   UnTruncate(r) = V r V^+        (density_matrix(), :177-191)
// The result in the full space does not depend on the phases or the order
// of the eigenvectors within the kept subspace (the HEOM with full bath
// couplings is covariant under a unitary change of basis), so any
// orthonormal eigenbasis reproduces PHI's.  This file computes V with the
// cyclic Jacobi eigenvalue method (Jacobi 1846; threshold strategy as in
// Rutishauser's formulation) for real symmetric Hamiltonians, the case where
// the truncated full-bath operators stay real.
#include "phi_truncation.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace phi {

int jacobi_eigh(int n, const double *a_in, double *w, double *v) {
  std::vector<double> a(a_in, a_in + (size_t)n * n);
  for (int i = 0; i < n * n; ++i) v[i] = 0.0;
  for (int i = 0; i < n; ++i) v[i + (size_t)i * n] = 1.0;
  auto A = [&](int i, int j) -> double & { return a[i + (size_t)j * n]; };
  double scale = 0.0;
  for (double x : a) scale = std::max(scale, std::fabs(x));
  if (scale == 0.0) {
    for (int i = 0; i < n; ++i) w[i] = 0.0;
    return 0;
  }
  const int max_sweeps = 100;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < j; ++i) off += A(i, j) * A(i, j);
    if (std::sqrt(off) <= 1e-16 * scale) break;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = A(p, q);
        if (std::fabs(apq) <= 1e-300) continue;
        // Rotation that zeroes A(p, q): t = sgn(th) / (|th| + sqrt(th^2 + 1)),
        // th = (A(q, q) - A(p, p)) / (2 A(p, q)).
        const double th = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        A(p, q) = A(q, p) = 0.0;
        for (int k = 0; k < n; ++k) {
          const double vkp = v[k + (size_t)p * n], vkq = v[k + (size_t)q * n];
          v[k + (size_t)p * n] = c * vkp - s * vkq;
          v[k + (size_t)q * n] = s * vkp + c * vkq;
        }
      }
    }
  }
  if (sweep == max_sweeps) return 1;
  // Ascending eigenvalues, columns of v in the same order.
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A(x, x) < A(y, y); });
  std::vector<double> vs(v, v + (size_t)n * n);
  for (int c = 0; c < n; ++c) {
    w[c] = A(order[c], order[c]);
    for (int r = 0; r < n; ++r) v[r + (size_t)c * n] = vs[r + (size_t)order[c] * n];
  }
  return 0;
}

namespace {

// V^+ A V for a complex F x F A (interleaved, column-major) and real V (F x k).
void project(int F, int k, const double *A, const double *V, std::vector<double> *out) {
  out->assign(2 * (size_t)k * k, 0.0);
  std::vector<double> av(2 * (size_t)F * k, 0.0);  // A V, F x k
  for (int j = 0; j < k; ++j)
    for (int l = 0; l < F; ++l) {
      const double vl = V[l + (size_t)j * F];
      if (vl == 0.0) continue;
      for (int i = 0; i < F; ++i) {
        av[2 * (i + (size_t)j * F)] += A[2 * (i + (size_t)l * F)] * vl;
        av[2 * (i + (size_t)j * F) + 1] += A[2 * (i + (size_t)l * F) + 1] * vl;
      }
    }
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) {
      double re = 0.0, im = 0.0;
      for (int l = 0; l < F; ++l) {
        const double vi = V[l + (size_t)i * F];
        re += vi * av[2 * (l + (size_t)j * F)];
        im += vi * av[2 * (l + (size_t)j * F) + 1];
      }
      (*out)[2 * (i + (size_t)j * k)] = re;
      (*out)[2 * (i + (size_t)j * k) + 1] = im;
    }
  // V^+ A V of a Hermitian A is Hermitian: mirror the upper triangle so the
  // rounding of the two products leaves no asymmetry.
  for (int j = 0; j < k; ++j)
    for (int i = j + 1; i < k; ++i) {
      (*out)[2 * (i + (size_t)j * k)] = (*out)[2 * (j + (size_t)i * k)];
      (*out)[2 * (i + (size_t)j * k) + 1] = -(*out)[2 * (j + (size_t)i * k) + 1];
    }
}

}  // namespace

int truncate_problem(const phi_problem_desc &d, TruncatedProblem *t, std::string *err) {
  const int F = d.hilbert_space_size, k = d.num_states;
  t->full = F;
  const bool annealing = d.annealing_h_x != nullptr;
  if (annealing) {
    if (F > kTruncatedAnnealingMaxFull) {
      *err = "Hilbert-space truncation of an annealing Hamiltonian is built for hilbert_space_size <= " +
             std::to_string(kTruncatedAnnealingMaxFull);
      return 1;
    }
    if (d.precision != PHI_PREC_FP64) {
      *err = "Hilbert-space truncation of an annealing Hamiltonian runs in FP64 (PHI_PREC_FP64)";
      return 1;
    }
    if (!d.annealing_h_z || !d.transverse_field || !d.longitudinal_field || d.transverse_field_size < 1 ||
        d.longitudinal_field_size < 1) {
      *err = "an annealing Hamiltonian needs H_X, H_Z and both field arrays";
      return 1;
    }
  }
  if (d.truncation_level > 1 || d.time_local) {
    if (d.bath_kind != PHI_BATH_FULL || !d.coupling) {
      *err = "Hilbert-space truncation needs full bath coupling operators (FullBathTerms), as PHI truncates "
             "only those (hierarchy_integrator.cc:1171-1187); a single tier without time-local truncation "
             "takes any";
      return 1;
    }
  }
  // The real symmetric F x F matrix of an interleaved complex one.
  auto real_symmetric = [&](const double *m, const char *what, std::vector<double> *out) {
    out->assign((size_t)F * F, 0.0);
    for (int e = 0; e < F * F; ++e) {
      if (!std::isfinite(m[2 * e]) || m[2 * e + 1] != 0.0) {
        *err = std::string("Hilbert-space truncation is built for real symmetric Hamiltonians (") + what + ")";
        return false;
      }
      (*out)[e] = m[2 * e];
    }
    for (int j = 0; j < F; ++j)
      for (int i = 0; i < j; ++i)
        if ((*out)[i + (size_t)j * F] != (*out)[j + (size_t)i * F]) {
          *err = std::string("the Hamiltonian is not symmetric (") + what + ")";
          return false;
        }
    return true;
  };
  std::vector<double> H;
  if (annealing) {
    // The truncator is first updated with H at alpha = 0, where PHI's
    // splines return the first samples (hierarchy_integrator.cc:934-946).
    if (!real_symmetric(d.annealing_h_x, "H_X", &t->hx_full) ||
        !real_symmetric(d.annealing_h_z, "H_Z", &t->hz_full))
      return 1;
    const double fx = d.transverse_field[0], fz = d.longitudinal_field[0];
    H.resize((size_t)F * F);
    for (int e = 0; e < F * F; ++e) H[e] = fx * t->hx_full[e] + fz * t->hz_full[e];
  } else if (!real_symmetric(d.hamiltonian, "H", &H)) {
    return 1;
  }
  std::vector<double> w(F), V((size_t)F * F);
  if (jacobi_eigh(F, H.data(), w.data(), V.data()) != 0) {
    *err = "Jacobi eigenvalue iteration did not converge";
    return 1;
  }
  double scale = 0.0;
  for (double x : w) scale = std::max(scale, std::fabs(x));
  if (k < F && w[k] - w[k - 1] <= 1e-12 * std::max(scale, 1.0)) {
    *err = "eigenvalues k and k+1 of the Hamiltonian are degenerate: the truncated subspace is not determined";
    return 1;
  }
  t->basis.assign(V.begin(), V.begin() + (size_t)F * k);
  t->eigenvalues.assign(w.begin(), w.begin() + k);
  if (annealing) {
    std::vector<double> c((size_t)2 * F * F, 0.0);
    for (int e = 0; e < F * F; ++e) c[2 * (size_t)e] = t->hx_full[e];
    project(F, k, c.data(), t->basis.data(), &t->hx_k);
    for (int e = 0; e < F * F; ++e) c[2 * (size_t)e] = t->hz_full[e];
    project(F, k, c.data(), t->basis.data(), &t->hz_k);
  } else {
    project(F, k, d.hamiltonian, t->basis.data(), &t->hamiltonian);
  }
  project(F, k, d.initial_density_matrix, t->basis.data(), &t->initial_density_matrix);
  t->coupling.clear();
  if (d.bath_kind == PHI_BATH_FULL && d.coupling) {
    std::vector<double> b(2 * (size_t)F * F, 0.0), bk;
    t->coupling.resize((size_t)d.num_baths * k * k);
    for (int m = 0; m < d.num_baths; ++m) {
      for (int e = 0; e < F * F; ++e) b[2 * (size_t)e] = d.coupling[(size_t)m * F * F + e];
      project(F, k, b.data(), t->basis.data(), &bk);
      for (int e = 0; e < k * k; ++e) t->coupling[(size_t)m * k * k + e] = bk[2 * (size_t)e];
    }
  }
  t->desc = d;
  t->desc.hilbert_space_size = k;
  t->desc.hamiltonian = annealing ? nullptr : t->hamiltonian.data();
  if (annealing) {
    t->desc.annealing_h_x = t->hx_k.data();
    t->desc.annealing_h_z = t->hz_k.data();
  }
  t->desc.initial_density_matrix = t->initial_density_matrix.data();
  t->desc.coupling = t->coupling.empty() ? nullptr : t->coupling.data();
  if (d.truncation_level == 1 && !d.time_local) {
    // A single tier without time-local truncation is PHI's Vacuum updater:
    // no bath operator is read.
    t->desc.bath_kind = PHI_BATH_INDEPENDENT;
    t->desc.coupling = nullptr;
    t->desc.bath_sites = nullptr;
  }
  return 0;
}

void untruncate(int F, int k, const double *V, const double *rho_k, double *rho_full) {
  // V rho V^+, V real F x k.
  std::vector<double> rv(2 * (size_t)k * F, 0.0);  // rho V^T, k x F
  for (int j = 0; j < F; ++j)
    for (int l = 0; l < k; ++l) {
      const double vj = V[j + (size_t)l * F];
      for (int i = 0; i < k; ++i) {
        rv[2 * (i + (size_t)j * k)] += rho_k[2 * (i + (size_t)l * k)] * vj;
        rv[2 * (i + (size_t)j * k) + 1] += rho_k[2 * (i + (size_t)l * k) + 1] * vj;
      }
    }
  for (int j = 0; j < F; ++j)
    for (int i = 0; i < F; ++i) {
      double re = 0.0, im = 0.0;
      for (int l = 0; l < k; ++l) {
        const double vi = V[i + (size_t)l * F];
        re += vi * rv[2 * (l + (size_t)j * k)];
        im += vi * rv[2 * (l + (size_t)j * k) + 1];
      }
      rho_full[2 * (i + (size_t)j * F)] = re;
      rho_full[2 * (i + (size_t)j * F) + 1] = im;
    }
}

}  // namespace phi
