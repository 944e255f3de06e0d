// phi_truncation.h -- Hilbert-space truncation of a problem (internal;
// phi_truncation.cpp).
#pragma once

#include <string>
#include <vector>

#include "../../include/phi_b200.h"

namespace phi {

// Largest hilbert_space_size of a truncated annealing run (the device
// eigensolver of heom_anneal.cu works on one warp).
constexpr int kTruncatedAnnealingMaxFull = 32;

// Eigenvalues (ascending) and orthonormal eigenvectors (columns, same order)
// of a real symmetric n x n matrix, column-major.  0 on success.
int jacobi_eigh(int n, const double *a, double *w, double *v);

// A problem given in the full space (desc.hilbert_space_size = F >
// desc.num_states = k) restated in the basis of the lowest k eigenvectors of
// its Hamiltonian; desc is the k-dimensional descriptor (arrays point into
// this object).
// For an annealing Hamiltonian the basis is that of H(0) = f_x(0) H_X +
// f_z(0) H_Z; the device re-diagonalises at every update from hx_full /
// hz_full (F x F real), and desc carries H_X, H_Z projected into the initial
// basis only so the k-dimensional context can be created.
struct TruncatedProblem {
  int full = 0;
  std::vector<double> basis;        // V: F x k, real, column-major
  std::vector<double> eigenvalues;  // k
  std::vector<double> hamiltonian, initial_density_matrix, coupling;
  std::vector<double> hx_full, hz_full;  // annealing: F x F real
  std::vector<double> hx_k, hz_k;        // annealing: projected, complex k x k
  phi_problem_desc desc{};
};
int truncate_problem(const phi_problem_desc &d, TruncatedProblem *t, std::string *err);

// rho_full = V rho_k V^+ (interleaved complex, column-major).
void untruncate(int F, int k, const double *V, const double *rho_k, double *rho_full);

}  // namespace phi
