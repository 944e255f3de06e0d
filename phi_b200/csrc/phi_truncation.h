// phi_truncation.h -- Hilbert-space truncation of a static problem (internal;
// phi_truncation.cpp).
#pragma once

#include <string>
#include <vector>

#include "../../include/phi_b200.h"

namespace phi {

// Eigenvalues (ascending) and orthonormal eigenvectors (columns, same order)
// of a real symmetric n x n matrix, column-major.  0 on success.
int jacobi_eigh(int n, const double *a, double *w, double *v);

// A problem given in the full space (desc.hilbert_space_size = F >
// desc.num_states = k) restated in the basis of the lowest k eigenvectors of
// its Hamiltonian; desc is the k-dimensional descriptor (arrays point into
// this object).
struct TruncatedProblem {
  int full = 0;
  std::vector<double> basis;        // V: F x k, real, column-major
  std::vector<double> eigenvalues;  // k
  std::vector<double> hamiltonian, initial_density_matrix, coupling;
  phi_problem_desc desc{};
};
int truncate_problem(const phi_problem_desc &d, TruncatedProblem *t, std::string *err);

// rho_full = V rho_k V^+ (interleaved complex, column-major).
void untruncate(int F, int k, const double *V, const double *rho_k, double *rho_full);

}  // namespace phi
