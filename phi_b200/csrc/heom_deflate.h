// heom_deflate.h -- deflation of the steady-state solve by the low tiers of
// the hierarchy (internal; kernels in heom_deflate.cu).
#pragma once

#include <cuda_runtime.h>

namespace phi {

struct BicgScalars;

// Largest deflation space: the coordinates of the deflated tiers' ADOs.
constexpr int kMaxDeflK = 256;

// Device view of one deflation space Z: the real coordinates of the ADOs of
// tiers 0..tiers-1 (tiers = 1 or 2) without element (0,0) of node 0 --
// k0 = N^2 - 1 of rho_0, then N^2 of each of the t1 first-tier nodes.  The
// Galerkin matrix Z^T A Z = [[A00, A01], [A10, D]] has a block-diagonal D
// (first-tier nodes are not neighbours of one another) and is kept factored:
// Dinv = D^-1 (t1 blocks of N^2 x N^2), F = D^-1 A10, A01 and
// Si = (A00 - A01 F)^-1.
struct DeflView {
  int N, E;          // states, N^2
  int k, k0, n1;     // coordinates: k = k0 + n1, n1 = t1 * E
  long long rows;    // complex entries of an A Z column (nodes of tiers 0..tiers, times E)
  long long unit_len;  // complex entries of one unit input (nodes of tiers 0..tiers+1, times E)
  double2 *AZ;       // rows x k, one column after another
  double2 *AZr;      // the same, one row after another
  double *Dinv;      // n1 x E: row r of block a at (a * E + r) * E
  double *F;         // n1 x k0
  double *A01;       // k0 x n1
  double *Si;        // k0 x k0
  double *g;         // k: <rhat, A Z_j>
  double *c;         // k: coefficients of the last projection
  double *work;      // scratch of the factorisation: max(k0, E)^2
  int *status;       // 0 ok, 1 the Galerkin matrix is singular
  const int *done;   // the solver's stop flag: projections return at once once it is set (NULL: always run)
  double2 *units;    // k unit inputs of unit_len elements (setup only)
};

// The unit inputs: units + j * unit_len holds Z_j (zeros elsewhere).
cudaError_t defl_launch_units(const DeflView &D, cudaStream_t st);
// After the batched apply wrote A Z: copy it row-major with element (0,0)
// of node 0 zeroed in every column (that equation is dropped; the
// column-major copy is only read at deflated coordinates, which exclude
// it), and factor the Galerkin matrix (one CTA; status 1 if a pivot is zero
// or not finite).
cudaError_t defl_launch_factor(const DeflView &D, cudaStream_t st);
// g_j = <rhat, A Z_j>.
cudaError_t defl_launch_g(const DeflView &D, const double2 *rhat, cudaStream_t st);
// c = (Z^T A Z)^-1 Z^T (v - b) (b may be NULL); with part != NULL also
// *part = -<g, c>, the change of <rhat, v> made by the update below.
cudaError_t defl_launch_coeff(const DeflView &D, const double2 *v, const double2 *b, double *part, cudaStream_t st);
// defl_launch_coeff (without b, part != NULL) followed by the BiCG scalar
// step of the inner product summed from parts[0..nparts-1], whose last
// entry is *part (rho: which = 0, gamma: which = 1), in one launch.
cudaError_t defl_launch_coeff_finish(const DeflView &D, const double2 *v, double *part, const double *parts,
                                     long long nparts, BicgScalars *sc, int which, cudaStream_t st);
// v -= A Z c over the rows of tiers 0..tiers: v becomes P v with
// P = I - A Z (Z^T A Z)^-1 Z^T (after defl_launch_coeff without b), or
// b - v becomes P (b - v) (with b).
cudaError_t defl_launch_update(const DeflView &D, double2 *v, cudaStream_t st);
// x -= Z c: the coarse correction of the final iterate.
cudaError_t defl_launch_correct(const DeflView &D, double2 *x, cudaStream_t st);

}  // namespace phi
