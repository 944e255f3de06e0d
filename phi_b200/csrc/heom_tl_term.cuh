// heom_tl_term.cuh -- the time-local truncation term of one ADO element
// (internal; shared by the tiled and the generic stage kernels).
//
// For an independent bath m on site m, IndependentBath::DoTimelocal
// (hierarchy_updater.cc:171-190) forms X_m = Q_m X - X Q_m^+ and adds its
// column m and subtracts its row m, so element (i, j) of the derivative of a
// deepest-tier ADO X gains X_j[i][j] - X_i[i][j].  With D = Q_j - Q_i and X
// Hermitian that is
//     (D X)_ij - conj((D X)_ji),
// the same shape as the commutator with H; for i == j it vanishes.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace phi {

// Q: nb*N*N sums Q_m, column-major per bath (read through the read-only
// cache; a few KB for the sizes the tile kernel serves).  X: the ADO,
// column-major.  The loop stays rolled so that, inlined into a stage kernel,
// it holds few registers.
template <class TX>
static __device__ __forceinline__ TX tl_pair_term(const TX *X, const double2 *__restrict__ Q, int N, int i, int j) {
  using R = decltype(X->x);
  const size_t E = (size_t)N * N;
  const double2 *Qi = Q + (size_t)i * E, *Qj = Q + (size_t)j * E;
  R ar = 0, ai = 0, br = 0, bi = 0;
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    const double2 qji = __ldg(Qj + i + k * N), qii = __ldg(Qi + i + k * N);
    const double2 qjj = __ldg(Qj + j + k * N), qij = __ldg(Qi + j + k * N);
    const R dir = (R)(qji.x - qii.x), dii = (R)(qji.y - qii.y);  // D[i][k]
    const R djr = (R)(qjj.x - qij.x), dji = (R)(qjj.y - qij.y);  // D[j][k]
    const TX xkj = X[k + j * N], xki = X[k + i * N];
    ar = fma(dir, xkj.x, ar);
    ar = fma(-dii, xkj.y, ar);
    ai = fma(dir, xkj.y, ai);
    ai = fma(dii, xkj.x, ai);
    br = fma(djr, xki.x, br);
    br = fma(-dji, xki.y, br);
    bi = fma(djr, xki.y, bi);
    bi = fma(dji, xki.x, bi);
  }
  TX out;
  out.x = ar - br;  // a - conj(b)
  out.y = ai + bi;
  return out;
}

}  // namespace phi
