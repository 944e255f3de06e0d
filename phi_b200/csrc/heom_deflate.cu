// heom_deflate.cu -- deflation of the steady-state BiCGSTAB(ell) by the low
// tiers of the hierarchy.
//
// The eliminated steady-state system A x = b (heom_bicgstab.cu) has a few
// eigenvalues close to zero -- population transfer between weakly coupled
// parts of the system, which lives in rho_0 and the first tiers -- and they,
// not the initial error, set the iteration count of the plain solver.  The
// deflated solver works on the complement of the space Z spanned by the real
// coordinates of the ADOs of tiers 0..tiers-1 (element (0,0) of node 0
// excluded; it is eliminated already):
//
//   E = Z^T A Z,  P = I - A Z E^-1 Z^T,
//   BiCGSTAB(ell) on P A y = P b, then x = y + Z E^-1 Z^T (b - A y),
//
// which has the same solution and the same residual b - A x = P (b - A y),
// so the stopping test is unchanged (Nicolaides, SIAM J. Numer. Anal. 24,
// 1987; the DEF1 form of Tang, Nabben, Vuik and Erlangga, J. Sci. Comput. 39,
// 2009).  Z is a set of unit vectors, so Z^T v is a gather of k coordinates
// and A Z is supported on the nodes of tiers 0..tiers: a projection is one
// small solve with E and one rows x k product, both L2-resident.  A Z is
// built once per solve by one batched launch of the generic Liouvillian
// kernel over those nodes (k unit inputs).  First-tier nodes are not
// neighbours of one another, so E = [[A00, A01], [A10, D]] with D block
// diagonal; E is kept factored through the Schur complement
// S = A00 - A01 D^-1 A10 of rho_0's coordinates.
//
// Coordinates follow the real vector space of Hermitian hierarchies the
// solver runs on: the inner product is sum Re(conj(a) b) over every element,
// and coordinate q of node m = q / N^2 is element l = q % N^2 at
// (i, j) = (l % N, l / N) of the column-major ADO: i == j the diagonal
// element (Z_q = E_ii), i < j the real part of pair (i, j)
// (Z_q = E_ij + E_ji), i > j the imaginary part of pair (j, i)
// (Z_q = i E_ji - i E_ij).
#include <cuda_runtime.h>

#include "heom_bicgstab.h"
#include "heom_deflate.h"

namespace phi {
namespace {

constexpr int kBlock = 256;
constexpr int kSolveBlock = 1024;
// Matrices of the factorisation up to this many doubles are inverted in
// shared memory, larger ones in the global work buffer (L2).
constexpr int kSmemDoubles = 16384;
// The projection's factors are staged in shared memory up to this size.
constexpr int kStageDoubles = 24576;

__device__ __forceinline__ double cdot_re(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

// Coordinate q >= 1 of the hierarchy: node base, the pair (a, b) with
// a <= b and which of its parts (0 diagonal, 1 real, 2 imaginary).
struct Coord {
  long long base;
  int a, b, part;
};

__device__ __forceinline__ Coord coord_of(int q, int N) {
  const int E = N * N;
  const int m = q / E, l = q - m * E;
  const int i = l % N, j = l / N;
  Coord c;
  c.base = (long long)m * E;
  c.a = i < j ? i : j;
  c.b = i < j ? j : i;
  c.part = i == j ? 0 : (i < j ? 1 : 2);
  return c;
}

// <Z_q, v>.
__device__ __forceinline__ double zcoord(const double2 *v, const Coord &c, int N) {
  const double2 ab = v[c.base + c.a + (long long)c.b * N];
  if (c.part == 0) return ab.x;
  const double2 ba = v[c.base + c.b + (long long)c.a * N];
  return c.part == 1 ? ab.x + ba.x : ab.y - ba.y;
}

// Entry (p, q) of E = Z^T A Z (deflated coordinates p, q in [0, k)).
__device__ __forceinline__ double galerkin(const DeflView &D, int p, int q) {
  return zcoord(D.AZ + (long long)q * D.rows, coord_of(p + 1, D.N), D.N);
}

// Z_j into units + j * unit_len (the buffer is zero on entry).
__global__ void units_kernel(DeflView D) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.k) return;
  const Coord c = coord_of(j + 1, D.N);
  double2 *s = D.units + (long long)j * D.unit_len;
  double2 *ab = s + c.base + c.a + (long long)c.b * D.N;
  double2 *ba = s + c.base + c.b + (long long)c.a * D.N;
  if (c.part == 0) {
    *ab = make_double2(1.0, 0.0);
  } else if (c.part == 1) {
    *ab = make_double2(1.0, 0.0);
    *ba = make_double2(1.0, 0.0);
  } else {
    *ab = make_double2(0.0, 1.0);
    *ba = make_double2(0.0, -1.0);
  }
}

// AZr = A Z row-major, element (0,0) of node 0 (row 0) zeroed.
__global__ void transpose_kernel(DeflView D) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D.rows * D.k) return;
  const long long r = idx / D.k;
  const int j = (int)(idx - r * D.k);
  D.AZr[idx] = r == 0 ? make_double2(0.0, 0.0) : D.AZ[(long long)j * D.rows + r];
}

// In-place inverse of the n x n row-major matrix A (shared or global
// memory) by the whole CTA: Gauss-Jordan elimination with partial pivoting
// (largest |pivot| in the column, the lowest row on ties); the row
// exchanges become column exchanges of the inverse, undone last step first.
// Returns false in every thread if a pivot is zero or not finite.
__device__ bool cta_invert(double *A, int n, int *swaps, double *prow, double *pcol, double *wv, int *wi,
                           int *bad) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) *bad = 0;
  __syncthreads();
  for (int p = 0; p < n; ++p) {
    double best = -1.0;
    int bi = n;
    for (int r = p + tid; r < n; r += nt) {
      const double v = fabs(A[r * n + p]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if ((tid & 31) == 0) {
      wv[tid >> 5] = best;
      wi[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double b = -1.0;
      int r = n;
      for (int w = 0; w < nt / 32; ++w)
        if (wv[w] > b || (wv[w] == b && wi[w] < r)) {
          b = wv[w];
          r = wi[w];
        }
      if (!(b > 0.0) || !(b - b == 0.0) || r >= n) *bad = 1;
      swaps[p] = r;
    }
    __syncthreads();
    if (*bad) return false;
    const int r = swaps[p];
    if (r != p)
      for (int j = tid; j < n; j += nt) {
        const double t = A[p * n + j];
        A[p * n + j] = A[r * n + j];
        A[r * n + j] = t;
      }
    __syncthreads();
    const double inv = 1.0 / A[p * n + p];
    for (int j = tid; j < n; j += nt) {
      prow[j] = (j == p ? 1.0 : A[p * n + j]) * inv;
      pcol[j] = A[j * n + p];
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += nt) {
      const int i = idx / n, j = idx - i * n;
      A[idx] = i == p ? prow[j] : (j == p ? 0.0 : A[idx]) - pcol[i] * prow[j];
    }
    __syncthreads();
  }
  for (int p = n - 1; p >= 0; --p) {
    const int r = swaps[p];
    if (r != p)
      for (int i = tid; i < n; i += nt) {
        const double t = A[i * n + p];
        A[i * n + p] = A[i * n + r];
        A[i * n + r] = t;
      }
    __syncthreads();
  }
  return true;
}

// In-place inverse of the n x n row-major matrix A (n <= 32, shared
// memory) by one warp, the same elimination as cta_invert: lane c owns
// column c during the elimination and row c during the column exchanges.
// Returns false in every lane if a pivot is zero or not finite.
__device__ bool warp_invert(double *A, int n, int *swaps) {
  const int lane = threadIdx.x & 31;
  for (int p = 0; p < n; ++p) {
    double best = lane >= p && lane < n ? fabs(A[lane * n + p]) : -1.0;
    int bi = lane >= p && lane < n ? lane : n;
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (!(best > 0.0) || !(best - best == 0.0) || bi >= n) return false;  // uniform: every lane holds the result
    if (lane == 0) swaps[p] = bi;
    if (lane < n && bi != p) {
      const double t = A[p * n + lane];
      A[p * n + lane] = A[bi * n + lane];
      A[bi * n + lane] = t;
    }
    __syncwarp();
    const double inv = 1.0 / A[p * n + p];
    const double prow = lane < n ? (lane == p ? 1.0 : A[p * n + lane]) * inv : 0.0;
    const double pcol = lane < n ? A[lane * n + p] : 0.0;
    __syncwarp();
    for (int i = 0; i < n; ++i) {
      const double f = __shfl_sync(0xffffffffu, pcol, i);
      if (lane < n) A[i * n + lane] = i == p ? prow : (lane == p ? 0.0 : A[i * n + lane]) - f * prow;
    }
    __syncwarp();
  }
  for (int p = n - 1; p >= 0; --p) {
    const int r = swaps[p];
    if (lane < n && r != p) {
      const double t = A[lane * n + p];
      A[lane * n + p] = A[lane * n + r];
      A[lane * n + r] = t;
    }
    __syncwarp();
  }
  return true;
}

// Factors E = Z^T A Z: A01, the inverses of the first-tier blocks of D,
// F = D^-1 A10 and the inverse of S = A00 - A01 F.  One CTA; matrices of at
// most kSmemDoubles entries are inverted in shared memory (mat_s).
__global__ void __launch_bounds__(kSolveBlock) factor_kernel(DeflView D) {
  extern __shared__ double mat_s[];
  __shared__ double prow[kMaxDeflK], pcol[kMaxDeflK], wv[kSolveBlock / 32];
  __shared__ int swaps[kMaxDeflK], wi[kSolveBlock / 32], bad;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int E = D.E, k0 = D.k0, n1 = D.n1, t1 = n1 / E;
  for (int idx = tid; idx < k0 * n1; idx += nt) {
    const int p = idx / n1, i = idx - p * n1;
    D.A01[idx] = galerkin(D, p, k0 + i);
  }
  const int regions = t1 < nw ? t1 : nw;
  if (E <= 32 && regions * E * E <= kSmemDoubles) {
    // one warp per block, each in its own region of shared memory
    __shared__ int wswaps[kSolveBlock / 32][32];
    if (tid == 0) bad = 0;
    __syncthreads();
    double *Mw = mat_s + warp * E * E;
    for (int a = warp; a < t1; a += nw) {
      const int o = k0 + a * E;
      for (int idx = lane; idx < E * E; idx += 32) Mw[idx] = galerkin(D, o + idx / E, o + idx % E);
      __syncwarp();
      if (!warp_invert(Mw, E, wswaps[warp])) {
        if (lane == 0) bad = 1;
        break;
      }
      for (int idx = lane; idx < E * E; idx += 32) D.Dinv[(long long)a * E * E + idx] = Mw[idx];
      __syncwarp();
    }
    __syncthreads();
    if (bad) {
      if (tid == 0) *D.status = 1;
      return;
    }
  } else {
    double *Mb = E * E <= kSmemDoubles ? mat_s : D.work;
    for (int a = 0; a < t1; ++a) {
      const int o = k0 + a * E;
      for (int idx = tid; idx < E * E; idx += nt) Mb[idx] = galerkin(D, o + idx / E, o + idx % E);
      __syncthreads();
      if (!cta_invert(Mb, E, swaps, prow, pcol, wv, wi, &bad)) {
        if (tid == 0) *D.status = 1;
        return;
      }
      for (int idx = tid; idx < E * E; idx += nt) D.Dinv[(long long)a * E * E + idx] = Mb[idx];
      __syncthreads();
    }
  }
  for (int idx = tid; idx < n1 * k0; idx += nt) {
    const int i = idx / k0, q = idx - i * k0;
    const int o = k0 + (i / E) * E;
    const double *drow = D.Dinv + (long long)i * E;
    double s = 0.0;
    for (int t = 0; t < E; ++t) s = fma(drow[t], galerkin(D, o + t, q), s);
    D.F[idx] = s;
  }
  __syncthreads();
  double *Ms = k0 * k0 <= kSmemDoubles ? mat_s : D.work;
  for (int ent = warp; ent < k0 * k0; ent += nw) {
    const int p = ent / k0, q = ent - p * k0;
    double s = 0.0;
    for (int i = lane; i < n1; i += 32) s = fma(D.A01[(long long)p * n1 + i], D.F[(long long)i * k0 + q], s);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) Ms[ent] = galerkin(D, p, q) - s;
  }
  __syncthreads();
  if (!cta_invert(Ms, k0, swaps, prow, pcol, wv, wi, &bad)) {
    if (tid == 0) *D.status = 1;
    return;
  }
  for (int idx = tid; idx < k0 * k0; idx += nt) D.Si[idx] = Ms[idx];
  if (tid == 0) *D.status = 0;
}

// g_j = <rhat, A Z_j>: one warp per column, lanes in row order.
__global__ void g_kernel(DeflView D, const double2 *rhat) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= D.k) return;
  const double2 *col = D.AZ + (long long)warp * D.rows;
  double s = 0.0;
  for (long long r = lane; r < D.rows; r += 32) s += cdot_re(rhat[r], col[r]);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) D.g[warp] = s;
}

// c = E^-1 Z^T (v - b) through the factors: w = D^-1 z1,
// c0 = S^-1 (z0 - A01 w), c1 = w - F c0; *part = -<g, c>.  One CTA.
// The factors (Dinv, F, A01, Si: one contiguous run of doubles) are first
// copied into shared memory when they fit (stage = true).
__device__ __forceinline__ void coeff_body(DeflView D, const double2 *v, const double2 *b, double *part,
                                           bool stage, double *fac_s) {
  __shared__ double z[kMaxDeflK], w[kMaxDeflK], cs[kMaxDeflK];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int E = D.E, k0 = D.k0, n1 = D.n1, k = D.k;
  if (stage) {
    const long long total = (long long)n1 * E + 2ll * n1 * k0 + (long long)k0 * k0;
    for (long long i = tid; i < total; i += nt) fac_s[i] = D.Dinv[i];
    D.Dinv = fac_s;
    D.F = D.Dinv + (long long)n1 * E;
    D.A01 = D.F + (long long)n1 * k0;
    D.Si = D.A01 + (long long)k0 * n1;
  }
  for (int p = tid; p < k; p += nt) {
    const Coord c = coord_of(p + 1, D.N);
    z[p] = zcoord(v, c, D.N) - (b ? zcoord(b, c, D.N) : 0.0);
  }
  __syncthreads();
  for (int i = tid; i < n1; i += nt) {
    const double *drow = D.Dinv + (long long)i * E;
    const double *zb = z + k0 + (i / E) * E;
    double s = 0.0;
#pragma unroll 8
    for (int t = 0; t < E; ++t) s = fma(drow[t], zb[t], s);
    w[i] = s;
  }
  __syncthreads();
  for (int p = warp; p < k0; p += nw) {  // z0 -> z0 - A01 w
    double s = 0.0;
    for (int i = lane; i < n1; i += 32) s = fma(D.A01[(long long)p * n1 + i], w[i], s);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) z[p] -= s;
  }
  __syncthreads();
  for (int p = warp; p < k0; p += nw) {
    double s = 0.0;
    for (int q = lane; q < k0; q += 32) s = fma(D.Si[(long long)p * k0 + q], z[q], s);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) cs[p] = s;
  }
  __syncthreads();
  for (int i = tid; i < n1; i += nt) {
    const double *frow = D.F + (long long)i * k0;
    double s = 0.0;
#pragma unroll 8
    for (int q = 0; q < k0; ++q) s = fma(frow[q], cs[q], s);
    cs[k0 + i] = w[i] - s;
  }
  __syncthreads();
  for (int j = tid; j < k; j += nt) D.c[j] = cs[j];
  if (part && warp == 0) {
    double s = 0.0;
    for (int j = lane; j < k; j += 32) s = fma(D.g[j], cs[j], s);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) *part = -s;
  }
}

__global__ void __launch_bounds__(kSolveBlock) coeff_kernel(DeflView D, const double2 *v, const double2 *b,
                                                          double *part, bool stage) {
  extern __shared__ double fac_s[];
  if (D.done && *(volatile const int *)D.done) return;  // uniform: the solve has stopped
  coeff_body(D, v, b, part, stage, fac_s);
}

// The coefficients of v's projection, then the BiCG scalar step of the
// inner product whose per-tile partials the apply left in parts[0..nparts-1]
// (the projection's change is parts[nparts-1] = *part): one launch instead
// of a coefficient kernel and a one-block finish.  Summed in part order.
__global__ void __launch_bounds__(kSolveBlock) coeff_finish_kernel(DeflView D, const double2 *v, double *part,
                                                                 const double *parts, long long nparts,
                                                                 BicgScalars *sc, int which, bool stage) {
  extern __shared__ double fac_s[];
  __shared__ double red[kSolveBlock / 32];
  if (D.done && *(volatile const int *)D.done) return;  // uniform: the solve has stopped
  coeff_body(D, v, nullptr, part, stage, fac_s);
  __syncthreads();  // *part is visible to the whole CTA
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double s = 0.0;
  for (long long i = threadIdx.x; i < nparts; i += blockDim.x) s += parts[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
    bicg_dot_step(sc, tot, which);
  }
}

// v[r] -= sum_j A Z[r, j] c_j for the rows of tiers 0..tiers: one warp per
// row of the row-major copy, lanes over j.
__global__ void update_kernel(DeflView D, double2 *v) {
  __shared__ double cs[kMaxDeflK];
  if (D.done && *(volatile const int *)D.done) return;
  for (int j = threadIdx.x; j < D.k; j += blockDim.x) cs[j] = D.c[j];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= D.rows) return;
  const double2 *row = D.AZr + r * D.k;
  double sx = 0.0, sy = 0.0;
  for (int j = lane; j < D.k; j += 32) {
    const double2 a = row[j];
    sx = fma(a.x, cs[j], sx);
    sy = fma(a.y, cs[j], sy);
  }
  for (int off = 16; off > 0; off >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, off);
    sy += __shfl_xor_sync(0xffffffffu, sy, off);
  }
  if (lane == 0) {
    const double2 x = v[r];
    v[r] = make_double2(x.x - sx, x.y - sy);
  }
}

// x -= Z c; the real and imaginary parts of a pair belong to different
// coordinates, so every thread writes its own doubles.
__global__ void correct_kernel(DeflView D, double2 *x) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= D.k) return;
  const Coord c = coord_of(p + 1, D.N);
  const double cv = D.c[p];
  double *ab = reinterpret_cast<double *>(x + c.base + c.a + (long long)c.b * D.N);
  double *ba = reinterpret_cast<double *>(x + c.base + c.b + (long long)c.a * D.N);
  if (c.part == 0) {
    ab[0] -= cv;
  } else if (c.part == 1) {
    ab[0] -= cv;
    ba[0] -= cv;
  } else {
    ab[1] -= cv;
    ba[1] += cv;
  }
}

}  // namespace

cudaError_t defl_launch_units(const DeflView &D, cudaStream_t st) {
  units_kernel<<<(D.k + kBlock - 1) / kBlock, kBlock, 0, st>>>(D);
  return cudaGetLastError();
}

cudaError_t defl_launch_factor(const DeflView &D, cudaStream_t st) {
  if (D.k < 1 || D.k > kMaxDeflK || D.k0 + D.n1 != D.k || (D.n1 && D.n1 % D.E)) return cudaErrorInvalidValue;
  const long long total = D.rows * D.k;
  transpose_kernel<<<(unsigned)((total + kBlock - 1) / kBlock), kBlock, 0, st>>>(D);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int big = D.E > D.k0 ? D.E : D.k0;
  const int t1 = D.n1 / D.E, regions = t1 < kSolveBlock / 32 ? t1 : kSolveBlock / 32;
  long long need = (long long)big * big;
  if (D.E <= 32 && (long long)regions * D.E * D.E <= kSmemDoubles && (long long)regions * D.E * D.E > need)
    need = (long long)regions * D.E * D.E;  // one region per warp for the first-tier blocks
  const size_t smem = (size_t)(need < kSmemDoubles ? need : kSmemDoubles) * sizeof(double);
  e = cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  factor_kernel<<<1, kSolveBlock, smem, st>>>(D);
  return cudaGetLastError();
}

cudaError_t defl_launch_g(const DeflView &D, const double2 *rhat, cudaStream_t st) {
  const int warps_per_block = kBlock / 32;
  g_kernel<<<(D.k + warps_per_block - 1) / warps_per_block, kBlock, 0, st>>>(D, rhat);
  return cudaGetLastError();
}

cudaError_t defl_launch_coeff(const DeflView &D, const double2 *v, const double2 *b, double *part, cudaStream_t st) {
  const long long total = (long long)D.n1 * D.E + 2ll * D.n1 * D.k0 + (long long)D.k0 * D.k0;
  const bool stage = total <= kStageDoubles;
  const size_t smem = stage ? (size_t)total * sizeof(double) : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(coeff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kStageDoubles * sizeof(double)));
    if (e != cudaSuccess) return e;
  }
  coeff_kernel<<<1, kSolveBlock, smem, st>>>(D, v, b, part, stage);
  return cudaGetLastError();
}

cudaError_t defl_launch_coeff_finish(const DeflView &D, const double2 *v, double *part, const double *parts,
                                     long long nparts, BicgScalars *sc, int which, cudaStream_t st) {
  const long long total = (long long)D.n1 * D.E + 2ll * D.n1 * D.k0 + (long long)D.k0 * D.k0;
  const bool stage = total <= kStageDoubles;
  const size_t smem = stage ? (size_t)total * sizeof(double) : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(coeff_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kStageDoubles * sizeof(double)));
    if (e != cudaSuccess) return e;
  }
  coeff_finish_kernel<<<1, kSolveBlock, smem, st>>>(D, v, part, parts, nparts, sc, which, stage);
  return cudaGetLastError();
}

cudaError_t defl_launch_update(const DeflView &D, double2 *v, cudaStream_t st) {
  const int rows_per_block = kBlock / 32;
  update_kernel<<<(unsigned)((D.rows + rows_per_block - 1) / rows_per_block), kBlock, 0, st>>>(D, v);
  return cudaGetLastError();
}

cudaError_t defl_launch_correct(const DeflView &D, double2 *x, cudaStream_t st) {
  correct_kernel<<<(D.k + kBlock - 1) / kBlock, kBlock, 0, st>>>(D, x);
  return cudaGetLastError();
}

}  // namespace phi
