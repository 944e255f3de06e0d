// heom_device.cuh -- device-side data layout shared by the HEOM kernels.
//
// HBM layout of one hierarchy instance (all node-major, PHI node-id order):
//   state   : M * N * N complex, column-major per node (PHI's ADO layout,
//             hierarchy_integrator.cc:1022-1027 contiguous per thread block)
//   mi      : M * T uint8   multi-index n_t of every node
//   next    : M * T int32   id of node + e_t, -1 when absent
//   prev    : M * T int32   id of node - e_t, -1 when absent
// Per-term and per-element constants are a few KB and stay L1/L2 resident.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phi {

constexpr int kMaxStates = 64;   // N limit (multi-index and smem sizing)
constexpr int kMaxTerms = 64;    // T limit
constexpr int kMaxTier = 250;    // L limit (multi-index stored as uint8)

enum BathKind : int { kIndependent = 0, kDiagonal = 1, kFull = 2 };

// Raises a kernel's dynamic shared-memory limit to `bytes` when that is above
// the default 48 KiB.  The limit belongs to the function on each device, so
// the largest size set so far is remembered per device ordinal in `seen`
// (one array per kernel, owned by its launcher; ordinals past the array set
// the attribute on every launch).
constexpr int kSmemLimitDevices = 64;
template <class Kernel>
inline cudaError_t raise_smem_limit(Kernel kern, size_t bytes, int (&seen)[kSmemLimitDevices]) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool tracked = dev >= 0 && dev < kSmemLimitDevices;
  if (tracked && seen[dev] >= (int)bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && tracked) seen[dev] = (int)bytes;
  return e;
}

// Read-only problem constants, built on the host once per context.  Mirrors
// what PHI keeps per node (HierarchyNode prefactors, hierarchy_node.h:139-208)
// but stores it per term: the per-node values are recomputed in registers.
struct HeomConsts {
  int N;            // states
  int T;            // terms = baths * (K+1)
  int K1;           // K + 1
  int nb;           // baths
  int L;            // deepest tier (truncation_level - 1)
  int kind;         // BathKind
  int vacuum;       // truncation_level == 1: unitary part only
  int identity_sites;  // independent baths: bath m couples to |m><m|
  int h_real;       // every Hamiltonian element has a zero imaginary part
  int64_t M;        // nodes
  double inv_hbar;  // 1 / hbar
  const uint8_t *mi;     // M*T
  const int32_t *next;   // M*T
  const int32_t *prev;   // M*T
  const double2 *H;      // N*N Hamiltonian
  const double2 *corr;   // T   c_t
  const double *nu;      // T   dephasing rate of term t
  const double *deph_node;  // M (+2 slack): sum_t n_t nu_t of every node
  const double *sq_next; // T*(L+2): |next prefactor| for n_t = 0..L+1
  const double *sq_prev; // T*(L+2): prev scale for n_t = 0..L+1
  const int32_t *term_site;  // T: independent -> site, diagonal/full -> bath
  const int32_t *site_ptr;   // N+1: CSR of the terms coupling to each site
  const int32_t *site_terms; // T
  const double *mats_elem;   // N*N: Matsubara factor per element (indep/diag)
  const double *bath_V;      // diagonal: nb*N, full: nb*N*N (real, col-major)
  const double *mats_bath;   // nb: Delta_b
  const uint8_t *pair_i;     // N(N+1)/2 upper-triangle pairs (i <= j)
  const uint8_t *pair_j;
  int *err_flag;             // set by a kernel whose bounded wait gave up
  // Poll limit of the tile kernels' first wait on a tile's bulk copy: 0 the
  // built-in limit, < 0 give up at once (a test of the timeout path; the
  // drain of the CTA's own copies keeps the built-in limit).
  long long first_wait_polls;
  // Tile-kernel schedule (host side only, chosen by the autotuner):
  // block-size variant (0 the default of the shape, 1 the alternative) and
  // persistent CTAs per SM (0: as many as fit).
  int tile_variant;
  int tile_cps;
  // Adaptive hierarchy filtering (PHI's FilterTolerance, independent baths):
  // a node whose largest |element| drops below filter_tol stops feeding its
  // neighbours until it rises above it again.
  int filtered;
  double filter_tol;
  // Time-local truncation (PHI's TimeLocal, independent baths on the
  // identity site map): nodes of the deepest tier add -[V_m, Q_m X - X Q_m^+]
  // for every bath m (hierarchy_updater.cc:171-190) instead of next terms.
  int time_local;
  const double2 *tl_q;       // nb*N*N: the sums Q_m, column-major per bath
};

// Device control block of the adaptive integrator; lives in device memory and
// is advanced by rkf45_control_kernel between steps.
struct Rkf45Ctl {
  double time;
  double end_time;
  double dt;          // step size of the next attempt
  double tol;
  double min_dt;
  double dtup;        // grow factor (replaced by the last-step clamp ratio)
  double dtdn;        // shrink factor
  double coef[24];    // b10..b54, c50..c54, c60..c65, pre-scaled by dt
  double max_error;   // largest accepted error estimate
  unsigned long long err_bits;  // max |y4 - y5| of the current attempt
  long long steps;
  long long accepted;
  long long max_steps;
  int ycur;           // which y buffer is current
  int done;           // 1 once time >= end_time or the step limit is hit
  int status;         // 0 ok, 1 step limit
  int nonfinite;      // 1 if a non-finite error estimate was seen
  // Time-local truncation: the stage offsets a1..a5 (scaled with dt like
  // coef), and what the last control step did -- 1 accepted (the matrices
  // then advance by tl_h_accept = dt - a5 of that attempt and are stored),
  // 2 rejected (restored), 0 nothing (run already done).
  int tl_pending;
  double a[5];
  double tl_h_accept;
  // Test hooks (null / 0 in normal runs): decisions to take instead of the
  // error test for the first forced_len attempts of a run (0 reject, 1
  // accept, 2 accept and grow the step), and the error estimate of each of
  // the first trace_cap attempts.
  const signed char *forced;
  long long forced_len;
  double *err_trace;
  long long trace_cap;
};

// RK4 device bookkeeping (only the rho_0 trajectory needs it).
struct Rk4Ctl {
  long long step;        // steps completed
  long long out_factor;  // ceil(output_min_step / dt)
  long long capacity;    // trajectory rows available
  long long nout;        // trajectory rows written
  double time;           // annealing Hamiltonian: time_now of the step in flight
};

}  // namespace phi
