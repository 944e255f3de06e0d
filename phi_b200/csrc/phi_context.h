// phi_context.h -- the opaque phi_ctx of the C ABI (internal).
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_device.cuh"
#include "heom_internal.h"
#include "heom_kernels.h"
#include "heom_tile.h"

// Device copies of the per-term / per-element constants (HeomConsts points here).
struct PhiConstBuffers {
  phi::DeviceBuffer H, corr, nu, sq_next, sq_prev, term_site, site_ptr, site_terms,
      mats_elem, bath_V, mats_bath, pair_i, pair_j, err_flag, deph_node;
};

struct phi_ctx {
  phi_problem_desc desc{};             // scalar fields; array pointers cleared
  std::vector<double> hamiltonian;     // 2*N*N
  std::vector<double> rho_init;        // 2*N*N
  std::vector<double> gamma, lambda;   // num_baths
  std::vector<double> coupling;        // diagonal / full operators
  std::vector<int32_t> bath_sites;     // independent: site of each bath
  std::vector<std::complex<double>> corr;
  std::vector<double> delta;

  cudaStream_t stream = nullptr;
  int num_sms = 148;
  int grid = 1;
  phi::DeviceHierarchy hier;
  PhiConstBuffers cbuf;
  phi::HeomConsts c{};

  // State and integrator work space (node-major).  y, y_alt and acc are
  // complex128; the stage inputs and k buffers are complex128, or complex64
  // with the node stride padded to even in mixed precision, where y32 /
  // y32_alt hold complex64 copies of y / y_alt.
  phi::DeviceBuffer y;         // current state
  phi::DeviceBuffer y_alt;     // RKF45 candidate state
  phi::DeviceBuffer y32, y32_alt;
  phi::DeviceBuffer xa, xb;    // stage inputs (ping-pong)
  phi::DeviceBuffer acc;       // RK4 accumulator
  phi::DeviceBuffer kbuf[5];   // RKF45 k0..k4
  phi::DeviceBuffer ctl;       // Rkf45Ctl / Rk4Ctl
  phi::DeviceBuffer traj;      // rho_0 rows
  // Filtering (c.filtered): active flags, M bytes each.  Between calls the
  // flags of the current state are in active[0].
  phi::DeviceBuffer active[2];
  // Time-local truncation (c.time_local): Q_{m,k} and the sums Q_m, with the
  // copies RKF45 stores and restores (see heom_timelocal.cu).
  phi::DeviceBuffer tl_qk, tl_qk_st, tl_q, tl_q_st;
  // Annealing Hamiltonian (desc.annealing_h_x set): H_X, H_Z, the two
  // splines' coefficients and the update state (see heom_anneal.cu); the
  // stage kernels read H from cbuf.H.
  bool annealing = false;
  phi::DeviceBuffer an_hx, an_hz, an_spline, an_state;
  int an_nx = 0, an_nz = 0;
  int work_level = 0;          // 1: xa/xb, 2: + acc, 3: + RKF45 buffers

  // Captured step graphs.
  cudaGraphExec_t rk4_graph = nullptr;
  int rk4_graph_steps = 0;
  double rk4_graph_dt = 0.0;
  void *rk4_graph_traj = nullptr;
  cudaGraphExec_t rkf45_graph = nullptr;   // kGraphSteps steps
  cudaGraphExec_t rkf45_graph1 = nullptr;  // one step
  int rkf45_graph_steps = 0;

  // Steady-state solve: x, rhat, b, r_0..r_ell, u_0..u_ell (complex128 state
  // size each, one allocation) and the device scalar block; the captured
  // graph replays outer iterations for bicg_ell.
  phi::DeviceBuffer bicg_vecs;
  phi::DeviceBuffer bicg_sc;
  // Per-tile partial sums of <rhat, A v> from the tiled FP64 apply (two
  // arrays of bicg_tiles doubles); empty where the generic kernel applies.
  phi::DeviceBuffer bicg_parts;
  long long bicg_tiles = 0;
  int bicg_ell = 0;
  int bicg_defl = 0;  // deflated tiers the graph was captured with
  cudaGraphExec_t bicg_graph = nullptr;
  // Deflation of the steady-state solve (heom_deflate.cu): requested tiers
  // (-1 automatic, 0 off) and the buffer of A Z, E^-1, g, c and the status.
  int steady_defl = -1;
  phi::DeviceBuffer defl_buf;

  // RKF45 test hooks: forced accept decisions and the per-attempt error
  // trace (phi_gpu_debug_set_rkf45_replay).
  phi::DeviceBuffer rkf45_forced, rkf45_trace;
  long long rkf45_forced_len = 0, rkf45_trace_cap = 0;

  // RKF45 state kept between calls (phi_gpu_rkf45_advance with dt0 <= 0).
  phi::Rkf45Ctl rkf45_last{};
  bool rkf45_started = false;
  void *host_ctl = nullptr;        // pinned copy of the control block
  long long graph_launches = 0;    // step graphs launched so far

  // Hilbert-space truncation: the full size F and the kept eigenvectors V
  // (F x num_states, real); hilbert_full == num_states without truncation.
  int hilbert_full = 0;
  std::vector<double> trunc_basis;
  // Truncated annealing (ta_F = F > 0): full H_X, H_Z (F x F real), the
  // current basis (F x k), the rotation of the last update (k x k) and its
  // flag, on the device; the bath operators truncated into the initial basis
  // (host, for resets).  The initial basis is trunc_basis.
  int ta_F = 0;
  phi::DeviceBuffer ta_hx, ta_hz, ta_V, ta_R, ta_rotate;
  std::vector<double> ta_bath0;

  // Schedule of the tiled stage kernel chosen at creation (tile-eligible
  // problems of at least kTuneMinElements elements; the choice is also in
  // c.tile_variant / c.tile_cps).
  phi::TileSchedule tile_sched{};

  double time = 0.0;
  std::string error;
  ~phi_ctx() {
    if (host_ctl) phi::cached_host_free(host_ctl, sizeof(phi::Rkf45Ctl));
  }

  size_t state_bytes() const {
    return (size_t)hier.M * desc.num_states * desc.num_states * sizeof(double2);
  }
  bool mixed() const { return desc.precision == PHI_PREC_MIXED; }
  // Node stride (elements) and bytes of the stage / k buffers.
  int work_stride() const;
  size_t work_bytes() const;
  int ensure_work(int level);
  void release_graphs();
  // PHI_E_TIMEOUT if a kernel's bounded wait gave up since the last check.
  int check_device_flag();
  int check_device_flag_on(cudaStream_t s);  // after the work queued on s
  // Marks every node active (a newly set state), enqueued on `stream`.
  cudaError_t reset_filter();
  // Points a stage launch at the flag buffers (no-op when filtering is off).
  void bind_filter(phi::StageLaunch &L, int par) const;
  // Zeroes the time-local truncation matrices (a newly set state).
  cudaError_t reset_time_local();
  // Enqueues one update of the time-local matrices (no-op when off).
  cudaError_t enqueue_time_local(int op, int stage, double h, cudaStream_t s);
  // Annealing: H zero and the update state of a fresh run.
  cudaError_t reset_annealing();
  // Enqueues one annealing update (no-op without annealing).
  cudaError_t enqueue_anneal(int op, int which, double dt, cudaStream_t s);
  // Truncated annealing: rotates the listed live ADO arrays (complex128, M
  // nodes each) and, with rkf45_y, the current RKF45 state into the basis
  // of the last update (no-op without truncation or when it kept the basis).
  cudaError_t enqueue_anneal_rotate(std::initializer_list<void *> bufs, bool rkf45_y, cudaStream_t s);
};

namespace phi {
int setup_constants(phi_ctx *ctx);
}
