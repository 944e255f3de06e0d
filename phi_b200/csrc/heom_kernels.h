// heom_kernels.h -- launch interface of the HEOM stage kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include "heom_device.cuh"

namespace phi {

enum StageMode : int { kModeApply = 0, kModeRk4 = 1, kModeRkf45 = 2 };

// Everything one stage launch needs; pointers are device pointers.
struct StageLaunch {
  HeomConsts c;
  int mode = kModeApply;
  int stage = 0;
  int grid = 1;
  const double2 *x = nullptr;   // stage input
  double2 *out = nullptr;       // apply output / next stage input
  double2 *y = nullptr;         // RK4 state
  double2 *acc = nullptr;       // RK4 accumulator
  double a_next = 0.0;          // RK4: X_{s+1} = y + a_next k_s
  double w_acc = 0.0;           // RK4: accumulator weight of k_s
  Rk4Ctl *rk4 = nullptr;
  double2 *traj = nullptr;      // RK4 rho_0 trajectory rows
  double2 *k[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // RKF45 k0..k4
  double2 *ybuf[2] = {nullptr, nullptr};                          // RKF45 state ping-pong
  Rkf45Ctl *ctl = nullptr;
  // Filtering (c.filtered): active flags of the current state in
  // act[act_par] (RKF45: act[ycur], chosen on the device); the stage that
  // writes the new state writes its flags to the other buffer.
  uint8_t *act[2] = {nullptr, nullptr};
  int act_par = 0;
  // FP64 apply of the steady-state solver (tiled kernel): element (0,0) of
  // node 0 of the output is zeroed and each tile writes its share of
  // <dot_w, out> to dot_part[tile].
  const double2 *dot_w = nullptr;
  double *dot_part = nullptr;
  // The generic kernel even where the tiled one applies (with c.M lowered,
  // the rows of the first c.M nodes only; neighbour ids index the whole x).
  bool generic = false;
  // Generic kernel, apply mode: `batch` inputs at x + i * x_bstride, outputs
  // at out + i * out_bstride (complex elements).
  int batch = 1;
  long long x_bstride = 0, out_bstride = 0;
  // Tiled kernel: stage input / output and k buffers in the context's
  // storage type (complex128, or complex64 in mixed precision), the
  // complex64 copies of the state, and the arithmetic.
  bool mixed = false;
  const void *xv = nullptr;
  void *outv = nullptr;
  void *kv[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  void *y32 = nullptr;
  void *y32buf[2] = {nullptr, nullptr};
};

int choose_group(int N);
size_t stage_smem_bytes(int N, int T, int kind);
int stage_grid(const HeomConsts &c, int num_sms);
cudaError_t launch_stage(const StageLaunch &L, cudaStream_t stream);
cudaError_t launch_rkf45_control(Rkf45Ctl *ctl, cudaStream_t stream);
// complex128 (node stride N*N) <-> complex64 (node stride `padded`).
cudaError_t launch_to_c64(const double2 *in, float2 *out, long long M, int E, int padded, cudaStream_t s);
cudaError_t launch_to_c128(const float2 *in, double2 *out, long long M, int E, int padded, cudaStream_t s);

// Small hierarchies (heom_small.cu): a whole FP64 RK4 run in one CTA with
// the state in shared memory.  Eligible: IndependentBath or DiagonalBath
// couplings the tiled kernel does not take, no filtering or time-local
// truncation, at most kSmallMaxElements complex elements.  The caller excludes annealing and
// mixed-precision contexts.  `steps` RK4 steps of dt on y in place, rho_0
// rows and the step / row counters kept in rk4 as the stage kernels keep them.
constexpr long long kSmallMaxElements = 2048;
constexpr size_t kSmallMaxSmem = 200 * 1024;
bool small_rk4_eligible(const HeomConsts &c);
cudaError_t launch_small_rk4(const HeomConsts &c, double2 *y, double dt, long long steps, Rk4Ctl *rk4,
                             double2 *traj, cudaStream_t stream);

}  // namespace phi
