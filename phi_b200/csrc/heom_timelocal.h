// heom_timelocal.h -- time-local truncation matrix updates (internal).
#pragma once

#include <cuda_runtime.h>

#include "heom_device.cuh"

namespace phi {

enum TlOp : int {
  kTlAdvance = 0,     // advance every Q_{m,k} by the step p.h
  kTlRkf45Stage = 1,  // RKF45 before stage p.stage (1..5), steps from the control block
  kTlRkf45Post = 2,   // RKF45 after the control step: store on accept, restore on reject
};

// One update of the time-local truncation matrices; device pointers.
struct TlLaunch {
  HeomConsts c;
  int op = kTlAdvance;
  int stage = 0;
  double h = 0.0;
  Rkf45Ctl *ctl = nullptr;
  double2 *qk = nullptr;     // nb*K1*N*N  Q_{m,k}
  double2 *qk_st = nullptr;  // stored copy
  double2 *q = nullptr;      // nb*N*N     Q_m = sum_k Q_{m,k} (what HeomConsts::tl_q points at)
  double2 *q_st = nullptr;   // stored copy
};

size_t tl_smem_bytes(int N);
cudaError_t launch_tl(const TlLaunch &p, cudaStream_t stream);

}  // namespace phi
