// phi_noalloc.cu -- an RK4 step that allocates no memory.
//
// Some callers cannot call cudaMalloc at the point where they step the
// hierarchy: code running under CUDA stream capture (an allocation would end
// or invalidate the capture), hosts that route every device byte through their
// own allocator or memory pool (a stray cudaMalloc fragments it or fails
// against its reservation), and loops with a hard latency budget (cudaMalloc
// can synchronise the device).  phi_gpu_rk4_step_noalloc serves them: the
// caller passes the input and output state buffers, and the two stage-input
// buffers the RK4 step needs live in a file-scope __device__ array that is
// part of the loaded library.
//
// Limits and sharing rules:
//  * the array holds two stage buffers of kNoAllocMaxStateBytes (8 MiB) each,
//    so the whole-hierarchy state (M * N * N * 16 bytes) must fit in 8 MiB;
//    every GPU that loads the library keeps these 16 MiB until the process
//    exits;
//  * all calls share the array: two calls whose kernels overlap on the GPU
//    (different streams, or different contexts on one device) race on it;
//  * every stage buffer is fully written before it is read within a step, so
//    nothing needs clearing between calls;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is kept for the life of the
//    library: after cudaDeviceReset on that device, reload the library;
//  * the step reads and advances the context's own step-dependent state as
//    one phi_gpu_rk4 step would: time-local truncation matrices (two half
//    steps of dt/2) and filter flags (the new flags become the current ones).
//    The context's time and its own state buffer do not change.  So d_out is
//    one step after d_in only when d_in continues the trajectory those
//    matrices and flags belong to (phi_gpu_set_state resets both);
//  * the call does not synchronise, so a bounded device wait that gave up
//    inside it is reported by the next call that checks the context's device
//    flag (phi_gpu_check_device_flag, or any synchronising entry point).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/phi_b200.h"
#include "heom_kernels.h"
#include "heom_timelocal.h"
#include "phi_context.h"

namespace {

constexpr size_t kNoAllocMaxStateBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

// Two RK4 stage-input buffers (X_a, X_b), back to back.
__device__ __align__(256) unsigned char g_rk4_stage_scratch[2 * kNoAllocMaxStateBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_rk4_stage_scratch on `device` (looked up once per
// device, with that device current).  In host code the symbol itself is only
// a host-side stand-in and must never be passed to a kernel.
cudaError_t scratch_address(int device, void **out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_rk4_stage_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" int phi_gpu_rk4_step_noalloc(phi_ctx *ctx, const void *d_in, void *d_out, double dt,
                                        void *stream) {
  if (!ctx) return PHI_E_INVALID;
  if (!d_in || !d_out || d_in == d_out || !(dt > 0)) {
    ctx->error = "rk4_step_noalloc: needs distinct non-NULL input and output buffers and dt > 0";
    return PHI_E_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15u) {
    ctx->error = "rk4_step_noalloc: device buffers must be 16-byte aligned";
    return PHI_E_INVALID;
  }
  if (ctx->mixed()) {
    ctx->error = "rk4_step_noalloc: complex128 (PHI_PREC_FP64) contexts only";
    return PHI_E_INVALID;
  }
  if (ctx->annealing) {
    ctx->error = "rk4_step_noalloc: an annealing Hamiltonian follows the step time kept by phi_gpu_rk4";
    return PHI_E_INVALID;
  }
  const size_t bytes = ctx->state_bytes();
  if (bytes > kNoAllocMaxStateBytes) {
    ctx->error = "rk4_step_noalloc: hierarchy state of " + std::to_string(bytes) +
                 " bytes exceeds the " + std::to_string(kNoAllocMaxStateBytes) +
                 "-byte limit of the built-in scratch; use phi_gpu_rk4";
    return PHI_E_INVALID;
  }
  int prev_device = -1;
  cudaError_t e = cudaGetDevice(&prev_device);
  const int device = ctx->desc.device;
  const bool restore = e == cudaSuccess && prev_device != device;
  if (restore) e = cudaSetDevice(device);
  void *scratch = nullptr;
  if (e == cudaSuccess) e = scratch_address(device, &scratch);
  if (e == cudaSuccess) {
    double2 *xa = static_cast<double2 *>(scratch);
    double2 *xb = reinterpret_cast<double2 *>(static_cast<unsigned char *>(scratch) +
                                              kNoAllocMaxStateBytes);
    const double2 *y = static_cast<const double2 *>(d_in);
    double2 *out = static_cast<double2 *>(d_out);
    // Same four fused stage kernels as phi_gpu_rk4; the caller's output buffer
    // doubles as the RK4 accumulator and receives the new state at stage 3.
    phi::StageLaunch L;
    L.c = ctx->c;
    L.mode = phi::kModeRk4;
    L.grid = ctx->grid;
    ctx->bind_filter(L, 0);
    const double a[4] = {dt / 2, dt / 2, dt, 0.0};
    const double w[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
    const double2 *in[4] = {y, xa, xb, xa};
    double2 *nxt[4] = {xa, xb, xa, nullptr};
    for (int st = 0; st < 4 && e == cudaSuccess; ++st) {
      // Time-local matrices to t + dt/2 and t + dt (no allocation: the
      // context's own buffers).
      if (st == 1 || st == 3) {
        e = ctx->enqueue_time_local(phi::kTlAdvance, 0, dt / 2, static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) break;
      }
      L.stage = st;
      L.x = in[st];
      L.out = nxt[st];
      L.y = st < 3 ? const_cast<double2 *>(y) : out;
      L.acc = out;
      L.a_next = a[st];
      L.w_acc = w[st];
      e = phi::launch_stage(L, static_cast<cudaStream_t>(stream));
    }
    // Filtering: the step wrote the new flags to active[1]; the current ones
    // live in active[0] between calls (a device copy, no allocation).
    if (e == cudaSuccess && ctx->c.filtered)
      e = cudaMemcpyAsync(ctx->active[0].ptr, ctx->active[1].ptr, (size_t)ctx->hier.M,
                          cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream));
  }
  if (restore) cudaSetDevice(prev_device);
  if (e != cudaSuccess) {
    ctx->error = std::string("rk4_step_noalloc: ") + cudaGetErrorString(e);
    return PHI_E_CUDA;
  }
  return PHI_OK;
}
