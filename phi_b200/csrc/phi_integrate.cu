// phi_integrate.cu -- RK4 and RKF45 drivers: fused stage kernels replayed
// from captured CUDA graphs.
//
// RK4 (Rk4Integrate, hierarchy_integrator.cc:2578-2939) keeps four state-size
// buffers: y, acc, and the stage inputs X_a / X_b.  Stage s computes
// k_s = L(X_s) and in the same kernel writes X_{s+1} = y + a_s k_s and the
// accumulator acc (= y + dt/6 k0 + dt/3 k1 + dt/3 k2, then y = acc + dt/6 k3).
//
// RKF45 (Rkf45Integrate, :1797-2573) keeps y, the candidate y5, k0..k4 and the
// stage inputs.  The accept/reject decision and the step-size update run on
// the device (rkf45_control_kernel) so a captured graph of many steps needs
// no host round trip; the host polls a done flag between graph launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_kernels.h"
#include "heom_tile.h"
#include "heom_timelocal.h"
#include "heom_anneal.h"
#include "phi_context.h"

namespace {

int cuda_err(phi_ctx *ctx, cudaError_t e, const char *where) {
  ctx->error = std::string(where) + ": " + cudaGetErrorString(e);
  return PHI_E_CUDA;
}

#define PHI_CK(call)                                              \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return cuda_err(ctx, e_, #call);       \
  } while (0)

constexpr int kGraphSteps = 16;
// Steps per launch of the one-CTA small-hierarchy RK4 kernel (bounds the
// duration of one launch).
constexpr long long kSmallChunk = 4096;

}  // namespace

int phi_ctx::work_stride() const {
  const int N = desc.num_states;
  return mixed() ? phi::mixed_node_stride(N) : N * N;
}

size_t phi_ctx::work_bytes() const {
  return (size_t)hier.M * work_stride() * (mixed() ? sizeof(float2) : sizeof(double2));
}

int phi_ctx::ensure_work(int level) {
  const size_t b = state_bytes(), wb = work_bytes();
  auto alloc = [&](phi::DeviceBuffer &buf, size_t bytes) -> bool {
    if (buf.ptr) return true;
    return buf.alloc(bytes) == cudaSuccess;
  };
  bool ok = true;
  if (level >= 1) ok = ok && alloc(xa, wb) && alloc(xb, wb);
  if (level >= 2) ok = ok && alloc(acc, b);
  if (level >= 2 && mixed()) ok = ok && alloc(y32, wb);
  if (level >= 3) {
    ok = ok && alloc(y_alt, b);
    if (mixed()) ok = ok && alloc(y32_alt, wb);
    for (auto &k : kbuf) ok = ok && alloc(k, wb);
  }
  if (ok && !ctl.ptr) ok = ctl.alloc(std::max(sizeof(phi::Rkf45Ctl), sizeof(phi::Rk4Ctl))) == cudaSuccess;
  if (!ok) {
    error = "work-space allocation failed (" + std::to_string(b) + " bytes per buffer)";
    return PHI_E_OOM;
  }
  work_level = std::max(work_level, level);
  return PHI_OK;
}

void phi_ctx::release_graphs() {
  if (rk4_graph) cudaGraphExecDestroy(rk4_graph);
  if (rkf45_graph) cudaGraphExecDestroy(rkf45_graph);
  if (rkf45_graph1) cudaGraphExecDestroy(rkf45_graph1);
  rkf45_graph1 = nullptr;
  if (bicg_graph) cudaGraphExecDestroy(bicg_graph);
  rk4_graph = nullptr;
  rkf45_graph = nullptr;
  bicg_graph = nullptr;
}

namespace {

// Enqueues one RK4 step (four fused stage kernels).  With filtering the step
// reads the flags in active[par] and its last stage writes active[par ^ 1].
cudaError_t enqueue_rk4_step(phi_ctx *ctx, double dt, double2 *traj, int par, cudaStream_t s) {
  phi::StageLaunch L;
  L.c = ctx->c;
  ctx->bind_filter(L, par);
  L.mode = phi::kModeRk4;
  L.grid = ctx->grid;
  L.y = ctx->y.as<double2>();
  L.acc = ctx->acc.as<double2>();
  L.rk4 = ctx->ctl.as<phi::Rk4Ctl>();
  L.traj = traj;
  L.mixed = ctx->mixed();
  L.y32 = ctx->y32.ptr;
  double2 *xa = ctx->xa.as<double2>(), *xb = ctx->xb.as<double2>();
  const double a[4] = {dt / 2, dt / 2, dt, 0.0};
  const double w[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
  const double2 *in[4] = {L.y, xa, xb, xa};
  double2 *outb[4] = {xa, xb, xa, nullptr};
  const void *inv[4] = {L.mixed ? ctx->y32.ptr : (const void *)L.y, ctx->xa.ptr, ctx->xb.ptr, ctx->xa.ptr};
  void *outv[4] = {ctx->xa.ptr, ctx->xb.ptr, ctx->xa.ptr, nullptr};
  for (int st = 0; st < 4; ++st) {
    // Time-local matrices to t + dt/2 before stage 1 and to t + dt before
    // stage 3 (hierarchy_integrator.cc:2721, :2784).
    if (st == 1 || st == 3) {
      cudaError_t e = ctx->enqueue_time_local(phi::kTlAdvance, 0, dt / 2, s);
      if (e != cudaSuccess) return e;
    }
    // Annealing Hamiltonian at t, t + dt/2 and t + dt (:2688, :2728, :2792);
    // under Hilbert-space truncation the live ADOs follow the basis (y at t;
    // then y, the accumulator holding y and the k_s so far, and the stage
    // input: :2693, :2733-2735, :2797-2801).
    if (st != 2) {
      cudaError_t e = ctx->enqueue_anneal(phi::kAnnealRk4, st == 0 ? 0 : (st == 1 ? 1 : 2), dt, s);
      if (e == cudaSuccess) {
        if (st == 0)
          e = ctx->enqueue_anneal_rotate({ctx->y.ptr}, false, s);
        else
          e = ctx->enqueue_anneal_rotate({ctx->y.ptr, ctx->acc.ptr, ctx->xa.ptr}, false, s);
      }
      if (e != cudaSuccess) return e;
    }
    L.stage = st;
    L.x = in[st];
    L.out = outb[st];
    L.xv = inv[st];
    L.outv = outv[st];
    L.a_next = a[st];
    L.w_acc = w[st];
    cudaError_t e = phi::launch_stage(L, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t enqueue_rkf45_step(phi_ctx *ctx, cudaStream_t s) {
  phi::StageLaunch L;
  L.c = ctx->c;
  L.mode = phi::kModeRkf45;
  L.grid = ctx->grid;
  L.ctl = ctx->ctl.as<phi::Rkf45Ctl>();
  ctx->bind_filter(L, 0);  // the kernels index the flags by ycur
  L.ybuf[0] = ctx->y.as<double2>();
  L.ybuf[1] = ctx->y_alt.as<double2>();
  L.mixed = ctx->mixed();
  L.y32buf[0] = ctx->y32.ptr;
  L.y32buf[1] = ctx->y32_alt.ptr;
  for (int i = 0; i < 5; ++i) {
    L.k[i] = ctx->kbuf[i].as<double2>();
    L.kv[i] = ctx->kbuf[i].ptr;
  }
  double2 *xa = ctx->xa.as<double2>(), *xb = ctx->xb.as<double2>();
  const double2 *in[6] = {nullptr, xa, xb, xa, xb, xa};
  double2 *outb[6] = {xa, xb, xa, xb, xa, nullptr};
  for (int st = 0; st < 6; ++st) {
    // Time-local matrices along the stage times (hierarchy_integrator.cc
    // :2028, :2079, :2132, :2188, :2246-2247), steps read on the device.
    if (st > 0) {
      cudaError_t e = ctx->enqueue_time_local(phi::kTlRkf45Stage, st, 0.0, s);
      if (e != cudaSuccess) return e;
    }
    // Annealing Hamiltonian at t + a_s (:1988, :2033, :2084, :2138, :2194, :2252);
    // under Hilbert-space truncation the live ADOs follow the basis: y, the
    // stage input and k_0..k_{s-1} (k_1 is not read after stage 4, :2259-2263).
    {
      cudaError_t e = ctx->enqueue_anneal(phi::kAnnealRkf45, st, 0.0, s);
      if (e == cudaSuccess && ctx->ta_F > 0) {
        void *x = const_cast<double2 *>(in[st]);
        void *k0 = ctx->kbuf[0].ptr, *k1 = ctx->kbuf[1].ptr, *k2 = ctx->kbuf[2].ptr, *k3 = ctx->kbuf[3].ptr,
             *k4 = ctx->kbuf[4].ptr;
        switch (st) {
          case 0: e = ctx->enqueue_anneal_rotate({}, true, s); break;
          case 1: e = ctx->enqueue_anneal_rotate({x, k0}, true, s); break;
          case 2: e = ctx->enqueue_anneal_rotate({x, k0, k1}, true, s); break;
          case 3: e = ctx->enqueue_anneal_rotate({x, k0, k1, k2}, true, s); break;
          case 4: e = ctx->enqueue_anneal_rotate({x, k0, k1, k2, k3}, true, s); break;
          default: e = ctx->enqueue_anneal_rotate({x, k0, k2, k3, k4}, true, s); break;
        }
      }
      if (e != cudaSuccess) return e;
    }
    L.stage = st;
    L.x = in[st];
    L.out = outb[st];
    L.xv = in[st];
    L.outv = outb[st];
    cudaError_t e = phi::launch_stage(L, s);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = phi::launch_rkf45_control(L.ctl, s);
  if (e != cudaSuccess) return e;
  // Accepted: advance to t + dt and store (:2388-2389); rejected: restore (:2479).
  return ctx->enqueue_time_local(phi::kTlRkf45Post, 0, 0.0, s);
}

template <class F>
cudaError_t capture(cudaStream_t s, F &&body, cudaGraphExec_t *exec) {
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t eb = body();
  e = cudaStreamEndCapture(s, &graph);
  if (eb != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return eb;
  }
  if (e != cudaSuccess) return e;
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  // Upload now, on the capturing stream, so the first launch does not pay it.
  if (e == cudaSuccess) e = cudaGraphUpload(*exec, s);
  return e;
}

}  // namespace

extern "C" int phi_gpu_rk4(phi_ctx *ctx, double dt, double t_end, double output_min_step,
                           double *traj, double *times, int64_t capacity, int64_t *num_steps,
                           int64_t *num_out) {
  if (!ctx) return PHI_E_INVALID;
  if (!(dt > 0) || !std::isfinite(t_end)) {
    ctx->error = "rk4: dt must be positive and t_end finite";
    return PHI_E_INVALID;
  }
  int rc = ctx->ensure_work(2);
  if (rc != PHI_OK) return rc;
  // Step count and output times: the reference's loop
  // `while (time_now < end_time) { ...; time_now += dt_f_; }` (:2682, :2856).
  const long long out_factor = (long long)std::ceil(output_min_step / dt);
  std::vector<double> out_times;
  long long steps = 0;
  double t = ctx->time;
  while (t < t_end) {
    t += dt;
    if (out_factor > 0 && steps % out_factor == 0) out_times.push_back(t);
    ++steps;
    if (steps > (1ll << 40)) {
      ctx->error = "rk4: step count overflow";
      return PHI_E_INVALID;
    }
  }
  const long long rows = std::min<long long>((long long)out_times.size(), traj ? capacity : 0);
  double2 *dtraj = nullptr;
  if (rows > 0) {
    const size_t need = (size_t)rows * ctx->desc.num_states * ctx->desc.num_states * sizeof(double2);
    if (ctx->traj.bytes < need && ctx->traj.alloc(need) != cudaSuccess) {
      ctx->error = "rk4: trajectory allocation failed";
      return PHI_E_OOM;
    }
    dtraj = ctx->traj.as<double2>();
  }
  if (ctx->mixed())
    PHI_CK(phi::launch_to_c64(ctx->y.as<double2>(), ctx->y32.as<float2>(), ctx->hier.M,
                              ctx->desc.num_states * ctx->desc.num_states, ctx->work_stride(), ctx->stream));
  phi::Rk4Ctl hc{};
  hc.time = ctx->time;
  hc.step = 0;
  hc.out_factor = out_factor;
  hc.capacity = rows;
  hc.nout = 0;
  PHI_CK(cudaMemcpyAsync(ctx->ctl.ptr, &hc, sizeof(hc), cudaMemcpyHostToDevice, ctx->stream));

  // A small hierarchy runs whole in one CTA (launches of at most
  // kSmallChunk steps each).
  if (!ctx->annealing && !ctx->mixed() && phi::small_rk4_eligible(ctx->c)) {
    for (long long done = 0; done < steps; done += kSmallChunk)
      PHI_CK(phi::launch_small_rk4(ctx->c, ctx->y.as<double2>(), dt, std::min<long long>(kSmallChunk, steps - done),
                                   ctx->ctl.as<phi::Rk4Ctl>(), dtraj, ctx->stream));
    if (rows > 0)
      PHI_CK(cudaMemcpyAsync(traj, dtraj, (size_t)rows * ctx->desc.num_states * ctx->desc.num_states * sizeof(double2),
                             cudaMemcpyDeviceToHost, ctx->stream));
    PHI_CK(cudaStreamSynchronize(ctx->stream));
    if (times)
      for (long long r = 0; r < std::min<long long>((long long)out_times.size(), capacity); ++r) times[r] = out_times[r];
    ctx->time = t;
    if (num_steps) *num_steps = steps;
    if (num_out) *num_out = (int64_t)out_times.size();
    return ctx->check_device_flag();
  }
  // Replay a graph of kGraphSteps steps; the tail runs as direct launches.
  if (steps >= kGraphSteps &&
      (!ctx->rk4_graph || ctx->rk4_graph_dt != dt || ctx->rk4_graph_traj != (void *)dtraj)) {
    if (ctx->rk4_graph) cudaGraphExecDestroy(ctx->rk4_graph);
    ctx->rk4_graph = nullptr;
    PHI_CK(capture(ctx->stream, [&]() {
      for (int i = 0; i < kGraphSteps; ++i) {  // kGraphSteps is even: flag parity i & 1
        cudaError_t e = enqueue_rk4_step(ctx, dt, dtraj, i & 1, ctx->stream);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    }, &ctx->rk4_graph));
    ctx->rk4_graph_dt = dt;
    ctx->rk4_graph_traj = dtraj;
  }
  long long done = 0;
  while (steps - done >= kGraphSteps) {
    PHI_CK(cudaGraphLaunch(ctx->rk4_graph, ctx->stream));
    done += kGraphSteps;
  }
  for (; done < steps; ++done) PHI_CK(enqueue_rk4_step(ctx, dt, dtraj, (int)(done & 1), ctx->stream));
  if (ctx->c.filtered && (steps & 1))  // the current flags back in active[0]
    PHI_CK(cudaMemcpyAsync(ctx->active[0].ptr, ctx->active[1].ptr, (size_t)ctx->hier.M,
                           cudaMemcpyDeviceToDevice, ctx->stream));
  if (rows > 0) {
    PHI_CK(cudaMemcpyAsync(traj, dtraj, (size_t)rows * ctx->desc.num_states * ctx->desc.num_states * sizeof(double2),
                           cudaMemcpyDeviceToHost, ctx->stream));
  }
  PHI_CK(cudaStreamSynchronize(ctx->stream));
  if (times)
    for (long long r = 0; r < std::min<long long>((long long)out_times.size(), capacity); ++r) times[r] = out_times[r];
  ctx->time = t;
  if (num_steps) *num_steps = steps;
  if (num_out) *num_out = (int64_t)out_times.size();
  return ctx->check_device_flag();
}

namespace {

// Shared driver of phi_gpu_rkf45 / phi_gpu_rkf45_advance.
int run_rkf45(phi_ctx *ctx, double dt0, double t_end, double tol, double min_dt,
              int64_t max_steps, bool limit_is_error, phi_rkf45_stats *stats) {
  if (!(tol > 0) || !(min_dt > 0) || !std::isfinite(t_end) || (limit_is_error && !(dt0 > 0))) {
    ctx->error = "rkf45: dt0, tol and min_dt must be positive and t_end finite";
    return PHI_E_INVALID;
  }
  const bool resume = !(dt0 > 0);
  if (resume && !ctx->rkf45_started) {
    ctx->error = "rkf45: dt0 <= 0 continues a previous run, but there is none";
    return PHI_E_STATE;
  }
  int rc = ctx->ensure_work(3);
  if (rc != PHI_OK) return rc;
  phi::Rkf45Ctl hc{};
  if (resume) {
    hc = ctx->rkf45_last;
  } else {
    hc.dt = dt0;
    hc.dtup = 1.1;
    hc.dtdn = 0.5;
    // Butcher tableau of Rkf45Integrate (:1937-1975), each entry scaled by dt0.
    const double tab[24] = {2. / 9.,   1. / 12.,  1. / 4.,   69. / 128., -243. / 128., 135. / 64.,
                            -17. / 12., 27. / 4.,  -27. / 5,  16. / 15,   65. / 432.,   -5. / 16,
                            13. / 16.,  4. / 27.,  5. / 144., 1. / 9,     9. / 20,      16. / 45,
                            1. / 12,    47. / 450, 12. / 25,  32. / 225,  1. / 30,      6. / 25};
    for (int q = 0; q < 24; ++q) hc.coef[q] = tab[q] * dt0;
    // Stage offsets a1..a5 (:1937, :1947-1951).
    const double offs[5] = {2. / 9, 1. / 3, 3. / 4, 1.0, 5. / 6};
    for (int s = 0; s < 5; ++s) hc.a[s] = offs[s] * dt0;
  }
  hc.tl_pending = 0;
  hc.time = ctx->time;
  hc.end_time = t_end;
  hc.tol = tol;
  hc.min_dt = min_dt;
  hc.max_error = 0.0;
  hc.err_bits = 0ull;
  hc.steps = 0;
  hc.accepted = 0;
  hc.max_steps = max_steps > 0 ? max_steps : 10000000ll;
  hc.ycur = 0;
  hc.done = ctx->time < t_end ? 0 : 1;
  hc.status = 0;
  hc.nonfinite = 0;
  hc.forced = ctx->rkf45_forced_len ? ctx->rkf45_forced.as<signed char>() : nullptr;
  hc.forced_len = ctx->rkf45_forced_len;
  hc.err_trace = ctx->rkf45_trace_cap ? ctx->rkf45_trace.as<double>() : nullptr;
  hc.trace_cap = ctx->rkf45_trace_cap;
  PHI_CK(cudaMemcpyAsync(ctx->ctl.ptr, &hc, sizeof(hc), cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->mixed())  // stage-0 input of the first step: complex64 copy of y (ycur = 0)
    PHI_CK(phi::launch_to_c64(ctx->y.as<double2>(), ctx->y32.as<float2>(), ctx->hier.M,
                              ctx->desc.num_states * ctx->desc.num_states, ctx->work_stride(), ctx->stream));
  if (!ctx->rkf45_graph) {
    PHI_CK(capture(ctx->stream, [&]() {
      for (int i = 0; i < kGraphSteps; ++i) {
        cudaError_t e = enqueue_rkf45_step(ctx, ctx->stream);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    }, &ctx->rkf45_graph));
    // One step, for the remainder of a call (fewer launch calls and
    // inter-kernel gaps than seven direct launches).
    PHI_CK(capture(ctx->stream, [&]() { return enqueue_rkf45_step(ctx, ctx->stream); }, &ctx->rkf45_graph1));
  }
  if (!ctx->host_ctl) PHI_CK(phi::cached_host_alloc(&ctx->host_ctl, sizeof(phi::Rkf45Ctl)));
  phi::Rkf45Ctl *hpin = static_cast<phi::Rkf45Ctl *>(ctx->host_ctl);
  int result = PHI_OK;
  // Exactly max_steps attempted steps are enqueued: whole graphs of
  // kGraphSteps, then the remainder as direct launches.  Two chunks are in
  // flight: the done flag after chunk j is read while chunk j+1 runs; steps
  // after completion are no-ops on the device.
  long long launched = 0, graphs = 0;
  auto enqueue_chunk = [&]() -> cudaError_t {
    const long long left = hc.max_steps - launched;
    if (left >= kGraphSteps) {
      launched += kGraphSteps;
      ++graphs;
      return cudaGraphLaunch(ctx->rkf45_graph, ctx->stream);
    }
    for (; launched < hc.max_steps; ++launched) {
      cudaError_t e = cudaGraphLaunch(ctx->rkf45_graph1, ctx->stream);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  PHI_CK(enqueue_chunk());
  for (;;) {
    cudaError_t e = cudaSuccess;
    if (launched < hc.max_steps) e = enqueue_chunk();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hpin, ctx->ctl.ptr, sizeof(phi::Rkf45Ctl), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      result = cuda_err(ctx, e, "rkf45 graph");
      break;
    }
    if (hpin->done) break;
    if (launched >= hc.max_steps) {  // every step ran and the device did not stop
      ctx->error = "rkf45: the device control block did not finish after max_steps steps";
      result = PHI_E_CUDA;
      break;
    }
  }
  ctx->graph_launches += graphs;
  if (result == PHI_OK) {
    hc = *hpin;
    if (hc.ycur == 1) {
      // The current state is in the alternate buffers: copy it back on the
      // device rather than swap the buffers, so the captured step graphs
      // (which bake in both pointers) stay valid for the next call.
      cudaError_t e = cudaMemcpyAsync(ctx->y.ptr, ctx->y_alt.ptr, ctx->state_bytes(), cudaMemcpyDeviceToDevice,
                                      ctx->stream);
      // (y32 is rebuilt from y at the start of every call.)
      if (e == cudaSuccess && ctx->c.filtered)
        e = cudaMemcpyAsync(ctx->active[0].ptr, ctx->active[1].ptr, (size_t)ctx->hier.M, cudaMemcpyDeviceToDevice,
                            ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) {
        result = cuda_err(ctx, e, "rkf45 state copy");
      }
      hc.ycur = 0;
    }
    ctx->time = hc.time;
    ctx->rkf45_last = hc;
    ctx->rkf45_started = true;
    if (stats) {
      stats->steps = hc.steps;
      stats->accepted = hc.accepted;
      stats->final_time = hc.time;
      stats->final_dt = hc.dt;
      stats->max_error = hc.max_error;
    }
    if (hc.status == 1 && limit_is_error) {
      ctx->error = "rkf45: step limit reached before t_end";
      result = PHI_E_STEP_COLLAPSE;
    } else if (hc.status == 2) {
      ctx->error = "rkf45: non-finite error estimate";
      result = PHI_E_NUMERIC;
    }
  }
  if (result == PHI_OK) result = ctx->check_device_flag();
  return result;
}

}  // namespace

extern "C" int phi_gpu_rkf45(phi_ctx *ctx, double dt0, double t_end, double tol, double min_dt,
                             int64_t max_steps, phi_rkf45_stats *stats) {
  if (!ctx) return PHI_E_INVALID;
  return run_rkf45(ctx, dt0, t_end, tol, min_dt, max_steps, true, stats);
}

extern "C" int phi_gpu_rkf45_advance(phi_ctx *ctx, double dt0, double t_end, double tol,
                                     double min_dt, int64_t steps, phi_rkf45_stats *stats) {
  if (!ctx) return PHI_E_INVALID;
  if (steps <= 0) {
    ctx->error = "rkf45_advance: steps must be positive";
    return PHI_E_INVALID;
  }
  return run_rkf45(ctx, dt0, t_end, tol, min_dt, steps, false, stats);
}

extern "C" int phi_gpu_debug_set_rkf45_replay(phi_ctx *ctx, const int8_t *decisions, int64_t count,
                                              int64_t trace_capacity) {
  if (!ctx || count < 0 || trace_capacity < 0 || (count > 0 && !decisions)) return PHI_E_INVALID;
  for (int64_t i = 0; i < count; ++i)
    if (decisions[i] < 0 || decisions[i] > 2) {
      ctx->error = "rkf45 replay: decisions are 0 (reject), 1 (accept) or 2 (accept and grow)";
      return PHI_E_INVALID;
    }
  ctx->rkf45_forced_len = 0;
  ctx->rkf45_trace_cap = 0;
  if (count > 0) {
    if (ctx->rkf45_forced.bytes < (size_t)count) {
      ctx->rkf45_forced.reset();
      PHI_CK(ctx->rkf45_forced.alloc((size_t)count));
    }
    PHI_CK(cudaMemcpy(ctx->rkf45_forced.ptr, decisions, (size_t)count, cudaMemcpyHostToDevice));
  }
  if (trace_capacity > 0 && ctx->rkf45_trace.bytes < (size_t)trace_capacity * sizeof(double)) {
    ctx->rkf45_trace.reset();
    PHI_CK(ctx->rkf45_trace.alloc((size_t)trace_capacity * sizeof(double)));
  }
  ctx->rkf45_forced_len = count;
  ctx->rkf45_trace_cap = trace_capacity;
  return PHI_OK;
}

extern "C" int phi_gpu_debug_get_rkf45_errors(phi_ctx *ctx, double *out, int64_t capacity, int64_t *count) {
  if (!ctx || !count || (capacity > 0 && !out)) return PHI_E_INVALID;
  const long long n = std::min<long long>(ctx->rkf45_last.steps, ctx->rkf45_trace_cap);
  *count = n;
  const long long m = std::min<long long>(n, capacity);
  if (m > 0) PHI_CK(cudaMemcpy(out, ctx->rkf45_trace.ptr, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost));
  return PHI_OK;
}

extern "C" int phi_gpu_stream(const phi_ctx *ctx, void **stream) {
  if (!ctx || !stream) return PHI_E_INVALID;
  *stream = (void *)ctx->stream;
  return PHI_OK;
}
