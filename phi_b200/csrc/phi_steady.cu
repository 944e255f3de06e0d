// phi_steady.cu -- phi_gpu_steady_state: the BiCGSTAB(ell) driver (kernels in
// heom_bicgstab.cu).  The operator applies are the Liouvillian kernels of the
// propagation path, always in FP64.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_bicgstab.h"
#include "heom_tile.h"
#include "heom_kernels.h"
#include "phi_context.h"

namespace {

int steady_err(phi_ctx *ctx, cudaError_t e, const char *where) {
  ctx->error = std::string("steady_state: ") + where + ": " + cudaGetErrorString(e);
  return PHI_E_CUDA;
}

#define PHI_SK(call)                                          \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return steady_err(ctx, e_, #call); \
  } while (0)

// out = L(in) over every node in FP64 (element (0,0) of node 0 is handled by
// the BiCGSTAB kernels).
cudaError_t apply_fp64(phi_ctx *ctx, const double2 *in, double2 *out, cudaStream_t s,
                       const double2 *dot_w = nullptr, double *dot_part = nullptr) {
  phi::StageLaunch L;
  L.dot_w = dot_w;
  L.dot_part = dot_part;
  L.c = ctx->c;
  L.mode = phi::kModeApply;
  L.grid = ctx->grid;
  L.x = in;
  L.out = out;
  L.xv = in;
  L.outv = out;
  L.mixed = false;
  ctx->bind_filter(L, 0);  // all active unless a filtered integration ran before
  return phi::launch_stage(L, s);
}

// One outer iteration: ell BiCG steps (two applies each), then the
// minimal-residual step and the stopping test.
cudaError_t outer_iteration(phi_ctx *ctx, const phi::BicgVectors &V, long long n, phi::BicgScalars *sc, int ell,
                            int grid, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  // With the tiled kernel the applies that produce u_{j+1} and r_{j+1} also
  // zero their element (0,0) of node 0 and sum <rhat, .> per tile, so gamma
  // and the next rho need only a one-block finish instead of a pass over
  // two state-size vectors each.
  const bool fused = ctx->bicg_parts.ptr != nullptr;
  double *pu = fused ? ctx->bicg_parts.as<double>() : nullptr;
  double *pr = fused ? pu + ctx->bicg_tiles : nullptr;
  for (int j = 0; j < ell && e == cudaSuccess; ++j) {
    if (j > 0) e = fused ? phi::bicg_launch_dot_finish(pr, ctx->bicg_tiles, sc, 0, s)
                         : phi::bicg_launch_rho(V, n, sc, j, grid, s);
    if (e == cudaSuccess) e = phi::bicg_launch_u_update(V, n, sc, j, grid, s);
    if (e == cudaSuccess) e = apply_fp64(ctx, V.u[j], V.u[j + 1], s, fused ? V.rhat : nullptr, pu);
    if (e == cudaSuccess)
      e = fused ? phi::bicg_launch_dot_finish(pu, ctx->bicg_tiles, sc, 1, s)
                : phi::bicg_launch_gamma(V, n, sc, j, grid, s);
    if (e == cudaSuccess) e = phi::bicg_launch_r_update(V, n, sc, j, grid, s);
    const bool rho_next = fused && j + 1 < ell;  // the last r_{j+1} goes to the Gram step instead
    if (e == cudaSuccess) e = apply_fp64(ctx, V.r[j], V.r[j + 1], s, rho_next ? V.rhat : nullptr, pr);
  }
  if (e == cudaSuccess) e = phi::bicg_launch_gram(V, n, sc, ell, grid, s);
  if (e == cudaSuccess) e = phi::bicg_launch_mr_update(V, n, sc, ell, grid, s);
  return e;
}

// Owns the timing events of one solve.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

const char *breakdown_text(int code) {
  switch (code) {
    case phi::kBicgRhoZero: return "BiCGSTAB breakdown: <rhat, r> = 0";
    case phi::kBicgGammaZero: return "BiCGSTAB breakdown: <rhat, A u> = 0";
    case phi::kBicgGramSingular: return "BiCGSTAB breakdown: singular minimal-residual system";
    case phi::kBicgNonFinite: return "BiCGSTAB breakdown: non-finite residual";
    default: return "BiCGSTAB breakdown";
  }
}

// guess: NULL (rho_0 = I/N), a whole hierarchy (guess_rho0 false) or rho_0
// only (guess_rho0 true; other nodes zero).
int steady_impl(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode, int32_t max_steps, const double *guess,
                bool guess_rho0, phi_solve_stats *stats) {
  if (!ctx) return PHI_E_INVALID;
  if (ctx->annealing) {
    ctx->error = "steady_state: an annealing Hamiltonian has no steady state (it changes with time)";
    return PHI_E_INVALID;
  }
  if (ctx->c.time_local) {
    // FixIncompatibleCombinations turns time-local truncation off for the
    // BiCGSTAB methods (phi_parameters.cc:831-837).
    ctx->error = "steady_state: time-local truncation is a propagation feature (PHI turns it off for steady states)";
    return PHI_E_INVALID;
  }
  if (ell < 1 || ell > phi::kMaxEll) {
    ctx->error = "steady_state: ell must be in 1.." + std::to_string(phi::kMaxEll);
    return PHI_E_INVALID;
  }
  if (!(tol > 0) || tol_mode < PHI_TOL_RELATIVE || tol_mode > PHI_TOL_ABS_SQUARED) {
    ctx->error = "steady_state: tol must be positive and tol_mode one of PHI_TOL_*";
    return PHI_E_INVALID;
  }
  if (max_steps <= 0) max_steps = 9999;
  const int N = ctx->desc.num_states;
  const long long n = ctx->hier.M * (long long)N * N;
  const size_t bytes = (size_t)n * sizeof(double2);
  const int nvec = 3 + 2 * (ell + 1);
  if (ctx->bicg_vecs.bytes < bytes * nvec) {
    if (ctx->bicg_vecs.alloc(bytes * nvec) != cudaSuccess) {
      ctx->error = "steady_state: allocation of " + std::to_string(nvec) + " Krylov vectors (" +
                   std::to_string(bytes * nvec) + " bytes) failed";
      return PHI_E_OOM;
    }
  }
  if (phi::tile_kernel_available(ctx->c) && !ctx->bicg_parts.ptr) {
    ctx->bicg_tiles = phi::tile_count(ctx->c, false);
    if (ctx->bicg_tiles > 0 && ctx->bicg_parts.alloc((size_t)2 * ctx->bicg_tiles * sizeof(double)) != cudaSuccess) {
      ctx->error = "steady_state: allocation of the per-tile partial sums failed";
      return PHI_E_OOM;
    }
  }
  if (!ctx->bicg_sc.ptr && ctx->bicg_sc.alloc(sizeof(phi::BicgScalars)) != cudaSuccess) {
    ctx->error = "steady_state: allocation failed";
    return PHI_E_OOM;
  }
  double2 *base = ctx->bicg_vecs.as<double2>();
  phi::BicgVectors V{};
  V.x = base;
  V.rhat = base + n;
  V.b = base + 2 * n;
  for (int i = 0; i <= ell; ++i) {
    V.r[i] = base + (3 + i) * n;
    V.u[i] = base + (4 + ell + i) * n;
  }
  phi::BicgScalars *sc = ctx->bicg_sc.as<phi::BicgScalars>();
  cudaStream_t s = ctx->stream;
  const int grid = phi::bicg_grid(ctx->num_sms);

  EventPair evs;
  PHI_SK(cudaEventCreate(&evs.a));
  PHI_SK(cudaEventCreate(&evs.b));
  cudaEvent_t ev0 = evs.a, ev1 = evs.b;
  PHI_SK(cudaEventRecord(ev0, s));
  // b = -L(E00), element (0,0) of node 0 dropped.
  const double2 one = make_double2(1.0, 0.0);
  PHI_SK(cudaMemsetAsync(V.r[0], 0, bytes, s));
  PHI_SK(cudaMemcpyAsync(V.r[0], &one, sizeof(double2), cudaMemcpyHostToDevice, s));
  PHI_SK(apply_fp64(ctx, V.r[0], V.b, s));
  PHI_SK(phi::bicg_launch_rhs(V.b, n, grid, s));
  // x0: the caller's hierarchy, or rho_0 = I / N; scaled to x_0[0,0] = 1.
  std::vector<double2> rho;
  if (guess && !guess_rho0) {
    PHI_SK(cudaMemcpyAsync(V.x, guess, bytes, cudaMemcpyHostToDevice, s));
  } else if (guess) {
    PHI_SK(cudaMemsetAsync(V.x, 0, bytes, s));
    PHI_SK(cudaMemcpyAsync(V.x, guess, (size_t)N * N * sizeof(double2), cudaMemcpyHostToDevice, s));
  } else {
    rho.assign((size_t)N * N, make_double2(0.0, 0.0));
    for (int i = 0; i < N; ++i) rho[(size_t)i * (N + 1)] = make_double2(1.0 / N, 0.0);
    PHI_SK(cudaMemsetAsync(V.x, 0, bytes, s));
    PHI_SK(cudaMemcpyAsync(V.x, rho.data(), rho.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  }
  PHI_SK(phi::bicg_launch_guess(V.x, n, grid, s));
  PHI_SK(apply_fp64(ctx, V.x, V.r[1], s));
  phi::BicgScalars init{};
  init.tol = tol;
  init.tol_mode = tol_mode;
  init.max_steps = max_steps;
  init.ell = ell;
  PHI_SK(cudaMemcpyAsync(sc, &init, offsetof(phi::BicgScalars, partials), cudaMemcpyHostToDevice, s));
  PHI_SK(phi::bicg_launch_init(V, n, sc, grid, s));
  PHI_SK(cudaStreamSynchronize(s));  // the host staging above is stack memory

  // Replay graphs of several outer iterations until the device says done.
  const int outer_per_graph = ell >= 8 ? 1 : 8 / ell;
  if (ctx->bicg_graph && ctx->bicg_ell != ell) {
    cudaGraphExecDestroy(ctx->bicg_graph);
    ctx->bicg_graph = nullptr;
  }
  if (!ctx->bicg_graph) {
    cudaGraph_t graph = nullptr;
    PHI_SK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t eb = cudaSuccess;
    for (int it = 0; it < outer_per_graph && eb == cudaSuccess; ++it) eb = outer_iteration(ctx, V, n, sc, ell, grid, s);
    cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (eb != cudaSuccess || ee != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return steady_err(ctx, eb != cudaSuccess ? eb : ee, "capture");
    }
    cudaError_t ei = cudaGraphInstantiate(&ctx->bicg_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ei == cudaSuccess) ei = cudaGraphUpload(ctx->bicg_graph, s);  // not on the first launch
    if (ei != cudaSuccess) return steady_err(ctx, ei, "instantiate");
    ctx->bicg_ell = ell;
  }
  phi::BicgScalars *host = nullptr;
  PHI_SK(phi::cached_host_alloc(reinterpret_cast<void **>(&host), offsetof(phi::BicgScalars, partials)));
  const long long max_graphs = (long long)max_steps / ((long long)ell * outer_per_graph) + 2;
  int result = PHI_OK;
  for (long long g = 0;; ++g) {
    cudaError_t e = cudaMemcpyAsync(host, sc, offsetof(phi::BicgScalars, partials), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      result = steady_err(ctx, e, "poll");
      break;
    }
    if (host->done) break;
    if (g >= max_graphs) {  // the device stops at max_steps; this bounds the host loop as well
      ctx->error = "steady_state: solver did not stop";
      result = PHI_E_CUDA;
      break;
    }
    e = cudaGraphLaunch(ctx->bicg_graph, s);
    if (e != cudaSuccess) {
      result = steady_err(ctx, e, "graph launch");
      break;
    }
  }
  if (result == PHI_OK) {
    // The context state becomes the solution: x_0[0,0] = 1, divided by tr rho_0.
    cudaError_t e = phi::bicg_launch_finalize(V.x, ctx->y.as<double2>(), n, N, sc, grid, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, sc, offsetof(phi::BicgScalars, partials), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) result = steady_err(ctx, e, "finalize");
  }
  if (result == PHI_OK) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (stats) {
      stats->iterations = host->steps;
      stats->converged = host->converged;
      // ||r|| / ||b|| under PHI_TOL_RELATIVE, ||r|| under PHI_TOL_ABSOLUTE,
      // ||r||^2 under PHI_TOL_ABS_SQUARED: the quantity compared with tol.
      stats->residual = tol_mode == PHI_TOL_ABS_SQUARED ? host->rr
                        : tol_mode == PHI_TOL_ABSOLUTE  ? std::sqrt(host->rr)
                        : host->bb > 0                  ? std::sqrt(host->rr / host->bb)
                                                        : std::sqrt(host->rr);
      stats->seconds = ms / 1e3;
    }
    if (!host->converged) {
      ctx->error = host->breakdown ? std::string("steady_state: ") + breakdown_text(host->breakdown)
                                   : "steady_state: step limit reached";
      result = PHI_E_NO_CONVERGENCE;
    }
  }
  // On an error path a copy into `host` may still be queued: drain the
  // stream before the buffer goes back to the cache for another owner.
  if (result != PHI_OK) cudaStreamSynchronize(s);
  phi::cached_host_free(host, offsetof(phi::BicgScalars, partials));
  if (result == PHI_OK || result == PHI_E_NO_CONVERGENCE) {
    const int flag = ctx->check_device_flag();
    if (flag != PHI_OK) result = flag;
  }
  return result;
}

}  // namespace

extern "C" int phi_gpu_steady_state(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode, int32_t max_steps,
                                    const double *guess, phi_solve_stats *stats) {
  return steady_impl(ctx, ell, tol, tol_mode, max_steps, guess, false, stats);
}

extern "C" int phi_gpu_steady_state_rho0(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode,
                                         int32_t max_steps, const double *rho0_guess, phi_solve_stats *stats) {
  if (!rho0_guess) {
    if (ctx) ctx->error = "steady_state_rho0: rho0_guess is NULL";
    return PHI_E_INVALID;
  }
  return steady_impl(ctx, ell, tol, tol_mode, max_steps, rho0_guess, true, stats);
}
