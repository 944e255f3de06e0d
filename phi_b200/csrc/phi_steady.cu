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
#include "heom_deflate.h"
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

// v = P v after an operator apply (deflated solves): the coefficients, the
// change of <rhat, v> into the extra partial slot (part, or NULL), the update.
cudaError_t project(const phi::DeflView *D, double2 *v, double *part, cudaStream_t s) {
  cudaError_t e = phi::defl_launch_coeff(*D, v, nullptr, part, s);
  return e == cudaSuccess ? phi::defl_launch_update(*D, v, s) : e;
}

// One outer iteration: ell BiCG steps (two applies each), then the
// minimal-residual step and the stopping test.  D: the deflation space, or
// NULL; every operator product is then followed by the projection P.
cudaError_t outer_iteration(phi_ctx *ctx, const phi::BicgVectors &V, long long n, phi::BicgScalars *sc, int ell,
                            int grid, cudaStream_t s, const phi::DeflView *D) {
  cudaError_t e = cudaSuccess;
  // With the tiled kernel the applies that produce u_{j+1} and r_{j+1} also
  // zero their element (0,0) of node 0 and sum <rhat, .> per tile, so gamma
  // and the next rho need only a one-block finish instead of a pass over
  // two state-size vectors each.  Each of the two partial arrays has one
  // slot more than there are tiles: the projection's change of the sum.
  const bool fused = ctx->bicg_parts.ptr != nullptr;
  const long long tiles = ctx->bicg_tiles;
  const long long nparts = tiles + (D ? 1 : 0);
  double *pu = fused ? ctx->bicg_parts.as<double>() : nullptr;
  double *pr = fused ? pu + tiles + 1 : nullptr;
  // Deflated and fused, the projection's coefficient kernel also finishes
  // the inner product (rho or gamma) before its update kernel runs.
  const bool fold = fused && D;
  for (int j = 0; j < ell && e == cudaSuccess; ++j) {
    if (j > 0 && !fold)
      e = fused ? phi::bicg_launch_dot_finish(pr, nparts, sc, 0, s) : phi::bicg_launch_rho(V, n, sc, j, grid, s);
    if (e == cudaSuccess) e = phi::bicg_launch_u_update(V, n, sc, j, grid, s);
    if (e == cudaSuccess) e = apply_fp64(ctx, V.u[j], V.u[j + 1], s, fused ? V.rhat : nullptr, pu);
    if (e == cudaSuccess && fold) {
      e = phi::defl_launch_coeff_finish(*D, V.u[j + 1], pu + tiles, pu, nparts, sc, 1, s);
      if (e == cudaSuccess) e = phi::defl_launch_update(*D, V.u[j + 1], s);
    } else {
      if (e == cudaSuccess && D) e = project(D, V.u[j + 1], nullptr, s);
      if (e == cudaSuccess)
        e = fused ? phi::bicg_launch_dot_finish(pu, nparts, sc, 1, s) : phi::bicg_launch_gamma(V, n, sc, j, grid, s);
    }
    if (e == cudaSuccess) e = phi::bicg_launch_r_update(V, n, sc, j, grid, s);
    const bool rho_next = fused && j + 1 < ell;  // the last r_{j+1} goes to the Gram step instead
    if (e == cudaSuccess) e = apply_fp64(ctx, V.r[j], V.r[j + 1], s, rho_next ? V.rhat : nullptr, pr);
    if (e == cudaSuccess && fold && rho_next) {
      e = phi::defl_launch_coeff_finish(*D, V.r[j + 1], pr + tiles, pr, nparts, sc, 0, s);
      if (e == cudaSuccess) e = phi::defl_launch_update(*D, V.r[j + 1], s);
    } else if (e == cudaSuccess && D) {
      e = project(D, V.r[j + 1], nullptr, s);
    }
  }
  if (e == cudaSuccess) e = phi::bicg_launch_gram(V, n, sc, ell, grid, s);
  if (e == cudaSuccess) e = phi::bicg_launch_mr_update(V, n, sc, ell, grid, s);
  return e;
}

// Deflation space of a solve: the tiers of the hierarchy whose ADOs' real
// coordinates span Z (0: none), k = their count, rows_nodes = the nodes of
// tiers 0..tiers (where A Z lives).  Tier l holds C(T + l - 1, l) nodes
// (every multi-index of T terms with sum l), tier by tier in node order.
struct DeflPlan {
  int tiers = 0;
  int k = 0;
  long long rows_nodes = 0;  // nodes of tiers 0..tiers (the rows of A Z)
  long long unit_nodes = 0;  // nodes of tiers 0..tiers+1 (their neighbours)
};

bool defl_fits(const phi_ctx *ctx, int tiers, DeflPlan *out) {
  const long long T = ctx->c.T, N = ctx->desc.num_states, E = N * N;
  const int L = ctx->c.L;
  if (N < 2 || tiers < 1 || tiers - 1 > L) return false;
  long long size = 1, deflated = 0, rows = 0, units = 0;  // size: nodes of tier l
  for (int l = 0; l <= tiers + 1 && l <= L; ++l) {
    if (l > 0) size = size * (T + l - 1) / l;
    if (l < tiers) deflated += size;
    if (l <= tiers) rows += size;
    units += size;
  }
  if (units > ctx->hier.M) return false;  // the node order is not tier by tier
  const long long k = deflated * E - 1;
  if (k < 1 || k > phi::kMaxDeflK) return false;
  out->tiers = tiers;
  out->k = (int)k;
  out->rows_nodes = rows;
  out->unit_nodes = units;
  return true;
}

// want: -1 automatic (ell <= 2 only: the minimal-residual step of
// BiCGSTAB(ell > 2) can lose its Gram matrix on a deflated operator), 0 off,
// 1 or 2 tiers.
int plan_deflation(phi_ctx *ctx, int want, int ell, DeflPlan *plan) {
  *plan = DeflPlan{};
  if (want == 0) return PHI_OK;
  if (want < 0) {  // automatic: the deepest space that fits
    if (ell <= 2 && !defl_fits(ctx, 2, plan)) defl_fits(ctx, 1, plan);
    return PHI_OK;
  }
  if (!defl_fits(ctx, want, plan)) {
    ctx->error = "steady_state: a deflation space of " + std::to_string(want) + " tiers has more than " +
                 std::to_string(phi::kMaxDeflK) + " coordinates for this hierarchy";
    return PHI_E_INVALID;
  }
  return PHI_OK;
}

// A Z by one batched apply of the generic kernel over the nodes of tiers
// 0..tiers (input j: the unit vector Z_j on the nodes of tiers
// 0..tiers+1, which hold every neighbour those rows read), then the
// factors of Z^T A Z.
cudaError_t build_deflation(phi_ctx *ctx, const phi::DeflView &D, const DeflPlan &plan, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(D.units, 0, (size_t)D.k * D.unit_len * sizeof(double2), s);
  if (e == cudaSuccess) e = phi::defl_launch_units(D, s);
  phi::StageLaunch L;
  L.c = ctx->c;
  L.c.M = plan.rows_nodes;
  L.mode = phi::kModeApply;
  L.generic = true;
  L.grid = phi::stage_grid(L.c, ctx->num_sms);
  L.x = D.units;
  L.out = D.AZ;
  L.batch = D.k;
  L.x_bstride = D.unit_len;
  L.out_bstride = D.rows;
  L.mixed = false;
  ctx->bind_filter(L, 0);
  if (e == cudaSuccess) e = phi::launch_stage(L, s);
  if (e == cudaSuccess) e = phi::defl_launch_factor(D, s);
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
                bool guess_rho0, int want_defl, bool *broke_down, phi_solve_stats *stats) {
  *broke_down = false;
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
    if (ctx->bicg_tiles > 0 &&
        ctx->bicg_parts.alloc((size_t)2 * (ctx->bicg_tiles + 1) * sizeof(double)) != cudaSuccess) {
      ctx->error = "steady_state: allocation of the per-tile partial sums failed";
      return PHI_E_OOM;
    }
  }
  DeflPlan plan;
  {
    const int rc = plan_deflation(ctx, want_defl, ell, &plan);
    if (rc != PHI_OK) return rc;
  }
  phi::DeflView D{};
  if (plan.tiers > 0) {
    D.N = N;
    D.E = N * N;
    D.k = plan.k;
    D.k0 = D.E - 1;
    D.n1 = D.k - D.k0;
    D.rows = plan.rows_nodes * D.E;
    D.unit_len = plan.unit_nodes * D.E;
    const int big = D.E > D.k0 ? D.E : D.k0;
    // doubles: Dinv, F, A01, Si, g, c, work
    const size_t dbl = (size_t)D.n1 * D.E + 2 * (size_t)D.n1 * D.k0 + (size_t)D.k0 * D.k0 + 2 * (size_t)D.k +
                       (size_t)big * big;
    const size_t az = (size_t)D.rows * D.k * sizeof(double2);
    const size_t units = (size_t)D.k * D.unit_len * sizeof(double2);
    const size_t dbl_bytes = (dbl * sizeof(double) + 15) / 16 * 16;
    const size_t need = 2 * az + units + dbl_bytes + 16;
    if (ctx->defl_buf.bytes < need) {
      if (ctx->bicg_graph) {  // captured with the old buffer
        cudaGraphExecDestroy(ctx->bicg_graph);
        ctx->bicg_graph = nullptr;
      }
      if (ctx->defl_buf.alloc(need) != cudaSuccess) {
        ctx->error = "steady_state: allocation of the deflation space (" + std::to_string(need) + " bytes) failed";
        return PHI_E_OOM;
      }
    }
    unsigned char *p = ctx->defl_buf.as<unsigned char>();
    D.AZ = reinterpret_cast<double2 *>(p);
    D.AZr = reinterpret_cast<double2 *>(p + az);
    D.units = reinterpret_cast<double2 *>(p + 2 * az);
    double *d = reinterpret_cast<double *>(p + 2 * az + units);
    D.Dinv = d;
    D.F = D.Dinv + (size_t)D.n1 * D.E;
    D.A01 = D.F + (size_t)D.n1 * D.k0;
    D.Si = D.A01 + (size_t)D.k0 * D.n1;
    D.g = D.Si + (size_t)D.k0 * D.k0;
    D.c = D.g + D.k;
    D.work = D.c + D.k;
    D.status = reinterpret_cast<int *>(p + 2 * az + units + dbl_bytes);
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
  // Deflation space; a singular Galerkin matrix leaves the solve undeflated.
  int defl_tiers = 0;
  if (plan.tiers > 0) {
    PHI_SK(build_deflation(ctx, D, plan, s));
    int status = 1;
    PHI_SK(cudaMemcpyAsync(&status, D.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    PHI_SK(cudaStreamSynchronize(s));
    if (status == 0) defl_tiers = plan.tiers;
  }
  const phi::DeflView *Dp = defl_tiers > 0 ? &D : nullptr;
  // The projections inside the iteration stop with the solver; the initial
  // and final ones (D itself, done == NULL) always run.
  phi::DeflView Dloop = D;
  Dloop.done = &sc->done;
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
  if (Dp) {  // r_1 -> r_1 + A Z E^-1 Z^T (b - r_1), so that b - r_1 = P (b - A x_0)
    PHI_SK(phi::defl_launch_coeff(D, V.r[1], V.b, nullptr, s));
    PHI_SK(phi::defl_launch_update(D, V.r[1], s));
  }
  phi::BicgScalars init{};
  init.tol = tol;
  init.tol_mode = tol_mode;
  init.max_steps = max_steps;
  init.ell = ell;
  PHI_SK(cudaMemcpyAsync(sc, &init, offsetof(phi::BicgScalars, partials), cudaMemcpyHostToDevice, s));
  PHI_SK(phi::bicg_launch_init(V, n, sc, grid, s));
  if (Dp) PHI_SK(phi::defl_launch_g(D, V.rhat, s));
  PHI_SK(cudaStreamSynchronize(s));  // the host staging above is stack memory

  // Replay graphs of several outer iterations until the device says done.
  const int outer_per_graph = ell >= 8 ? 1 : 8 / ell;
  if (ctx->bicg_graph && (ctx->bicg_ell != ell || ctx->bicg_defl != defl_tiers)) {
    cudaGraphExecDestroy(ctx->bicg_graph);
    ctx->bicg_graph = nullptr;
  }
  if (!ctx->bicg_graph) {
    cudaGraph_t graph = nullptr;
    PHI_SK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t eb = cudaSuccess;
    for (int it = 0; it < outer_per_graph && eb == cudaSuccess; ++it)
      eb = outer_iteration(ctx, V, n, sc, ell, grid, s, Dp ? &Dloop : nullptr);
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
    ctx->bicg_defl = defl_tiers;
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
  if (result == PHI_OK && Dp) {
    // The coarse part: x = y + Z E^-1 Z^T (b - A y).
    cudaError_t e = apply_fp64(ctx, V.x, V.r[1], s);
    if (e == cudaSuccess) e = phi::defl_launch_coeff(D, V.r[1], V.b, nullptr, s);
    if (e == cudaSuccess) e = phi::defl_launch_correct(D, V.x, s);
    if (e != cudaSuccess) result = steady_err(ctx, e, "coarse correction");
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
      stats->deflated_tiers = defl_tiers;
      stats->deflation_size = defl_tiers > 0 ? D.k : 0;
    }
    if (!host->converged) {
      *broke_down = host->breakdown != 0;
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

// The solve with the context's deflation setting; an automatically
// deflated solve that breaks down is run again undeflated from the same
// guess (the statistics then count both runs' steps and time).
int steady_solve(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode, int32_t max_steps, const double *guess,
                 bool guess_rho0, phi_solve_stats *stats) {
  if (!ctx) return PHI_E_INVALID;
  phi_solve_stats first{};
  bool broke = false;
  int rc = steady_impl(ctx, ell, tol, tol_mode, max_steps, guess, guess_rho0, ctx->steady_defl, &broke, &first);
  if (rc == PHI_E_NO_CONVERGENCE && broke && ctx->steady_defl < 0 && first.deflated_tiers > 0) {
    phi_solve_stats again{};
    rc = steady_impl(ctx, ell, tol, tol_mode, max_steps, guess, guess_rho0, 0, &broke, &again);
    again.iterations += first.iterations;
    again.seconds += first.seconds;
    first = again;
  }
  if (stats) *stats = first;
  return rc;
}

}  // namespace

extern "C" int phi_gpu_steady_state(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode, int32_t max_steps,
                                    const double *guess, phi_solve_stats *stats) {
  return steady_solve(ctx, ell, tol, tol_mode, max_steps, guess, false, stats);
}

extern "C" int phi_gpu_steady_state_rho0(phi_ctx *ctx, int32_t ell, double tol, int32_t tol_mode,
                                         int32_t max_steps, const double *rho0_guess, phi_solve_stats *stats) {
  if (!rho0_guess) {
    if (ctx) ctx->error = "steady_state_rho0: rho0_guess is NULL";
    return PHI_E_INVALID;
  }
  return steady_solve(ctx, ell, tol, tol_mode, max_steps, rho0_guess, true, stats);
}

extern "C" int phi_gpu_set_steady_deflation(phi_ctx *ctx, int32_t tiers) {
  if (!ctx) return PHI_E_INVALID;
  if (tiers < -1 || tiers > 2) {
    ctx->error = "set_steady_deflation: tiers must be -1 (automatic), 0, 1 or 2";
    return PHI_E_INVALID;
  }
  if (tiers > 0) {
    DeflPlan plan;
    if (!defl_fits(ctx, tiers, &plan)) {
      ctx->error = "set_steady_deflation: a deflation space of " + std::to_string(tiers) +
                   " tiers has more than " + std::to_string(phi::kMaxDeflK) + " coordinates for this hierarchy";
      return PHI_E_INVALID;
    }
  }
  ctx->steady_defl = tiers;
  return PHI_OK;
}
