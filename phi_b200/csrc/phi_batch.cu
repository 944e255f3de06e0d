// phi_batch.cu -- phi_gpu_batch_*: many independent hierarchies, every RK4
// stage of all of them in one persistent launch (heom_tile_batch.cu), the
// step loop replayed from a CUDA graph, the launch schedule picked by timing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_kernels.h"
#include "heom_tile.h"
#include "phi_context.h"

namespace {

constexpr int kBatchGraphSteps = 16;
std::string g_batch_create_error;

// Device arrays of one stage plan (tile parameters in work order + the
// prefix of tile counts).
struct StagePlan {
  phi::DeviceBuffer params, tile_start;
  phi::TileBatchPlan plan;
};

}  // namespace

struct phi_batch {
  std::vector<phi_ctx *> inst;
  int num_sms = 148;
  int device = 0;
  bool mixed = false;
  cudaStream_t stream = nullptr;
  phi::DeviceBuffer err;  // batch-level flag of the persistent kernel
  phi_batch_schedule sched{1, 1, 0.0};
  // RK4 stage plans for (dt, schedule) and the captured graph of them.
  double plan_dt = 0.0;
  int plan_order = -1;
  StagePlan rk4[4];
  cudaGraphExec_t graph = nullptr;
  int graph_grid = 0;
  std::string error;

  ~phi_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    for (phi_ctx *c : inst) phi_gpu_destroy(c);
    if (stream) cudaStreamDestroy(stream);
  }
  int fail(int code, const std::string &msg) {
    error = msg;
    return code;
  }
  int cuda_fail(cudaError_t e, const char *where) {
    error = std::string(where) + ": " + cudaGetErrorString(e);
    return PHI_E_CUDA;
  }
  std::vector<int> work_order(int order) const {
    std::vector<int> idx(inst.size());
    std::iota(idx.begin(), idx.end(), 0);
    if (order == 1) {
      // Largest per-tile work first (N^2 * tile nodes ~ constant per tile, so
      // order by N, then by tile count), so the tail of the launch is made of
      // short tiles.
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        const phi::HeomConsts &ca = inst[a]->c, &cb = inst[b]->c;
        if (ca.N != cb.N) return ca.N > cb.N;
        return phi::tile_count(ca, inst[a]->mixed()) > phi::tile_count(cb, inst[b]->mixed());
      });
    }
    return idx;
  }
  int grid() const { return std::max(1, sched.ctas_per_sm) * num_sms; }
};

namespace {

// Stage launch of instance c for RK4 stage `st` (as enqueue_rk4_step builds
// it for one context), or the plain apply y -> xb when st < 0.
phi::StageLaunch stage_launch(phi_ctx *c, int st, double dt) {
  phi::StageLaunch L;
  L.c = c->c;
  L.grid = c->grid;
  L.mixed = c->mixed();
  L.y = c->y.as<double2>();
  L.acc = c->acc.as<double2>();
  L.y32 = c->y32.ptr;
  L.rk4 = c->ctl.as<phi::Rk4Ctl>();
  L.traj = nullptr;
  const void *y_in = L.mixed ? c->y32.ptr : c->y.ptr;
  if (st < 0) {
    L.mode = phi::kModeApply;
    L.xv = y_in;
    L.outv = c->xb.ptr;
    L.x = static_cast<const double2 *>(y_in);
    L.out = c->xb.as<double2>();
    return L;
  }
  const double a[4] = {dt / 2, dt / 2, dt, 0.0};
  const double w[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
  const void *inv[4] = {y_in, c->xa.ptr, c->xb.ptr, c->xa.ptr};
  void *outv[4] = {c->xa.ptr, c->xb.ptr, c->xa.ptr, nullptr};
  L.mode = phi::kModeRk4;
  L.stage = st;
  L.xv = inv[st];
  L.outv = outv[st];
  L.x = static_cast<const double2 *>(inv[st]);
  L.out = static_cast<double2 *>(outv[st]);
  L.a_next = a[st];
  L.w_acc = w[st];
  return L;
}

int build_plan(phi_batch *b, int st, double dt, int order, StagePlan *sp) {
  const std::vector<int> idx = b->work_order(order);
  const size_t pb = phi::tile_params_bytes();
  std::vector<unsigned char> params(pb * idx.size());
  std::vector<long long> start(idx.size() + 1, 0);
  size_t smem = 0;
  for (size_t k = 0; k < idx.size(); ++k) {
    const phi::StageLaunch L = stage_launch(b->inst[idx[k]], st, dt);
    phi::tile_params_host(L, params.data() + k * pb);
    start[k + 1] = start[k] + phi::tile_count(L.c, L.mixed);
    smem = std::max(smem, phi::tile_stage_smem(L));
  }
  if (!sp->params.ptr || sp->params.bytes < params.size()) {
    if (sp->params.alloc(params.size()) != cudaSuccess) return b->fail(PHI_E_OOM, "batch plan allocation failed");
  }
  if (!sp->tile_start.ptr || sp->tile_start.bytes < start.size() * sizeof(long long)) {
    if (sp->tile_start.alloc(start.size() * sizeof(long long)) != cudaSuccess)
      return b->fail(PHI_E_OOM, "batch plan allocation failed");
  }
  cudaError_t e = cudaMemcpyAsync(sp->params.ptr, params.data(), params.size(), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sp->tile_start.ptr, start.data(), start.size() * sizeof(long long), cudaMemcpyHostToDevice,
                        b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);  // host staging is local
  if (e != cudaSuccess) return b->cuda_fail(e, "batch plan upload");
  sp->plan.params = sp->params.ptr;
  sp->plan.tile_start = sp->tile_start.as<long long>();
  sp->plan.count = (int)idx.size();
  sp->plan.total_tiles = start.back();
  sp->plan.smem = smem;
  sp->plan.mixed = b->mixed;
  sp->plan.err_flag = b->err.as<int>();
  return PHI_OK;
}

int check_flags(phi_batch *b) {
  int flag = 0;
  cudaError_t e = cudaMemcpy(&flag, b->err.ptr, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return b->cuda_fail(e, "batch flag read");
  for (size_t i = 0; i < b->inst.size(); ++i) {
    const int rc = b->inst[i]->check_device_flag();
    if (rc != PHI_OK) return b->fail(rc, "instance " + std::to_string(i) + ": " + b->inst[i]->error);
  }
  if (flag) return b->fail(PHI_E_TIMEOUT, "a bounded device wait of the batch kernel gave up");
  return PHI_OK;
}

}  // namespace

extern "C" int phi_gpu_batch_create(const phi_problem_desc *descs, int32_t count, phi_batch **out) {
  if (!out) return PHI_E_INVALID;
  *out = nullptr;
  if (!descs || count <= 0) {
    g_batch_create_error = "descs is NULL or count <= 0";
    return PHI_E_INVALID;
  }
  std::unique_ptr<phi_batch> b(new phi_batch());
  b->mixed = descs[0].precision == PHI_PREC_MIXED;
  b->device = descs[0].device;
  for (int i = 0; i < count; ++i) {
    if (descs[i].precision != descs[0].precision || descs[i].device != descs[0].device) {
      g_batch_create_error = "instance " + std::to_string(i) + ": every instance needs the same precision and device";
      return PHI_E_INVALID;
    }
    if (descs[i].annealing_h_x) {
      g_batch_create_error = "instance " + std::to_string(i) +
                             ": annealing Hamiltonians run on single hierarchies (phi_gpu_rk4 / phi_gpu_rkf45)";
      return PHI_E_INVALID;
    }
    if (descs[i].time_local) {
      g_batch_create_error = "instance " + std::to_string(i) +
                             ": time-local truncation runs on single hierarchies (phi_gpu_rk4 / phi_gpu_rkf45)";
      return PHI_E_INVALID;
    }
    if (descs[i].filter_tolerance > 0 && descs[i].bath_kind == PHI_BATH_INDEPENDENT) {
      g_batch_create_error = "instance " + std::to_string(i) +
                             ": hierarchy filtering runs on single hierarchies (phi_gpu_rk4 / phi_gpu_rkf45)";
      return PHI_E_INVALID;
    }
    phi_ctx *c = nullptr;
    const int rc = phi_gpu_create(&descs[i], &c);
    if (rc != PHI_OK) {
      char buf[512];
      phi_gpu_last_error(nullptr, buf, sizeof buf);
      g_batch_create_error = "instance " + std::to_string(i) + ": " + buf;
      return rc;
    }
    b->inst.push_back(c);
    if (!phi::tile_kernel_available(c->c)) {
      g_batch_create_error = "instance " + std::to_string(i) +
                             ": batching needs IndependentBath on the identity site map, K + 1 <= 3 and N in "
                             "{2..8, 10, 12, 16, 24}";
      return PHI_E_INVALID;
    }
    const int wr = c->ensure_work(2);
    if (wr != PHI_OK) {
      g_batch_create_error = "instance " + std::to_string(i) + ": " + c->error;
      return wr;
    }
  }
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
  if (e == cudaSuccess) e = b->err.alloc(sizeof(int)) == cudaSuccess ? cudaMemset(b->err.ptr, 0, sizeof(int)) : cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaDeviceSynchronize();  // instance streams idle before the batch stream uses their buffers
  if (e != cudaSuccess) {
    g_batch_create_error = std::string("batch setup: ") + cudaGetErrorString(e);
    return PHI_E_CUDA;
  }
  *out = b.release();
  return PHI_OK;
}

extern "C" int phi_gpu_batch_destroy(phi_batch *batch) {
  if (!batch) return PHI_OK;
  if (batch->stream) cudaStreamSynchronize(batch->stream);
  delete batch;
  return PHI_OK;
}

extern "C" int phi_gpu_batch_instance(phi_batch *batch, int32_t index, phi_ctx **ctx) {
  if (!batch || !ctx) return PHI_E_INVALID;
  if (index < 0 || index >= (int)batch->inst.size()) return batch->fail(PHI_E_INVALID, "instance index out of range");
  if (batch->stream) cudaStreamSynchronize(batch->stream);
  *ctx = batch->inst[index];
  return PHI_OK;
}

extern "C" int phi_gpu_batch_set_schedule(phi_batch *batch, const phi_batch_schedule *s) {
  if (!batch || !s) return PHI_E_INVALID;
  if (s->ctas_per_sm < 1 || s->ctas_per_sm > 32 || (s->order != 0 && s->order != 1))
    return batch->fail(PHI_E_INVALID, "schedule: ctas_per_sm in 1..32 and order 0 or 1");
  if (s->ctas_per_sm != batch->sched.ctas_per_sm || s->order != batch->sched.order) {
    if (batch->graph) cudaGraphExecDestroy(batch->graph);
    batch->graph = nullptr;
    batch->plan_order = -1;
  }
  batch->sched = *s;
  return PHI_OK;
}

extern "C" int phi_gpu_batch_autotune(phi_batch *batch, phi_batch_schedule *chosen) {
  if (!batch) return PHI_E_INVALID;
  // Mixed: the apply reads the complex64 copy of y.
  if (batch->mixed) {
    for (phi_ctx *c : batch->inst) {
      cudaError_t e = phi::launch_to_c64(c->y.as<double2>(), c->y32.as<float2>(), c->hier.M,
                                         c->desc.num_states * c->desc.num_states, c->work_stride(), batch->stream);
      if (e != cudaSuccess) return batch->cuda_fail(e, "autotune");
    }
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return batch->fail(PHI_E_CUDA, "autotune: event creation failed");
  phi_batch_schedule best{1, 0, 0.0};
  double best_ms = 1e300;
  int rc = PHI_OK;
  for (int order = 0; order <= 1 && rc == PHI_OK; ++order) {
    StagePlan sp;
    rc = build_plan(batch, -1, 0.0, order, &sp);
    if (rc != PHI_OK) break;
    const int occ = std::max(1, phi::tile_batch_occupancy(sp.plan));
    for (int cps = 1; cps <= occ && rc == PHI_OK; ++cps) {
      const int grid = cps * batch->num_sms;
      cudaError_t e = phi::launch_tile_batch(sp.plan, grid, batch->stream);  // warm-up
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventRecord(e0, batch->stream);
      for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = phi::launch_tile_batch(sp.plan, grid, batch->stream);
      if (e == cudaSuccess) e = cudaEventRecord(e1, batch->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        rc = batch->cuda_fail(e, "autotune");
        break;
      }
      if (ms / 3 < best_ms) {
        best_ms = ms / 3;
        best = phi_batch_schedule{cps, order, ms / 3.0};
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != PHI_OK) return rc;
  rc = check_flags(batch);
  if (rc != PHI_OK) return rc;
  rc = phi_gpu_batch_set_schedule(batch, &best);
  batch->sched.ms_per_stage = best.ms_per_stage;
  if (chosen) *chosen = batch->sched;
  return rc;
}

extern "C" int phi_gpu_batch_rk4(phi_batch *batch, double dt, int64_t steps, phi_batch_stats *stats) {
  if (!batch) return PHI_E_INVALID;
  if (!(dt > 0) || steps < 0) return batch->fail(PHI_E_INVALID, "batch rk4: dt must be positive and steps >= 0");
  cudaStream_t s = batch->stream;
  // Stage plans for this dt and schedule (dt enters the stage coefficients).
  if (batch->plan_dt != dt || batch->plan_order != batch->sched.order) {
    for (int st = 0; st < 4; ++st) {
      const int rc = build_plan(batch, st, dt, batch->sched.order, &batch->rk4[st]);
      if (rc != PHI_OK) return rc;
    }
    batch->plan_dt = dt;
    batch->plan_order = batch->sched.order;
    if (batch->graph) cudaGraphExecDestroy(batch->graph);
    batch->graph = nullptr;
  }
  const int grid = batch->grid();
  if (batch->graph && batch->graph_grid != grid) {
    cudaGraphExecDestroy(batch->graph);
    batch->graph = nullptr;
  }
  auto enqueue_step = [&]() -> cudaError_t {
    for (int st = 0; st < 4; ++st) {
      cudaError_t e = phi::launch_tile_batch(batch->rk4[st].plan, grid, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  if (batch->mixed) {
    for (phi_ctx *c : batch->inst) {
      cudaError_t e = phi::launch_to_c64(c->y.as<double2>(), c->y32.as<float2>(), c->hier.M,
                                         c->desc.num_states * c->desc.num_states, c->work_stride(), s);
      if (e != cudaSuccess) return batch->cuda_fail(e, "batch rk4");
    }
  }
  if (!batch->graph && steps >= kBatchGraphSteps) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return batch->cuda_fail(e, "batch capture");
    cudaError_t eb = cudaSuccess;
    for (int k = 0; k < kBatchGraphSteps && eb == cudaSuccess; ++k) eb = enqueue_step();
    e = cudaStreamEndCapture(s, &g);
    if (eb != cudaSuccess || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return batch->cuda_fail(eb != cudaSuccess ? eb : e, "batch capture");
    }
    e = cudaGraphInstantiate(&batch->graph, g, 0);
    cudaGraphDestroy(g);
    if (e == cudaSuccess) e = cudaGraphUpload(batch->graph, s);  // not on the first launch
    if (e != cudaSuccess) return batch->cuda_fail(e, "batch graph instantiate");
    batch->graph_grid = grid;
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return batch->fail(PHI_E_CUDA, "batch rk4: event creation failed");
  cudaError_t e = cudaEventRecord(e0, s);
  long long done = 0, launches = 0;
  while (e == cudaSuccess && done + kBatchGraphSteps <= steps && batch->graph) {
    e = cudaGraphLaunch(batch->graph, s);
    done += kBatchGraphSteps;
    launches += 4 * kBatchGraphSteps;
  }
  while (e == cudaSuccess && done < steps) {
    e = enqueue_step();
    ++done;
    launches += 4;
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return batch->cuda_fail(e, "batch rk4");
  const int rc = check_flags(batch);
  if (rc != PHI_OK) return rc;
  long long nodes = 0;
  for (phi_ctx *c : batch->inst) {
    nodes += c->hier.M;
    for (long long k = 0; k < steps; ++k) c->time += dt;  // the reference's time accumulation
  }
  if (stats) {
    stats->steps = steps;
    stats->node_applies = 4 * steps * nodes;
    stats->seconds = ms / 1e3;
    stats->launches = launches;
  }
  return PHI_OK;
}

extern "C" int phi_gpu_batch_last_error(const phi_batch *batch, char *buf, size_t len) {
  if (!buf || len == 0) return PHI_E_INVALID;
  const std::string &s = batch ? batch->error : g_batch_create_error;
  std::snprintf(buf, len, "%s", s.c_str());
  return PHI_OK;
}
