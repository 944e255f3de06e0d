// phi_capi.cu -- the C ABI (include/phi_b200.h): one hierarchy instance on
// one GPU.  Host-side setup restates the constants PHI computes in
// HierarchyIntegrator::Initialize / InitializePrefactors
// (hierarchy_integrator.cc:376-594, :1343-1466); everything per node lives on
// the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_device.cuh"
#include "heom_internal.h"
#include "heom_kernels.h"
#include "heom_tile.h"
#include "heom_timelocal.h"
#include "heom_anneal.h"
#include "phi_context.h"
#include "phi_truncation.h"

using phi::DeviceBuffer;

namespace {

thread_local std::string g_create_error;

// hierarchy_node.h:7
constexpr double kPi = 3.14159265358979323846264338327950288419716939937510;

int fail(phi_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->error = msg;
  else g_create_error = msg;
  return code;
}

int cuda_fail(phi_ctx *ctx, cudaError_t e, const char *where) {
  return fail(ctx, PHI_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define PHI_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
  } while (0)

template <class T>
cudaError_t upload(DeviceBuffer &buf, const std::vector<T> &v, cudaStream_t s) {
  cudaError_t e = buf.alloc(std::max<size_t>(v.size() * sizeof(T), 16));
  if (e != cudaSuccess) return e;
  if (v.empty()) return cudaSuccess;
  return cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

bool is_hermitian(const double *m, int N, double *scale_out) {
  double scale = 0;
  for (int k = 0; k < N * N; ++k) scale = std::max(scale, std::hypot(m[2 * k], m[2 * k + 1]));
  const double tol = 1e-12 * std::max(scale, 1e-300);
  for (int r = 0; r < N; ++r)
    for (int c = 0; c < N; ++c) {
      const double *a = m + 2 * (r + c * N), *b = m + 2 * (c + r * N);
      if (std::fabs(a[0] - b[0]) > tol || std::fabs(a[1] + b[1]) > tol) return false;
    }
  if (scale_out) *scale_out = scale;
  return true;
}

}  // namespace

namespace phi {

// Builds the per-term / per-element constant tables and the device copy of
// the problem (see HeomConsts).
namespace {
// Dephasing rate of every node, sum_t n_t nu_t in term order (the tile
// kernels' per-node dephasing, DoDephasing, hierarchy_updater.h:71-75).
__global__ void node_dephasing_kernel(const uint8_t *__restrict__ mi, const double *__restrict__ nu, long long M,
                                      int T, double *__restrict__ out) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < M; n += (long long)gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int t = 0; t < T; ++t) d = fma((double)mi[n * T + t], nu[t], d);
    out[n] = d;
  }
}
}  // namespace

int setup_constants(phi_ctx *ctx) {
  const phi_problem_desc &d = ctx->desc;
  const int N = d.num_states, nb = d.num_baths, K1 = d.num_matsubara_terms;
  const int T = nb * K1, L = d.truncation_level - 1, E = N * N;
  const double hbar = d.hbar;
  const double thermal = d.boltzmann_constant * d.temperature;
  const double nu = 2 * kPi * thermal / hbar;

  // Correlation-function constants c_t, t = b*(K+1) + k
  // (hierarchy_integrator.cc:427-473).
  std::vector<std::complex<double>> corr(T, 0.0);
  std::vector<double> abs_corr(T, 0.0), rates(T, 0.0), delta(nb, 0.0);
  for (int b = 0; b < nb; ++b) {
    const double g = ctx->gamma[b], l = ctx->lambda[b];
    if (g > 0) {
      const double a = g * l / hbar;
      corr[b * K1] = std::complex<double>(a / std::tan(g * hbar / (2 * thermal)), -a);
      for (int k = 1; k < K1; ++k)
        corr[b * K1 + k] = 4 * l * g * thermal / hbar / hbar * (nu * k) /
                           (std::pow(nu * k, 2) - std::pow(g, 2));
      // Matsubara/residual correction (:1375-1389).
      double dl = 2 * l * thermal / hbar / hbar / g - l / hbar / std::tan(hbar * g / (2 * thermal));
      for (int k = 1; k < K1; ++k) dl -= 4 * l * thermal / hbar / hbar * g / (std::pow(nu * k, 2) - std::pow(g, 2));
      delta[b] = dl;
    }
    for (int k = 0; k < K1; ++k) abs_corr[b * K1 + k] = std::abs(corr[b * K1 + k]);
    // Dephasing rate of each term (:1362-1371): gamma for k = 0, nu*k else.
    for (int k = 0; k < K1; ++k) rates[b * K1 + k] = k == 0 ? g : nu * k;
  }
  ctx->corr = corr;
  ctx->delta = delta;

  // A single tier runs PHI's Vacuum updater (unitary part only) unless
  // time-local truncation is on, which selects NoHierarchyIndependentBath:
  // unitary + Matsubara + time-local (hierarchy_integrator.cc:1741-1758).
  const bool single_tier = d.truncation_level == 1;
  const bool vacuum = single_tier && !d.time_local;
  const bool normalized = d.normalized != 0;
  if (!single_tier && d.bath_kind != PHI_BATH_DIAGONAL && normalized) {
    for (int t = 0; t < T; ++t)
      if (!(abs_corr[t] > 0))
        return fail(ctx, PHI_E_INVALID,
                    "correlation constant |c_" + std::to_string(t) +
                        "| is zero (gamma or lambda <= 0): the normalised hierarchy is undefined");
  }
  // Prefactor magnitudes for n_t = 0..L+1 (:1393-1441).
  const int W = L + 2;
  std::vector<double> sq_next((size_t)T * W, 1.0), sq_prev((size_t)T * W, 0.0);
  for (int t = 0; t < T; ++t)
    for (int n = 0; n < W; ++n) {
      sq_next[(size_t)t * W + n] = normalized ? std::sqrt((n + 1) * abs_corr[t]) : 1.0;
      sq_prev[(size_t)t * W + n] =
          normalized ? (n > 0 ? std::sqrt(n / abs_corr[t]) : 0.0) : (double)n;
    }

  // Coupling map.  IndependentBath: term t couples to site s_{t/(K+1)};
  // DiagonalBath / FullBath: to bath operator t/(K+1)
  // (LinkHierarchyNodes, :1291-1293 and :1320-1322).
  std::vector<int32_t> term_site(T), site_ptr(N + 1, 0), site_terms(T);
  std::vector<double> site_delta(N, 0.0);
  for (int t = 0; t < T; ++t) {
    const int b = t / K1;
    term_site[t] = d.bath_kind == PHI_BATH_INDEPENDENT ? ctx->bath_sites[b] : b;
  }
  if (d.bath_kind == PHI_BATH_INDEPENDENT) {
    for (int t = 0; t < T; ++t) site_ptr[term_site[t] + 1]++;
    for (int s = 0; s < N; ++s) site_ptr[s + 1] += site_ptr[s];
    std::vector<int32_t> fill(site_ptr.begin(), site_ptr.end() - 1);
    for (int t = 0; t < T; ++t) site_terms[fill[term_site[t]]++] = t;
    for (int b = 0; b < nb; ++b) site_delta[ctx->bath_sites[b]] += delta[b];
  }
  // Element-wise Matsubara factor: IndependentBath::DoMatsubara
  // (hierarchy_updater.cc:129-144) and DiagonalBath same operator
  // (hierarchy.cc:167-168); FullBath and Vacuum use none here.
  std::vector<double> mats_elem(E, 0.0);
  if (!vacuum) {
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double f = 0.0;
        if (d.bath_kind == PHI_BATH_INDEPENDENT) {
          if (i != j) f = site_delta[i] + site_delta[j];
        } else if (d.bath_kind == PHI_BATH_DIAGONAL) {
          for (int b = 0; b < nb; ++b) {
            const double dv = ctx->coupling[(size_t)b * N + i] - ctx->coupling[(size_t)b * N + j];
            f += delta[b] * dv * dv;
          }
        }
        mats_elem[i + j * N] = f;
      }
  }
  std::vector<uint8_t> pi, pj;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i <= j; ++i) {
      pi.push_back((uint8_t)i);
      pj.push_back((uint8_t)j);
    }
  std::vector<double2> H(E), corr2(T);
  for (int k = 0; k < E; ++k) H[k] = make_double2(ctx->hamiltonian[2 * k], ctx->hamiltonian[2 * k + 1]);
  for (int t = 0; t < T; ++t) corr2[t] = make_double2(corr[t].real(), corr[t].imag());

  cudaStream_t s = ctx->stream;
  auto &cb = ctx->cbuf;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
  chk(upload(cb.H, H, s));
  chk(upload(cb.corr, corr2, s));
  chk(upload(cb.nu, rates, s));
  chk(upload(cb.sq_next, sq_next, s));
  chk(upload(cb.sq_prev, sq_prev, s));
  chk(upload(cb.term_site, term_site, s));
  chk(upload(cb.site_ptr, site_ptr, s));
  chk(upload(cb.site_terms, site_terms, s));
  chk(upload(cb.mats_elem, mats_elem, s));
  chk(upload(cb.bath_V, ctx->coupling, s));
  chk(upload(cb.mats_bath, delta, s));
  chk(upload(cb.pair_i, pi, s));
  chk(upload(cb.pair_j, pj, s));
  chk(cb.err_flag.alloc(sizeof(int)));
  chk(cudaMemsetAsync(cb.err_flag.ptr, 0, sizeof(int), s));
  // Per-node dephasing rates, 2 doubles of slack: the tile kernels copy a
  // tile's rates as a 16-byte aligned window.
  const long long Mn = ctx->hier.M;
  chk(cb.deph_node.alloc((size_t)(Mn + 2) * sizeof(double)));
  chk(cudaMemsetAsync(cb.deph_node.ptr, 0, (size_t)(Mn + 2) * sizeof(double), s));
  if (e == cudaSuccess && T > 0 && Mn > 0) {
    node_dephasing_kernel<<<(unsigned)std::min<long long>((Mn + 255) / 256, 4096), 256, 0, s>>>(
        ctx->hier.mi.as<uint8_t>(), cb.nu.as<double>(), Mn, T, cb.deph_node.as<double>());
    chk(cudaGetLastError());
  }
  chk(cudaStreamSynchronize(s));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "constant upload");

  HeomConsts &c = ctx->c;
  c.N = N;
  c.T = T;
  c.K1 = K1;
  c.nb = nb;
  c.L = L;
  c.kind = d.bath_kind;
  c.vacuum = vacuum ? 1 : 0;
  c.identity_sites = 0;
  if (d.bath_kind == PHI_BATH_INDEPENDENT && nb == N) {
    c.identity_sites = 1;
    for (int b = 0; b < nb; ++b)
      if (ctx->bath_sites[b] != b) c.identity_sites = 0;
  }
  c.h_real = 1;
  for (int k = 0; k < N * N; ++k)
    if (ctx->hamiltonian[2 * k + 1] != 0.0) c.h_real = 0;
  c.M = ctx->hier.M;
  c.inv_hbar = 1.0 / hbar;
  c.mi = ctx->hier.mi.as<uint8_t>();
  c.next = ctx->hier.next.as<int32_t>();
  c.prev = ctx->hier.prev.as<int32_t>();
  c.H = cb.H.as<double2>();
  c.corr = cb.corr.as<double2>();
  c.nu = cb.nu.as<double>();
  c.deph_node = cb.deph_node.as<double>();
  c.sq_next = cb.sq_next.as<double>();
  c.sq_prev = cb.sq_prev.as<double>();
  c.term_site = cb.term_site.as<int32_t>();
  c.site_ptr = cb.site_ptr.as<int32_t>();
  c.site_terms = cb.site_terms.as<int32_t>();
  c.mats_elem = cb.mats_elem.as<double>();
  c.bath_V = cb.bath_V.as<double>();
  c.mats_bath = cb.mats_bath.as<double>();
  c.pair_i = cb.pair_i.as<uint8_t>();
  c.pair_j = cb.pair_j.as<uint8_t>();
  c.err_flag = cb.err_flag.as<int>();
  // FixIncompatibleCombinations keeps filtering for independent baths only
  // (phi_parameters.cc:847-851); a single tier has no neighbours to filter.
  c.filtered = (d.bath_kind == PHI_BATH_INDEPENDENT && d.filter_tolerance > 0 && !single_tier) ? 1 : 0;
  c.filter_tol = c.filtered ? d.filter_tolerance : 0.0;
  c.time_local = d.time_local ? 1 : 0;
  c.tl_q = nullptr;  // bound once the matrices are allocated
  return PHI_OK;
}

void set_create_error(const std::string &msg) { g_create_error = msg; }

}  // namespace phi

// --------------------------------------------------------------------------

namespace {

// Tile-kernel schedules chosen so far in this process, per (device, N, K+1,
// arithmetic, log2 of the node count).
std::mutex g_sched_mu;
std::map<std::tuple<int, int, int, int, int>, phi::TileSchedule> g_sched;
constexpr long long kTuneMinElements = 1ll << 20;  // smaller problems keep the default schedule

// The tile-shape autotuner: for a tile-eligible problem of at least
// kTuneMinElements complex elements, times one Liouvillian apply for each
// block-size variant and CTAs-per-SM cap (phi::tile_autotune) and keeps the
// fastest; every result is the same bit for bit (each element's arithmetic
// does not depend on the tile it falls in), only the time changes.
int tune_tile_schedule(phi_ctx *ctx) {
  if (!phi::tile_kernel_available(ctx->c)) return PHI_OK;
  const int N = ctx->desc.num_states;
  if (ctx->hier.M * N * N < kTuneMinElements) return PHI_OK;
  int lg = 0;
  for (long long m = ctx->hier.M; m > 1; m >>= 1) ++lg;
  const auto key = std::make_tuple(ctx->desc.device, N, ctx->c.K1, ctx->mixed() ? 1 : 0, lg);
  {
    std::lock_guard<std::mutex> lock(g_sched_mu);
    auto it = g_sched.find(key);
    if (it != g_sched.end()) {
      ctx->tile_sched = it->second;
      ctx->c.tile_variant = it->second.variant;
      ctx->c.tile_cps = it->second.cps;
      return PHI_OK;
    }
  }
  int rc = ctx->ensure_work(1);
  if (rc != PHI_OK) return rc;
  phi::StageLaunch L;
  L.c = ctx->c;
  L.mode = phi::kModeApply;
  L.grid = ctx->grid;
  L.mixed = ctx->mixed();
  if (L.mixed) {  // complex64 input from the state, output to the other stage buffer
    PHI_CUDA(ctx, phi::launch_to_c64(ctx->y.as<double2>(), ctx->xa.as<float2>(), ctx->hier.M, N * N,
                                     ctx->work_stride(), ctx->stream));
    L.xv = ctx->xa.ptr;
    L.outv = ctx->xb.ptr;
  } else {
    L.xv = ctx->y.ptr;
    L.outv = ctx->xa.ptr;
  }
  L.x = static_cast<const double2 *>(L.xv);
  L.out = static_cast<double2 *>(L.outv);
  ctx->bind_filter(L, 0);
  phi::TileSchedule sched;
  PHI_CUDA(ctx, phi::tile_autotune(L, ctx->stream, &sched));
  rc = ctx->check_device_flag();
  if (rc != PHI_OK) return rc;
  ctx->tile_sched = sched;
  ctx->c.tile_variant = sched.variant;
  ctx->c.tile_cps = sched.cps;
  std::lock_guard<std::mutex> lock(g_sched_mu);
  g_sched[key] = sched;
  return PHI_OK;
}

}  // namespace

extern "C" int phi_gpu_create(const phi_problem_desc *desc, phi_ctx **out) {
  if (!out) return fail(nullptr, PHI_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!desc) return fail(nullptr, PHI_E_INVALID, "desc is NULL");
  const phi_problem_desc &d = *desc;
  const int N = d.num_states;
  if (N < 1 || N > phi::kMaxStates) return fail(nullptr, PHI_E_INVALID, "num_states must be in [1, 64]");
  if (d.num_baths < 1) return fail(nullptr, PHI_E_INVALID, "num_baths must be >= 1");
  if (d.num_matsubara_terms < 1) return fail(nullptr, PHI_E_INVALID, "num_matsubara_terms (K+1) must be >= 1");
  if (d.truncation_level < 1) return fail(nullptr, PHI_E_INVALID, "truncation_level must be >= 1");
  const long long T = (long long)d.num_baths * d.num_matsubara_terms;
  if (T > phi::kMaxTerms) return fail(nullptr, PHI_E_INVALID, "num_baths * (K+1) must be <= 64");
  if (d.truncation_level - 1 > phi::kMaxTier) return fail(nullptr, PHI_E_INVALID, "truncation_level must be <= 251");
  if (d.bath_kind < PHI_BATH_INDEPENDENT || d.bath_kind > PHI_BATH_FULL)
    return fail(nullptr, PHI_E_INVALID, "unknown bath_kind");
  if (d.precision != PHI_PREC_FP64 && d.precision != PHI_PREC_MIXED)
    return fail(nullptr, PHI_E_INVALID, "unknown precision");
  if (d.hilbert_space_size != 0 && d.hilbert_space_size < N)
    return fail(nullptr, PHI_E_INVALID, "hilbert_space_size cannot be less than num_states");
  if (d.hilbert_space_size > N) {
    // Hilbert-space truncation: restate the problem in the lowest num_states
    // eigenvectors of the Hamiltonian, then build an ordinary context.
    if (d.hilbert_space_size > 1024) return fail(nullptr, PHI_E_INVALID, "hilbert_space_size must be <= 1024");
    const bool anneal_t = d.annealing_h_x != nullptr;
    if ((!d.hamiltonian && !anneal_t) || !d.initial_density_matrix)
      return fail(nullptr, PHI_E_INVALID, "hamiltonian and initial_density_matrix are required");
    const int F = d.hilbert_space_size;
    for (int k = 0; k < 2 * F * F; ++k)
      if ((!anneal_t && !std::isfinite(d.hamiltonian[k])) || !std::isfinite(d.initial_density_matrix[k]))
        return fail(nullptr, PHI_E_INVALID, "non-finite value in the Hamiltonian or the initial density matrix");
    phi::TruncatedProblem t;
    std::string err;
    if (phi::truncate_problem(d, &t, &err) != 0) return fail(nullptr, PHI_E_INVALID, err);
    const int rc = phi_gpu_create(&t.desc, out);
    if (rc != PHI_OK) return rc;
    phi_ctx *ctx = *out;
    ctx->hilbert_full = F;
    ctx->trunc_basis = std::move(t.basis);
    if (anneal_t) {
      // The device re-diagonalises H(t) at every update: full H_X, H_Z, the
      // current basis and the rotation of the last update live on the device.
      static_assert(phi::kTruncatedAnnealingMaxFull == phi::kAnnealMaxFull, "eigensolver size");
      const int k = ctx->desc.num_states;
      const size_t fb = (size_t)F * F * sizeof(double);
      std::vector<double> hx(t.hx_full), hz(t.hz_full);
      cudaError_t e = cudaSuccess;
      if (ctx->ta_hx.alloc(fb) != cudaSuccess || ctx->ta_hz.alloc(fb) != cudaSuccess ||
          ctx->ta_V.alloc((size_t)F * k * sizeof(double)) != cudaSuccess ||
          ctx->ta_R.alloc((size_t)k * k * sizeof(double)) != cudaSuccess ||
          ctx->ta_rotate.alloc(sizeof(int)) != cudaSuccess)
        e = cudaErrorMemoryAllocation;
      if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->ta_hx.ptr, hx.data(), fb, cudaMemcpyHostToDevice, ctx->stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->ta_hz.ptr, hz.data(), fb, cudaMemcpyHostToDevice, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // hx, hz are locals
      if (e == cudaSuccess) {
        ctx->ta_F = F;
        ctx->ta_bath0 = ctx->coupling;  // the bath operators truncated into the initial basis
        e = ctx->reset_annealing();
      }
      if (e != cudaSuccess) {
        phi_gpu_destroy(ctx);
        *out = nullptr;
        return fail(nullptr, e == cudaErrorMemoryAllocation ? PHI_E_OOM : PHI_E_CUDA,
                    std::string("truncated annealing setup: ") + cudaGetErrorString(e));
      }
    }
    return PHI_OK;
  }
  const bool annealing = d.annealing_h_x != nullptr;
  if ((!d.hamiltonian && !annealing) || !d.initial_density_matrix || !d.gamma || !d.lambda)
    return fail(nullptr, PHI_E_INVALID, "hamiltonian, initial_density_matrix, gamma and lambda are required");
  if (annealing) {
    if (!d.annealing_h_z || !d.transverse_field || !d.longitudinal_field)
      return fail(nullptr, PHI_E_INVALID, "an annealing Hamiltonian needs H_X, H_Z and both field arrays");
    if (d.transverse_field_size < 2 || d.longitudinal_field_size < 2)
      return fail(nullptr, PHI_E_INVALID, "annealing fields need at least 2 samples each");
    if (!(d.integration_time > 0) || !std::isfinite(d.integration_time) || !(d.minimum_field_change >= 0) ||
        !std::isfinite(d.minimum_field_change))
      return fail(nullptr, PHI_E_INVALID, "annealing needs integration_time > 0 and minimum_field_change >= 0");
    for (int k = 0; k < 2 * N * N; ++k)
      if (!std::isfinite(d.annealing_h_x[k]) || !std::isfinite(d.annealing_h_z[k]))
        return fail(nullptr, PHI_E_INVALID, "non-finite value in H_X or H_Z");
    for (int k = 0; k < d.transverse_field_size; ++k)
      if (!std::isfinite(d.transverse_field[k])) return fail(nullptr, PHI_E_INVALID, "non-finite transverse field");
    for (int k = 0; k < d.longitudinal_field_size; ++k)
      if (!std::isfinite(d.longitudinal_field[k]))
        return fail(nullptr, PHI_E_INVALID, "non-finite longitudinal field");
  }
  if (!(d.hbar > 0) || !(d.boltzmann_constant > 0) || !(d.temperature > 0))
    return fail(nullptr, PHI_E_INVALID, "hbar, boltzmann_constant and temperature must be positive");
  if (d.bath_kind != PHI_BATH_INDEPENDENT && !d.coupling)
    return fail(nullptr, PHI_E_INVALID, "diagonal and full baths need coupling operators");
  for (int k = 0; k < 2 * N * N; ++k)
    if ((!annealing && !std::isfinite(d.hamiltonian[k])) || !std::isfinite(d.initial_density_matrix[k]))
      return fail(nullptr, PHI_E_INVALID, "non-finite value in the Hamiltonian or initial density matrix");
  if (d.truncation_level > 1 && (d.normalized || d.bath_kind == PHI_BATH_DIAGONAL)) {
    // The normalised prefactors divide by sqrt(n |c_t|) (hierarchy_integrator.cc
    // :1430-1436); c_t vanishes when gamma <= 0 or lambda == 0 (:441-469).
    for (int b = 0; b < d.num_baths; ++b)
      if (!(d.gamma[b] > 0) || d.lambda[b] == 0 || !std::isfinite(d.gamma[b]) || !std::isfinite(d.lambda[b]))
        if (d.normalized && d.bath_kind != PHI_BATH_DIAGONAL)
          return fail(nullptr, PHI_E_INVALID,
                      "bath " + std::to_string(b) + ": gamma must be > 0 and lambda non-zero for a "
                      "normalised hierarchy");
  }
  if (!is_hermitian(d.initial_density_matrix, N, nullptr))
    return fail(nullptr, PHI_E_INVALID,
                "initial density matrix is not Hermitian (PHI's hierarchy keeps every ADO Hermitian)");
  if (!(d.filter_tolerance >= 0) || !std::isfinite(d.filter_tolerance))
    return fail(nullptr, PHI_E_INVALID, "filter_tolerance must be finite and >= 0");
  if (d.time_local != 0 && d.time_local != 1)
    return fail(nullptr, PHI_E_INVALID, "time_local must be 0 or 1");
  if (d.time_local && d.bath_kind == PHI_BATH_INDEPENDENT) {
    // PHI's independent-bath matrices put c at (b, b) whatever site bath b
    // couples to (hierarchy.cc:298-300), while its DoTimelocal works on site
    // b's row and column: only the identity site map is consistent.
    bool identity = d.num_baths == N;
    if (identity && d.bath_sites)
      for (int b = 0; b < d.num_baths; ++b) identity = identity && d.bath_sites[b] == b;
    if (!identity)
      return fail(nullptr, PHI_E_INVALID,
                  "time-local truncation with independent baths needs PHI's identity site map "
                  "(bath j on |j><j|)");
  }

  std::unique_ptr<phi_ctx> ctx(new phi_ctx());
  ctx->desc = d;
  // An annealing Hamiltonian starts at zero (PHI copies no static H).
  if (annealing)
    ctx->hamiltonian.assign((size_t)2 * N * N, 0.0);
  else
    ctx->hamiltonian.assign(d.hamiltonian, d.hamiltonian + 2 * N * N);
  ctx->annealing = annealing;
  ctx->rho_init.assign(d.initial_density_matrix, d.initial_density_matrix + 2 * N * N);
  ctx->gamma.assign(d.gamma, d.gamma + d.num_baths);
  ctx->lambda.assign(d.lambda, d.lambda + d.num_baths);
  if (d.bath_kind == PHI_BATH_DIAGONAL) ctx->coupling.assign(d.coupling, d.coupling + (size_t)d.num_baths * N);
  if (d.bath_kind == PHI_BATH_FULL) {
    ctx->coupling.assign(d.coupling, d.coupling + (size_t)d.num_baths * N * N);
    for (int b = 0; b < d.num_baths; ++b)
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c)
          if (ctx->coupling[(size_t)b * N * N + r + c * N] != ctx->coupling[(size_t)b * N * N + c + r * N])
            return fail(nullptr, PHI_E_INVALID, "full bath coupling operators must be symmetric");
  }
  ctx->bath_sites.resize(d.num_baths);
  if (d.bath_kind == PHI_BATH_INDEPENDENT) {
    if (d.bath_sites) {
      for (int b = 0; b < d.num_baths; ++b) {
        if (d.bath_sites[b] < 0 || d.bath_sites[b] >= N)
          return fail(nullptr, PHI_E_INVALID, "bath_sites entries must be in [0, num_states)");
        ctx->bath_sites[b] = d.bath_sites[b];
      }
    } else {
      if (d.num_baths != N && d.truncation_level > 1)
        return fail(nullptr, PHI_E_INVALID,
                    "independent baths without bath_sites need num_baths == num_states "
                    "(PHI couples bath j to |j><j|)");
      for (int b = 0; b < d.num_baths; ++b) ctx->bath_sites[b] = b < N ? b : 0;
    }
  }
  ctx->desc.hamiltonian = nullptr;
  ctx->desc.initial_density_matrix = nullptr;
  ctx->desc.gamma = ctx->desc.lambda = ctx->desc.coupling = nullptr;
  ctx->desc.bath_sites = nullptr;
  ctx->desc.annealing_h_x = ctx->desc.annealing_h_z = nullptr;
  ctx->desc.transverse_field = ctx->desc.longitudinal_field = nullptr;

  cudaError_t e = cudaSetDevice(d.device);
  if (e != cudaSuccess) return fail(nullptr, PHI_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(nullptr, PHI_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, d.device);

  ctx->hier.budget = d.max_nodes;
  std::string err;
  int rc = phi::build_hierarchy_device((int)T, d.truncation_level - 1, &ctx->hier, &err, ctx->stream);
  if (rc != 0) {
    const int code = rc == 2 ? PHI_E_OOM : rc == 3 ? PHI_E_BUDGET : rc == 7 ? PHI_E_CUDA : PHI_E_INVALID;
    return fail(nullptr, code, err);
  }
  rc = phi::setup_constants(ctx.get());
  if (rc != PHI_OK) {
    g_create_error = ctx->error;
    return rc;
  }
  if (d.precision == PHI_PREC_MIXED && !phi::tile_kernel_available(ctx->c))
    return fail(nullptr, PHI_E_INVALID,
                "mixed precision is built for independent baths on PHI's identity site map, K+1 <= 3 and "
                "N in {2..8, 10, 12, 16, 24}");
  ctx->grid = phi::stage_grid(ctx->c, ctx->num_sms);
  const size_t state_bytes = (size_t)ctx->hier.M * N * N * sizeof(double2);
  e = ctx->y.alloc(state_bytes);
  if (e != cudaSuccess) return fail(nullptr, PHI_E_OOM, "state allocation failed: " + std::to_string(state_bytes) + " bytes");
  // InitializeDensityMatrix (hierarchy_integrator.cc:1070-1096): rho(0) in
  // node 0, scaled by prod sqrt(|c|^n n!) = 1 at tier 0; zero elsewhere.
  e = cudaMemsetAsync(ctx->y.ptr, 0, state_bytes, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->y.ptr, ctx->rho_init.data(), (size_t)N * N * sizeof(double2),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && annealing) {
    const size_t hb = (size_t)N * N * sizeof(double2);
    const int nx = d.transverse_field_size, nz = d.longitudinal_field_size;
    std::vector<double> coef((size_t)5 * (nx + nz));
    phi::anneal_spline_host(d.transverse_field, nx, coef.data());
    phi::anneal_spline_host(d.longitudinal_field, nz, coef.data() + 5 * nx);
    if (ctx->an_hx.alloc(hb) != cudaSuccess || ctx->an_hz.alloc(hb) != cudaSuccess ||
        ctx->an_spline.alloc(coef.size() * sizeof(double)) != cudaSuccess ||
        ctx->an_state.alloc(sizeof(phi::AnnealState)) != cudaSuccess)
      return fail(nullptr, PHI_E_OOM, "annealing buffer allocation failed");
    ctx->an_nx = nx;
    ctx->an_nz = nz;
    e = cudaMemcpyAsync(ctx->an_hx.ptr, d.annealing_h_x, hb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->an_hz.ptr, d.annealing_h_z, hb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ctx->an_spline.ptr, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // coef is a local buffer
    // The real-H fast path of the tiled kernel holds when H_X and H_Z are real.
    ctx->c.h_real = 1;
    for (int k = 0; k < N * N; ++k)
      if (d.annealing_h_x[2 * k + 1] != 0.0 || d.annealing_h_z[2 * k + 1] != 0.0) ctx->c.h_real = 0;
    if (e == cudaSuccess) e = ctx->reset_annealing();
  }
  if (e == cudaSuccess && ctx->c.time_local) {
    const size_t nq = (size_t)d.num_baths * N * N * sizeof(double2);
    if (ctx->tl_qk.alloc(nq * d.num_matsubara_terms) != cudaSuccess ||
        ctx->tl_qk_st.alloc(nq * d.num_matsubara_terms) != cudaSuccess || ctx->tl_q.alloc(nq) != cudaSuccess ||
        ctx->tl_q_st.alloc(nq) != cudaSuccess)
      return fail(nullptr, PHI_E_OOM, "time-local matrix allocation failed");
    ctx->c.tl_q = ctx->tl_q.as<double2>();
    e = ctx->reset_time_local();
  }
  if (e == cudaSuccess && ctx->c.filtered) {
    if (ctx->active[0].alloc((size_t)ctx->hier.M) != cudaSuccess || ctx->active[1].alloc((size_t)ctx->hier.M) != cudaSuccess)
      return fail(nullptr, PHI_E_OOM, "filter flag allocation failed");
    e = ctx->reset_filter();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(nullptr, PHI_E_CUDA, std::string("initial state: ") + cudaGetErrorString(e));
  ctx->time = 0.0;
  rc = tune_tile_schedule(ctx.get());
  if (rc != PHI_OK) {
    g_create_error = ctx->error;
    return rc;
  }
  *out = ctx.release();
  return PHI_OK;
}

extern "C" int phi_gpu_destroy(phi_ctx *ctx) {
  if (!ctx) return PHI_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->release_graphs();
  cudaStream_t s = ctx->stream;
  delete ctx;
  if (s) cudaStreamDestroy(s);
  return PHI_OK;
}

extern "C" int phi_gpu_dims(const phi_ctx *ctx, int64_t *num_nodes, int32_t *num_terms,
                            int32_t *num_states) {
  if (!ctx) return PHI_E_INVALID;
  if (num_nodes) *num_nodes = ctx->hier.M;
  if (num_terms) *num_terms = ctx->hier.T;
  if (num_states) *num_states = ctx->desc.num_states;
  return PHI_OK;
}

extern "C" int phi_gpu_num_baths(const phi_ctx *ctx, int32_t *num_baths) {
  if (!ctx || !num_baths) return PHI_E_INVALID;
  *num_baths = ctx->desc.num_baths;
  return PHI_OK;
}

extern "C" int phi_gpu_get_node_table(const phi_ctx *cctx, int32_t *multi_index, int32_t *next,
                                      int32_t *prev) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx) return PHI_E_INVALID;
  const size_t n = (size_t)ctx->hier.M * ctx->hier.T;
  if (multi_index) {
    std::vector<uint8_t> tmp(n);
    PHI_CUDA(ctx, cudaMemcpyAsync(tmp.data(), ctx->hier.mi.ptr, n, cudaMemcpyDeviceToHost, ctx->stream));
    PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < n; ++i) multi_index[i] = tmp[i];
  }
  if (next) PHI_CUDA(ctx, cudaMemcpyAsync(next, ctx->hier.next.ptr, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (prev) PHI_CUDA(ctx, cudaMemcpyAsync(prev, ctx->hier.prev.ptr, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

cudaError_t phi_ctx::reset_filter() {
  if (!c.filtered) return cudaSuccess;
  return cudaMemsetAsync(active[0].ptr, 1, (size_t)hier.M, stream);
}

cudaError_t phi_ctx::reset_time_local() {
  if (!c.time_local) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(tl_qk.ptr, 0, tl_qk.bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(tl_qk_st.ptr, 0, tl_qk_st.bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(tl_q.ptr, 0, tl_q.bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(tl_q_st.ptr, 0, tl_q_st.bytes, stream);
  return e;
}

cudaError_t phi_ctx::enqueue_time_local(int op, int stage, double h, cudaStream_t s) {
  if (!c.time_local) return cudaSuccess;
  if (op == phi::kTlAdvance && !(h >= 1e-9)) return cudaSuccess;  // skipped as PHI does
  phi::TlLaunch L;
  L.c = c;
  L.op = op;
  L.stage = stage;
  L.h = h;
  L.ctl = ctl.as<phi::Rkf45Ctl>();
  L.qk = tl_qk.as<double2>();
  L.qk_st = tl_qk_st.as<double2>();
  L.q = tl_q.as<double2>();
  L.q_st = tl_q_st.as<double2>();
  return phi::launch_tl(L, s);
}

cudaError_t phi_ctx::reset_annealing() {
  if (!annealing) return cudaSuccess;
  const phi::AnnealState st{DBL_MAX, DBL_MAX, 0, 0};  // numeric_limits<Float>::max() (:518-523)
  cudaError_t e = cudaMemcpyAsync(an_state.ptr, &st, sizeof(st), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(cbuf.H.ptr, 0, cbuf.H.bytes, stream);
  if (ta_F > 0) {
    // Truncated: the initial basis and the bath operators truncated into it.
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ta_V.ptr, trunc_basis.data(), trunc_basis.size() * sizeof(double),
                          cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && !ta_bath0.empty())
      e = cudaMemcpyAsync(cbuf.bath_V.ptr, ta_bath0.data(), ta_bath0.size() * sizeof(double),
                          cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ta_rotate.ptr, 0, sizeof(int), stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // st is a local
  return e;
}

cudaError_t phi_ctx::enqueue_anneal(int op, int which, double dt, cudaStream_t s) {
  if (!annealing) return cudaSuccess;
  phi::AnnealLaunch L;
  L.op = op;
  L.which = which;
  L.dt = dt;
  L.rk4 = ctl.as<phi::Rk4Ctl>();
  L.ctl = ctl.as<phi::Rkf45Ctl>();
  const double *sp = an_spline.as<double>();
  L.sx = phi::AnnealSpline{sp, sp + an_nx, sp + 2 * an_nx, sp + 3 * an_nx, sp + 4 * an_nx, an_nx};
  const double *sz = sp + 5 * an_nx;
  L.sz = phi::AnnealSpline{sz, sz + an_nz, sz + 2 * an_nz, sz + 3 * an_nz, sz + 4 * an_nz, an_nz};
  L.st = an_state.as<phi::AnnealState>();
  L.hx = an_hx.as<double2>();
  L.hz = an_hz.as<double2>();
  L.H = cbuf.H.as<double2>();
  L.E = desc.num_states * desc.num_states;
  L.integration_time = desc.integration_time;
  L.min_field_change = desc.minimum_field_change;
  if (ta_F > 0) {
    L.tr.F = ta_F;
    L.tr.k = desc.num_states;
    L.tr.hx = ta_hx.as<double>();
    L.tr.hz = ta_hz.as<double>();
    L.tr.V = ta_V.as<double>();
    L.tr.R = ta_R.as<double>();
    L.tr.rotate = static_cast<int *>(ta_rotate.ptr);
    // PHI rotates the bath operators only when it reads them: more than one
    // tier or time-local truncation (hierarchy_integrator.cc:1661-1668).
    const bool bath = desc.bath_kind == PHI_BATH_FULL && (desc.truncation_level > 1 || desc.time_local);
    L.tr.bath = bath ? cbuf.bath_V.as<double>() : nullptr;
    L.tr.nb = bath ? desc.num_baths : 0;
  }
  return phi::launch_anneal(L, s);
}

cudaError_t phi_ctx::enqueue_anneal_rotate(std::initializer_list<void *> bufs, bool rkf45_y, cudaStream_t s) {
  if (ta_F == 0) return cudaSuccess;
  phi::AnnealRotate r;
  r.rotate = static_cast<const int *>(ta_rotate.ptr);
  r.R = ta_R.as<double>();
  r.k = desc.num_states;
  r.M = hier.M;
  for (void *b : bufs) {
    if (r.nbuf == phi::kAnnealMaxRotate) return cudaErrorInvalidValue;
    r.buf[r.nbuf++] = static_cast<double2 *>(b);
  }
  if (rkf45_y) {
    r.ybuf[0] = y.as<double2>();
    r.ybuf[1] = y_alt.as<double2>();
    r.ctl = ctl.as<phi::Rkf45Ctl>();
  }
  return phi::launch_anneal_rotate(r, num_sms, s);
}

extern "C" int phi_gpu_get_hamiltonian(const phi_ctx *cctx, double *h) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !h) return PHI_E_INVALID;
  PHI_CUDA(ctx, cudaMemcpyAsync(h, ctx->cbuf.H.ptr, (size_t)ctx->desc.num_states * ctx->desc.num_states * sizeof(double2),
                                cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

extern "C" int phi_gpu_get_time_local(const phi_ctx *cctx, double *q) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !q) return PHI_E_INVALID;
  const size_t n = (size_t)ctx->desc.num_baths * ctx->desc.num_states * ctx->desc.num_states;
  if (!ctx->c.time_local) {
    std::memset(q, 0, n * sizeof(double2));
    return PHI_OK;
  }
  PHI_CUDA(ctx, cudaMemcpyAsync(q, ctx->tl_q.ptr, n * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

void phi_ctx::bind_filter(phi::StageLaunch &L, int par) const {
  if (!c.filtered) return;
  L.act[0] = static_cast<uint8_t *>(active[0].ptr);
  L.act[1] = static_cast<uint8_t *>(active[1].ptr);
  L.act_par = par;
}

extern "C" int phi_gpu_get_active(const phi_ctx *cctx, uint8_t *flags) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !flags) return PHI_E_INVALID;
  if (!ctx->c.filtered) {
    std::memset(flags, 1, (size_t)ctx->hier.M);
    return PHI_OK;
  }
  PHI_CUDA(ctx, cudaMemcpyAsync(flags, ctx->active[0].ptr, (size_t)ctx->hier.M, cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

extern "C" int phi_gpu_set_state(phi_ctx *ctx, const double *state) {
  if (!ctx || !state) return PHI_E_INVALID;
  PHI_CUDA(ctx, cudaMemcpyAsync(ctx->y.ptr, state, ctx->state_bytes(), cudaMemcpyHostToDevice, ctx->stream));
  PHI_CUDA(ctx, ctx->reset_filter());
  PHI_CUDA(ctx, ctx->reset_time_local());
  PHI_CUDA(ctx, ctx->reset_annealing());
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

extern "C" int phi_gpu_get_state(const phi_ctx *cctx, double *state) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !state) return PHI_E_INVALID;
  PHI_CUDA(ctx, cudaMemcpyAsync(state, ctx->y.ptr, ctx->state_bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

extern "C" int phi_gpu_get_tile_schedule(const phi_ctx *ctx, phi_tile_schedule *out) {
  if (!ctx || !out) return PHI_E_INVALID;
  const bool tiled = phi::tile_kernel_available(ctx->c);
  out->threads = tiled ? phi::tile_block_threads(ctx->c, ctx->mixed(), ctx->c.tile_variant) : 0;
  out->ctas_per_sm = ctx->c.tile_cps;
  out->ms_per_apply = ctx->tile_sched.ms;
  out->ms_per_apply_default = ctx->tile_sched.ms_default;
  return PHI_OK;
}

extern "C" int phi_gpu_set_tile_schedule(phi_ctx *ctx, int32_t threads, int32_t ctas_per_sm) {
  if (!ctx) return PHI_E_INVALID;
  if (!phi::tile_kernel_available(ctx->c)) {
    ctx->error = "set_tile_schedule: this problem does not run on the tiled kernel";
    return PHI_E_INVALID;
  }
  int variant = -1;
  for (int v = 0; v < 2; ++v)
    if (phi::tile_block_threads(ctx->c, ctx->mixed(), v) == threads) variant = v;
  if (variant < 0 || ctas_per_sm < 0) {
    ctx->error = "set_tile_schedule: threads must be " + std::to_string(phi::tile_block_threads(ctx->c, ctx->mixed(), 0)) +
                 " or " + std::to_string(phi::tile_block_threads(ctx->c, ctx->mixed(), 1)) +
                 " and ctas_per_sm >= 0";
    return PHI_E_INVALID;
  }
  ctx->c.tile_variant = variant;
  ctx->c.tile_cps = ctas_per_sm;
  ctx->release_graphs();  // captured launches carry the old schedule
  return PHI_OK;
}

extern "C" int phi_gpu_hilbert_space_size(const phi_ctx *ctx, int32_t *size) {
  if (!ctx || !size) return PHI_E_INVALID;
  *size = ctx->hilbert_full > 0 ? ctx->hilbert_full : ctx->desc.num_states;
  return PHI_OK;
}

extern "C" int phi_gpu_get_rho0_full(const phi_ctx *cctx, double *rho0) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !rho0) return PHI_E_INVALID;
  const int k = ctx->desc.num_states;
  if (ctx->hilbert_full <= k) return phi_gpu_get_rho0(ctx, rho0);
  std::vector<double> rk(2 * (size_t)k * k);
  const int rc = phi_gpu_get_rho0(ctx, rk.data());
  if (rc != PHI_OK) return rc;
  std::vector<double> basis(ctx->trunc_basis);
  if (ctx->ta_F > 0) {  // an annealing run's basis follows H(t)
    PHI_CUDA(ctx, cudaMemcpyAsync(basis.data(), ctx->ta_V.ptr, basis.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  phi::untruncate(ctx->hilbert_full, k, basis.data(), rk.data(), rho0);
  return PHI_OK;
}

extern "C" int phi_gpu_get_rho0(const phi_ctx *cctx, double *rho0) {
  phi_ctx *ctx = const_cast<phi_ctx *>(cctx);
  if (!ctx || !rho0) return PHI_E_INVALID;
  const size_t b = (size_t)ctx->desc.num_states * ctx->desc.num_states * sizeof(double2);
  PHI_CUDA(ctx, cudaMemcpyAsync(rho0, ctx->y.ptr, b, cudaMemcpyDeviceToHost, ctx->stream));
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHI_OK;
}

int phi_ctx::check_device_flag() { return check_device_flag_on(stream); }

int phi_ctx::check_device_flag_on(cudaStream_t s) {
  int flag = 0;
  cudaError_t e = cudaMemcpyAsync(&flag, cbuf.err_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(this, e, "device flag read");
  if (flag) {
    cudaMemsetAsync(cbuf.err_flag.ptr, 0, sizeof(int), s);
    error = "a device wait on a bulk copy gave up (bounded mbarrier wait)";
    return PHI_E_TIMEOUT;
  }
  return PHI_OK;
}

extern "C" int phi_gpu_check_device_flag(phi_ctx *ctx, void *stream) {
  if (!ctx) return PHI_E_INVALID;
  return ctx->check_device_flag_on(stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

extern "C" int phi_gpu_apply_device(phi_ctx *ctx, const void *d_in, void *d_out, void *stream) {
  if (!ctx || !d_in || !d_out) return PHI_E_INVALID;
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15u) {
    ctx->error = "apply_device: device buffers must be 16-byte aligned";
    return PHI_E_INVALID;
  }
  phi::StageLaunch L;
  L.c = ctx->c;
  L.mode = phi::kModeApply;
  L.grid = ctx->grid;
  L.x = static_cast<const double2 *>(d_in);
  L.out = static_cast<double2 *>(d_out);
  L.xv = d_in;
  L.outv = d_out;
  L.mixed = ctx->mixed();
  ctx->bind_filter(L, 0);
  PHI_CUDA(ctx, phi::launch_stage(L, static_cast<cudaStream_t>(stream)));
  return PHI_OK;
}

extern "C" int phi_gpu_apply(phi_ctx *ctx, const double *in, double *out) {
  if (!ctx || !in || !out) return PHI_E_INVALID;
  int rc = ctx->ensure_work(ctx->mixed() ? 2 : 1);
  if (rc != PHI_OK) return rc;
  const size_t b = ctx->state_bytes();
  const int E = ctx->desc.num_states * ctx->desc.num_states;
  if (ctx->mixed()) {  // complex128 host data through the complex64 stage buffers
    PHI_CUDA(ctx, cudaMemcpyAsync(ctx->acc.ptr, in, b, cudaMemcpyHostToDevice, ctx->stream));
    PHI_CUDA(ctx, phi::launch_to_c64(ctx->acc.as<double2>(), ctx->xa.as<float2>(), ctx->hier.M, E,
                                     ctx->work_stride(), ctx->stream));
  } else {
    PHI_CUDA(ctx, cudaMemcpyAsync(ctx->xa.ptr, in, b, cudaMemcpyHostToDevice, ctx->stream));
  }
  rc = phi_gpu_apply_device(ctx, ctx->xa.ptr, ctx->xb.ptr, ctx->stream);
  if (rc != PHI_OK) return rc;
  if (ctx->mixed()) {
    PHI_CUDA(ctx, phi::launch_to_c128(ctx->xb.as<float2>(), ctx->acc.as<double2>(), ctx->hier.M, E,
                                      ctx->work_stride(), ctx->stream));
    PHI_CUDA(ctx, cudaMemcpyAsync(out, ctx->acc.ptr, b, cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    PHI_CUDA(ctx, cudaMemcpyAsync(out, ctx->xb.ptr, b, cudaMemcpyDeviceToHost, ctx->stream));
  }
  PHI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ctx->check_device_flag();
}

extern "C" int phi_gpu_get_time(const phi_ctx *ctx, double *time) {
  if (!ctx || !time) return PHI_E_INVALID;
  *time = ctx->time;
  return PHI_OK;
}

extern "C" int phi_gpu_reset(phi_ctx *ctx, double time) {
  if (!ctx) return PHI_E_INVALID;
  const int N = ctx->desc.num_states;
  PHI_CUDA(ctx, cudaMemsetAsync(ctx->y.ptr, 0, ctx->state_bytes(), ctx->stream));
  PHI_CUDA(ctx, cudaMemcpyAsync(ctx->y.ptr, ctx->rho_init.data(), (size_t)N * N * sizeof(double2),
                                cudaMemcpyHostToDevice, ctx->stream));
  PHI_CUDA(ctx, ctx->reset_filter());
  PHI_CUDA(ctx, ctx->reset_time_local());
  PHI_CUDA(ctx, ctx->reset_annealing());
  ctx->time = time;
  ctx->rkf45_started = false;
  return PHI_OK;
}

extern "C" int phi_gpu_debug_set_wait_limit(phi_ctx *ctx, int64_t polls) {
  if (!ctx) return PHI_E_INVALID;
  ctx->c.first_wait_polls = polls;
  ctx->release_graphs();  // captured launches carry the old constants
  return PHI_OK;
}

extern "C" int phi_gpu_set_time(phi_ctx *ctx, double time) {
  if (!ctx) return PHI_E_INVALID;
  ctx->time = time;
  return PHI_OK;
}

extern "C" int phi_gpu_last_error(const phi_ctx *ctx, char *buf, size_t len) {
  if (!buf || len == 0) return PHI_E_INVALID;
  const std::string &s = ctx ? ctx->error : g_create_error;
  std::snprintf(buf, len, "%s", s.c_str());
  return PHI_OK;
}
