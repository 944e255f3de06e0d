// phi_restart.cpp -- restart files: PHI's text layout (RestartHelper,
// restart_helper.cc:20-84) and a binary fast path, on host buffers and on a
// context's state.
//
// Text layout: the time, the step size, then one line per hierarchy node with
// its N*N elements in storage (column-major) order, each written as
// std::complex prints it, "(re,im)".  PHI writes 6 significant digits; this
// writer uses 17 so a state round-trips exactly.  The reader accepts both, as
// well as bare "re im" pairs.
//
// Binary layout: 8-byte magic "PHIB200S", uint32 version (1), uint32 N,
// int64 M, double time, double step size, then 2*M*N*N doubles.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/phi_b200.h"
#include "phi_context.h"

namespace {

thread_local std::string g_restart_error;  // per calling thread, as the create error is

int fail(int code, const std::string &msg) {
  g_restart_error = msg;
  return code;
}

// Next number in the text, skipping whitespace, '(', ')' and ','.
bool next_number(const char *&s, double *v) {
  while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r' || *s == '(' || *s == ')' || *s == ',') ++s;
  if (!*s) return false;
  char *end = nullptr;
  errno = 0;
  const double x = std::strtod(s, &end);
  if (end == s) return false;
  s = end;
  *v = x;
  return true;
}

bool read_all(const char *path, std::string *out) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) out->append(buf, n);
  std::fclose(f);
  return true;
}

const char kMagic[8] = {'P', 'H', 'I', 'B', '2', '0', '0', 'S'};

}  // namespace

extern "C" int phi_restart_read_file_ex(const char *path, int32_t num_states, int64_t num_nodes, double *state,
                                        double *time, double *timestep, double *matrices, int64_t num_matrices) {
  if (!path || num_states <= 0 || num_nodes <= 0 || !state || num_matrices < 0 || (num_matrices > 0 && !matrices))
    return fail(PHI_E_INVALID, "restart: bad arguments");
  std::string text;
  if (!read_all(path, &text)) return fail(PHI_E_INVALID, std::string("restart: cannot open ") + path);
  const char *s = text.c_str();
  double t = 0, dt = 0;
  if (!next_number(s, &t) || !next_number(s, &dt)) return fail(PHI_E_INVALID, "restart: missing time / step size");
  const long long count = 2ll * num_nodes * num_states * num_states;
  for (long long k = 0; k < count; ++k)
    if (!next_number(s, &state[k]))
      return fail(PHI_E_INVALID, "restart: file ends after " + std::to_string(k / 2) + " of " +
                                     std::to_string(count / 2) + " elements");
  // Time-local truncation matrices follow the nodes in a time-local run's file.
  const long long extra_count = 2ll * num_matrices * num_states * num_states;
  for (long long k = 0; k < extra_count; ++k)
    if (!next_number(s, &matrices[k]))
      return fail(PHI_E_INVALID, "restart: file ends inside the time-local matrices (" + std::to_string(k / 2) +
                                     " of " + std::to_string(extra_count / 2) + " elements)");
  double extra;
  if (next_number(s, &extra))
    return fail(PHI_E_INVALID, "restart: more values than " + std::to_string(num_nodes) + " nodes of " +
                                   std::to_string(num_states) + "x" + std::to_string(num_states) + " and " +
                                   std::to_string(num_matrices) + " time-local matrices");
  if (time) *time = t;
  if (timestep) *timestep = dt;
  return PHI_OK;
}

extern "C" int phi_restart_read_file(const char *path, int32_t num_states, int64_t num_nodes, double *state,
                                     double *time, double *timestep) {
  return phi_restart_read_file_ex(path, num_states, num_nodes, state, time, timestep, nullptr, 0);
}

extern "C" int phi_restart_write_file_ex(const char *path, int32_t num_states, int64_t num_nodes,
                                         const double *state, double time, double timestep,
                                         const double *matrices, int64_t num_matrices) {
  if (!path || num_states <= 0 || num_nodes <= 0 || !state || num_matrices < 0 || (num_matrices > 0 && !matrices))
    return fail(PHI_E_INVALID, "restart: bad arguments");
  FILE *f = std::fopen(path, "w");
  if (!f) return fail(PHI_E_INVALID, std::string("restart: cannot create ") + path);
  std::fprintf(f, "%.17g\n%.17g\n", time, timestep);
  const long long E = (long long)num_states * num_states;
  auto write_rows = [&](const double *base, long long rows) {
    for (long long n = 0; n < rows; ++n) {
      const double *z = base + 2 * n * E;
      for (long long e = 0; e < E; ++e)
        std::fprintf(f, e ? " (%.17g,%.17g)" : "(%.17g,%.17g)", z[2 * e], z[2 * e + 1]);
      std::fputc('\n', f);
    }
  };
  write_rows(state, num_nodes);
  if (num_matrices > 0) write_rows(matrices, num_matrices);
  const bool ok = std::fclose(f) == 0;
  return ok ? PHI_OK : fail(PHI_E_INVALID, std::string("restart: write failed: ") + path);
}

extern "C" int phi_restart_write_file(const char *path, int32_t num_states, int64_t num_nodes, const double *state,
                                      double time, double timestep) {
  return phi_restart_write_file_ex(path, num_states, num_nodes, state, time, timestep, nullptr, 0);
}

extern "C" int phi_restart_last_error(char *buf, size_t len) {
  if (!buf || !len) return PHI_E_INVALID;
  std::snprintf(buf, len, "%s", g_restart_error.c_str());
  return PHI_OK;
}

// ---- on a context ------------------------------------------------------------

namespace {

// Number of time-local matrices a context's files carry (nb * (K + 1)), 0 when off.
int64_t tl_matrix_count(const phi_ctx *ctx) {
  return ctx->c.time_local ? (int64_t)ctx->desc.num_baths * ctx->desc.num_matsubara_terms : 0;
}

// The stored Q_{m,k} (time_local_truncation_store_th_, what PHI's files hold).
int get_tl_store(phi_ctx *ctx, std::vector<double> *out) {
  const size_t bytes = ctx->tl_qk_st.bytes;
  out->resize(bytes / sizeof(double));
  cudaError_t e = cudaMemcpyAsync(out->data(), ctx->tl_qk_st.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    ctx->error = std::string("restart: ") + cudaGetErrorString(e);
    return fail(PHI_E_CUDA, ctx->error);
  }
  return PHI_OK;
}

// Loads read Q_{m,k} as PHI's Initialize does (hierarchy_integrator.cc
// :1046-1068): into the stored copies, their per-bath sums (SumMatrices:
// copy of k = 0, then += k) into the stored sums, then restored as current.
int put_tl_store(phi_ctx *ctx, const std::vector<double> &qk) {
  const int N = ctx->desc.num_states, K1 = ctx->desc.num_matsubara_terms, nb = ctx->desc.num_baths;
  const size_t E2 = (size_t)2 * N * N;
  std::vector<double> q((size_t)nb * E2);
  for (int m = 0; m < nb; ++m)
    for (int k = 0; k < K1; ++k)
      for (size_t i = 0; i < E2; ++i) {
        const double v = qk[((size_t)m * K1 + k) * E2 + i];
        q[m * E2 + i] = k == 0 ? v : q[m * E2 + i] + v;
      }
  cudaError_t e = cudaMemcpyAsync(ctx->tl_qk_st.ptr, qk.data(), ctx->tl_qk_st.bytes, cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->tl_qk.ptr, qk.data(), ctx->tl_qk.bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->tl_q_st.ptr, q.data(), ctx->tl_q_st.bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->tl_q.ptr, q.data(), ctx->tl_q.bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    ctx->error = std::string("restart: ") + cudaGetErrorString(e);
    return fail(PHI_E_CUDA, ctx->error);
  }
  return PHI_OK;
}

// A truncated annealing run's ADOs are expressed in the basis of its last
// Hamiltonian update, which a state file does not carry.
int refuse_truncated_annealing(phi_ctx *ctx) {
  ctx->error = "restart and state files of a Hilbert-space truncated annealing run are not built";
  return fail(PHI_E_INVALID, ctx->error);
}

}  // namespace

extern "C" int phi_gpu_write_restart(phi_ctx *ctx, const char *path, double timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->ta_F > 0) return refuse_truncated_annealing(ctx);
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  std::vector<double> st((size_t)2 * M * N * N), tl;
  int rc = phi_gpu_get_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  const int64_t ntl = tl_matrix_count(ctx);
  if (ntl > 0 && (rc = get_tl_store(ctx, &tl)) != PHI_OK) return rc;
  double t = 0;
  phi_gpu_get_time(ctx, &t);
  return phi_restart_write_file_ex(path, N, M, st.data(), t, timestep, tl.data(), ntl);
}

extern "C" int phi_gpu_read_restart(phi_ctx *ctx, const char *path, double *timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->ta_F > 0) return refuse_truncated_annealing(ctx);
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  const int64_t ntl = tl_matrix_count(ctx);
  std::vector<double> st((size_t)2 * M * N * N), tl((size_t)2 * ntl * N * N);
  double t = 0, dt = 0;
  int rc = phi_restart_read_file_ex(path, N, M, st.data(), &t, &dt, tl.data(), ntl);
  if (rc != PHI_OK) return rc;
  rc = phi_gpu_set_state(ctx, st.data());  // also resets flags, Q and H as a fresh run
  if (rc != PHI_OK) return rc;
  if (ntl > 0 && (rc = put_tl_store(ctx, tl)) != PHI_OK) return rc;
  rc = phi_gpu_set_time(ctx, t);
  if (timestep) *timestep = dt;
  return rc;
}

extern "C" int phi_gpu_save_state(phi_ctx *ctx, const char *path, double timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->ta_F > 0) return refuse_truncated_annealing(ctx);
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  std::vector<double> st((size_t)2 * M * N * N), tl;
  int rc = phi_gpu_get_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  const int64_t ntl = tl_matrix_count(ctx);
  if (ntl > 0 && (rc = get_tl_store(ctx, &tl)) != PHI_OK) return rc;
  double t = 0;
  phi_gpu_get_time(ctx, &t);
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(PHI_E_INVALID, std::string("save_state: cannot create ") + path);
  const uint32_t version = ntl > 0 ? 2 : 1, n32 = (uint32_t)N;
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
            std::fwrite(&n32, 4, 1, f) == 1 && std::fwrite(&M, 8, 1, f) == 1 && std::fwrite(&t, 8, 1, f) == 1 &&
            std::fwrite(&timestep, 8, 1, f) == 1 && std::fwrite(st.data(), 8, st.size(), f) == st.size();
  if (ok && version == 2)
    ok = std::fwrite(&ntl, 8, 1, f) == 1 && std::fwrite(tl.data(), 8, tl.size(), f) == tl.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PHI_OK : fail(PHI_E_INVALID, std::string("save_state: write failed: ") + path);
}

extern "C" int phi_gpu_load_state(phi_ctx *ctx, const char *path, double *timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->ta_F > 0) return refuse_truncated_annealing(ctx);
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(PHI_E_INVALID, std::string("load_state: cannot open ") + path);
  char magic[8];
  uint32_t version = 0, n32 = 0;
  int64_t m = 0;
  double t = 0, dt = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(&version, 4, 1, f) == 1 && (version == 1 || version == 2) &&
            std::fread(&n32, 4, 1, f) == 1 && std::fread(&m, 8, 1, f) == 1 && std::fread(&t, 8, 1, f) == 1 &&
            std::fread(&dt, 8, 1, f) == 1;
  if (!ok || (int32_t)n32 != N || m != M) {
    std::fclose(f);
    return fail(PHI_E_INVALID, "load_state: not a state file of this hierarchy (" + std::to_string(M) +
                                   " nodes of " + std::to_string(N) + "x" + std::to_string(N) + ")");
  }
  std::vector<double> st((size_t)2 * M * N * N), tl;
  ok = std::fread(st.data(), 8, st.size(), f) == st.size();
  int64_t ntl = 0;
  if (ok && version == 2) ok = std::fread(&ntl, 8, 1, f) == 1 && ntl >= 0 && ntl <= (int64_t)1 << 20;
  if (ok && ntl > 0) {
    tl.resize((size_t)2 * ntl * N * N);
    ok = std::fread(tl.data(), 8, tl.size(), f) == tl.size();
  }
  std::fclose(f);
  if (!ok) return fail(PHI_E_INVALID, "load_state: file is truncated");
  if (ntl != tl_matrix_count(ctx))
    return fail(PHI_E_INVALID, "load_state: the file holds " + std::to_string(ntl) +
                                   " time-local matrices, this context " + std::to_string(tl_matrix_count(ctx)));
  int rc = phi_gpu_set_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  if (ntl > 0 && (rc = put_tl_store(ctx, tl)) != PHI_OK) return rc;
  rc = phi_gpu_set_time(ctx, t);
  if (timestep) *timestep = dt;
  return rc;
}
