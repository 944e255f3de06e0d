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

std::string g_restart_error;

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

extern "C" int phi_restart_read_file(const char *path, int32_t num_states, int64_t num_nodes, double *state,
                                     double *time, double *timestep) {
  if (!path || num_states <= 0 || num_nodes <= 0 || !state) return fail(PHI_E_INVALID, "restart: bad arguments");
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
  double extra;
  // Time-local truncation matrices may follow in PHI's files; they are not
  // part of this library's state, and anything else is an error.
  if (next_number(s, &extra))
    return fail(PHI_E_INVALID, "restart: more values than " + std::to_string(num_nodes) + " nodes of " +
                                   std::to_string(num_states) + "x" + std::to_string(num_states) +
                                   " (time-local truncation data is not supported)");
  if (time) *time = t;
  if (timestep) *timestep = dt;
  return PHI_OK;
}

extern "C" int phi_restart_write_file(const char *path, int32_t num_states, int64_t num_nodes, const double *state,
                                      double time, double timestep) {
  if (!path || num_states <= 0 || num_nodes <= 0 || !state) return fail(PHI_E_INVALID, "restart: bad arguments");
  FILE *f = std::fopen(path, "w");
  if (!f) return fail(PHI_E_INVALID, std::string("restart: cannot create ") + path);
  std::fprintf(f, "%.17g\n%.17g\n", time, timestep);
  const long long E = (long long)num_states * num_states;
  for (long long n = 0; n < num_nodes; ++n) {
    const double *z = state + 2 * n * E;
    for (long long e = 0; e < E; ++e)
      std::fprintf(f, e ? " (%.17g,%.17g)" : "(%.17g,%.17g)", z[2 * e], z[2 * e + 1]);
    std::fputc('\n', f);
  }
  const bool ok = std::fclose(f) == 0;
  return ok ? PHI_OK : fail(PHI_E_INVALID, std::string("restart: write failed: ") + path);
}

extern "C" int phi_restart_last_error(char *buf, size_t len) {
  if (!buf || !len) return PHI_E_INVALID;
  std::snprintf(buf, len, "%s", g_restart_error.c_str());
  return PHI_OK;
}

// ---- on a context ------------------------------------------------------------

extern "C" int phi_gpu_write_restart(phi_ctx *ctx, const char *path, double timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->c.time_local) {
    ctx->error = "write_restart: a time-local run's restart state includes its Q matrices, which these files do not carry";
    return fail(PHI_E_INVALID, ctx->error);
  }
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  std::vector<double> st((size_t)2 * M * N * N);
  int rc = phi_gpu_get_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  double t = 0;
  phi_gpu_get_time(ctx, &t);
  return phi_restart_write_file(path, N, M, st.data(), t, timestep);
}

extern "C" int phi_gpu_read_restart(phi_ctx *ctx, const char *path, double *timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->c.time_local) {
    ctx->error = "read_restart: a time-local run's restart state includes its Q matrices, which these files do not carry";
    return fail(PHI_E_INVALID, ctx->error);
  }
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  std::vector<double> st((size_t)2 * M * N * N);
  double t = 0, dt = 0;
  int rc = phi_restart_read_file(path, N, M, st.data(), &t, &dt);
  if (rc != PHI_OK) return rc;
  rc = phi_gpu_set_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  rc = phi_gpu_set_time(ctx, t);
  if (timestep) *timestep = dt;
  return rc;
}

extern "C" int phi_gpu_save_state(phi_ctx *ctx, const char *path, double timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->c.time_local) {
    ctx->error = "save_state: a time-local run's restart state includes its Q matrices, which these files do not carry";
    return fail(PHI_E_INVALID, ctx->error);
  }
  int64_t M = 0;
  int32_t N = 0;
  phi_gpu_dims(ctx, &M, nullptr, &N);
  std::vector<double> st((size_t)2 * M * N * N);
  int rc = phi_gpu_get_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  double t = 0;
  phi_gpu_get_time(ctx, &t);
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(PHI_E_INVALID, std::string("save_state: cannot create ") + path);
  const uint32_t version = 1, n32 = (uint32_t)N;
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
            std::fwrite(&n32, 4, 1, f) == 1 && std::fwrite(&M, 8, 1, f) == 1 && std::fwrite(&t, 8, 1, f) == 1 &&
            std::fwrite(&timestep, 8, 1, f) == 1 && std::fwrite(st.data(), 8, st.size(), f) == st.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PHI_OK : fail(PHI_E_INVALID, std::string("save_state: write failed: ") + path);
}

extern "C" int phi_gpu_load_state(phi_ctx *ctx, const char *path, double *timestep) {
  if (!ctx || !path) return PHI_E_INVALID;
  if (ctx->c.time_local) {
    ctx->error = "load_state: a time-local run's restart state includes its Q matrices, which these files do not carry";
    return fail(PHI_E_INVALID, ctx->error);
  }
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
            std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(&n32, 4, 1, f) == 1 &&
            std::fread(&m, 8, 1, f) == 1 && std::fread(&t, 8, 1, f) == 1 && std::fread(&dt, 8, 1, f) == 1;
  if (!ok || (int32_t)n32 != N || m != M) {
    std::fclose(f);
    return fail(PHI_E_INVALID, "load_state: not a state file of this hierarchy (" + std::to_string(M) +
                                   " nodes of " + std::to_string(N) + "x" + std::to_string(N) + ")");
  }
  std::vector<double> st((size_t)2 * M * N * N);
  ok = std::fread(st.data(), 8, st.size(), f) == st.size();
  std::fclose(f);
  if (!ok) return fail(PHI_E_INVALID, "load_state: file is truncated");
  int rc = phi_gpu_set_state(ctx, st.data());
  if (rc != PHI_OK) return rc;
  rc = phi_gpu_set_time(ctx, t);
  if (timestep) *timestep = dt;
  return rc;
}
