// hierarchy_integrator.cpp -- drop-in HierarchyIntegrator facade over the C ABI
// and PHI's output-file layout (hierarchy_integrator.cc:313-319 header,
// :1148-1157 initial line, :2859-2880 RK4 rows, :2530-2558 / :2905-2924
// closing lines).
#include "../../include/phi/hierarchy_integrator.h"

#include <algorithm>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <vector>

namespace phi {

void set_create_error(const std::string &msg);

int descriptor_from_parameters(const PhiParameters &p, phi_problem_desc *d, std::string *err) {
  auto reject = [&](const std::string &m) {
    *err = m;
    return PHI_E_INVALID;
  };
  if (!p.are_parameters_valid || p.run_method == BROKENINPUT) return reject("parameter error");
  const bool annealing = p.time_indepenent_hamiltonian == nullptr;
  if (annealing && (p.initial_annealing_hamiltonian == nullptr || p.final_annealing_hamiltonian == nullptr ||
                    p.initial_hamiltonian_field_size < 2 || p.final_hamiltonian_field_size < 2))
    return reject("an annealing Hamiltonian needs TransverseHamiltonian, LongitudinalHamiltonian and both "
                  "field arrays (2 samples or more)");

  if (p.use_time_local_truncation && p.is_multiple_independent_baths && !p.is_diagonal_bath_coupling &&
      !p.is_full_bath_coupling)
    return reject("time-local truncation with independent baths needs PHI's identity site map");
  if (p.is_spectrum_calculation) return reject("spectrum calculations are outside this library's scope");
  const bool steady = p.run_method == BICGSTAB || p.run_method == BICGSTABL || p.run_method == BICGSTABU;
  if (p.initial_density_matrix == nullptr && !steady && !p.is_restarted)
    return reject("InitialDensityMatrix is required (the thermal guess needs LAPACK and is not supported)");
  if (p.gamma == nullptr || p.lambda == nullptr) return reject("Gamma and Lambda are required");
  *d = phi_problem_desc{};
  d->num_states = p.num_states;
  d->num_baths = p.num_bath_couplings;
  d->num_matsubara_terms = p.num_matsubara_terms;
  d->truncation_level = p.hierarchy_truncation_level;
  d->bath_kind = p.is_full_bath_coupling ? PHI_BATH_FULL
                 : p.is_diagonal_bath_coupling ? PHI_BATH_DIAGONAL : PHI_BATH_INDEPENDENT;
  d->normalized = p.is_rho_normalized ? 1 : 0;
  d->hbar = p.hbar;
  d->boltzmann_constant = p.boltzmann_constant;
  d->temperature = p.temperature;
  d->hamiltonian = reinterpret_cast<const double *>(p.time_indepenent_hamiltonian);
  d->initial_density_matrix = reinterpret_cast<const double *>(p.initial_density_matrix);
  if (!d->initial_density_matrix) {
    // Steady-state runs need no initial state; the context starts from I/N
    // (copied by phi_gpu_create before this buffer is reused).
    static thread_local std::vector<Complex> uniform;
    uniform.assign((size_t)p.num_states * p.num_states, Complex(0, 0));
    for (int i = 0; i < p.num_states; ++i) uniform[(size_t)i * (p.num_states + 1)] = 1.0 / p.num_states;
    d->initial_density_matrix = reinterpret_cast<const double *>(uniform.data());
  }
  d->gamma = p.gamma;
  d->lambda = p.lambda;
  d->coupling = (p.is_full_bath_coupling || p.is_diagonal_bath_coupling) ? p.bath_coupling_op : nullptr;
  d->bath_sites = (p.is_multiple_independent_baths && d->bath_kind == PHI_BATH_INDEPENDENT)
                      ? p.multiple_independent_bath_indices : nullptr;
  d->precision = p.precision;
  d->device = p.device;
  d->max_nodes = 0;
  d->filter_tolerance = p.filter_tolerance;  // already 0 for diagonal / full baths
  d->time_local = p.use_time_local_truncation ? 1 : 0;  // already 0 for the steady-state methods
  // Hilbert-space truncation: the matrices above are given in the full space.
  d->hilbert_space_size = p.hilbert_space_size > p.num_states ? p.hilbert_space_size : 0;
  if (annealing) {
    d->hamiltonian = nullptr;
    d->annealing_h_x = reinterpret_cast<const double *>(p.initial_annealing_hamiltonian);
    d->annealing_h_z = reinterpret_cast<const double *>(p.final_annealing_hamiltonian);
    d->transverse_field = p.initial_hamiltonian_field;
    d->transverse_field_size = p.initial_hamiltonian_field_size;
    d->longitudinal_field = p.final_hamiltonian_field;
    d->longitudinal_field_size = p.final_hamiltonian_field_size;
    d->integration_time = p.integration_time;
    d->minimum_field_change = p.minimum_field_change;
  }
  return PHI_OK;
}

}  // namespace phi

HierarchyIntegrator::HierarchyIntegrator(PhiParameters *p) : parameters_(p) {}

HierarchyIntegrator::~HierarchyIntegrator() {
  if (ctx_) phi_gpu_destroy(ctx_);
  delete[] result_;
}

void HierarchyIntegrator::Fail(int code, const std::string &msg) {
  status_ = code;
  error_ = msg;
  if (parameters_->verbose > -2) std::cerr << "phi_b200: " << msg << "\n";
}

bool HierarchyIntegrator::Prepare() {
  phi_problem_desc d;
  std::string err;
  int rc = phi::descriptor_from_parameters(*parameters_, &d, &err);
  if (rc != PHI_OK) {
    Fail(rc, err);
    return false;
  }
  rc = phi_gpu_create(&d, &ctx_);
  if (rc != PHI_OK) {
    char buf[512];
    phi_gpu_last_error(nullptr, buf, sizeof buf);
    Fail(rc, buf);
    return false;
  }
  phi_gpu_set_time(ctx_, parameters_->start_time);
  return true;
}

void HierarchyIntegrator::Launch() {
  if (!parameters_->are_parameters_valid || parameters_->run_method == BROKENINPUT ||
      parameters_->run_method == NONE) {
    if (!parameters_->are_parameters_valid) std::cout << "Parameter error.\n";
    status_ = PHI_E_INVALID;
    return;
  }
  Run(0, parameters_->num_threads, parameters_->run_method);
  if (parameters_->verbose > -2) std::cout << "Done.\n";
}

void HierarchyIntegrator::Run(int, int, RunMethod method) {
  const bool steady = method == BICGSTAB || method == BICGSTABL || method == BICGSTABU;
  if (method != RK4 && method != RKF45 && !steady) {
    Fail(PHI_E_INVALID, "run method not provided by this build of the library");
    return;
  }
  if (!Prepare()) return;
  const int N = parameters_->num_states;
  if (parameters_->is_restarted && !steady) {
    // InitializeDensityMatrix with RestartInput (hierarchy_integrator.cc:
    // 1045-1061): the whole hierarchy, the start time and the step size
    // come from the restart file.
    double dt = parameters_->timestep;
    int rc = phi_gpu_read_restart(ctx_, parameters_->restart_input_filename.c_str(), &dt);
    if (rc != PHI_OK) {
      char buf[512];
      phi_restart_last_error(buf, sizeof buf);
      Fail(rc, std::string("RestartInput: ") + buf);
      return;
    }
    double t0 = parameters_->start_time;
    phi_gpu_get_time(ctx_, &t0);
    parameters_->start_time = t0;
    parameters_->timestep = dt;
  }
  int64_t M = 0;
  phi_gpu_dims(ctx_, &M, nullptr, nullptr);
  std::ofstream out;
  if (!parameters_->output_filename.empty()) out.open(parameters_->output_filename.c_str());
  // PrepareForOutput (hierarchy_integrator.cc:313-319) and the t = start line
  // of InitializeDensityMatrix (:1148-1157).
  if (out.is_open()) {
    // PhiParameters::Write, its run-method lines (phi_parameters.cc:1087-
    // 1117) and PrepareForOutput (hierarchy_integrator.cc:313-319).
    parameters_->Write(&out, M);
    out << "#Threads=" << parameters_->num_threads << "\n";
    if (!steady)
      out << "#Integrator=" << (method == RK4 ? "rk4" : "rkf45") << "\n";
    else if (method == BICGSTABL)
      out << "#Calculating steady-state using BiCGSTAB(" << parameters_->bicgstab_ell << ")\n";
    else
      out << "#Calculating steady-state using BiCGSTAB\n";
    out << "#Total Number of matrices:" << M << std::endl;
    WriteMemoryLines(out, M);
    out << "#-------------\n";
    if (!steady) {
      out << parameters_->start_time << " ";
      std::vector<Complex> rho0((size_t)N * N);
      phi_gpu_get_rho0(ctx_, reinterpret_cast<double *>(rho0.data()));  // rho(0) or the restart's rho_0
      for (int i = 0; i < N * N; ++i) out << rho0[i] << " ";
      out << "\n";
    }
    out << std::flush;
  }
  if (method == RK4) RunRk4(out);
  else if (method == RKF45) RunRkf45(out);
  else RunSteadyState(out);
  if (status_ == PHI_OK || (steady && status_ == PHI_E_NO_CONVERGENCE)) {
    // rho_0 in the full Hilbert space (UnTruncate under truncation).
    int32_t F = N;
    phi_gpu_hilbert_space_size(ctx_, &F);
    delete[] result_;
    result_ = new Complex[(size_t)F * F];
    result_size_ = F;
    phi_gpu_get_rho0_full(ctx_, reinterpret_cast<double *>(result_));
    has_result_ = true;
  }
}

void HierarchyIntegrator::RunRk4(std::ofstream &out) {
  const PhiParameters &p = *parameters_;
  const int N = p.num_states;
  const double dt = p.timestep;
  // Rows written after steps i with i % ceil(OutputMinimumTimestep/dt) == 0
  // (hierarchy_integrator.cc:2617-2618, :2858-2880).
  const long long of = (long long)std::ceil(p.output_minimum_timestep / dt);
  long long rows = 0;
  {
    double t = p.start_time;
    long long i = 0;
    while (t < p.integration_time) {
      t += dt;
      if (of > 0 && i % of == 0) ++rows;
      ++i;
    }
  }
  std::vector<double> traj((size_t)std::max<long long>(rows, 1) * 2 * N * N);
  std::vector<double> times((size_t)std::max<long long>(rows, 1));
  int64_t nsteps = 0, nout = 0;
  const std::time_t t1 = std::time(nullptr);
  int rc = phi_gpu_rk4(ctx_, dt, p.integration_time, p.output_minimum_timestep, traj.data(),
                       times.data(), rows, &nsteps, &nout);
  const std::time_t t2 = std::time(nullptr);
  if (rc != PHI_OK) {
    char buf[512];
    phi_gpu_last_error(ctx_, buf, sizeof buf);
    Fail(rc, buf);
    return;
  }
  steps_ = nsteps;
  accepted_ = nsteps;
  WriteRestartIfAsked(dt);
  if (!out.is_open()) return;
  const Complex *rows_c = reinterpret_cast<const Complex *>(traj.data());
  for (long long r = 0; r < std::min<long long>(nout, rows); ++r) {
    out << times[r];
    for (int j = 0; j < N * N; ++j) out << " " << rows_c[r * N * N + j];
    out << "\n";
  }
  std::vector<Complex> rho((size_t)N * N);
  phi_gpu_get_rho0(ctx_, reinterpret_cast<double *>(rho.data()));
  double tnow = 0;
  phi_gpu_get_time(ctx_, &tnow);
  if (p.verbose > -1) {
    out << "#Total number of integration steps = " << nsteps << "\n"
        << "#Total integration time = " << std::difftime(t2, t1) / 60 << " mins\n";
  }
  out << std::setw(20) << std::setprecision(6) << tnow << std::setw(6) << std::setprecision(4);
  for (int j = 0; j < N * N; ++j) out << " " << rho[j];
  out << "\n";
}

void HierarchyIntegrator::RunRkf45(std::ofstream &out) {
  const PhiParameters &p = *parameters_;
  const int N = p.num_states;
  phi_rkf45_stats st{};
  const std::time_t t1 = std::time(nullptr);
  int rc = phi_gpu_rkf45(ctx_, p.timestep, p.integration_time, p.rkf45_tolerance,
                         p.rkf45_minimum_timestep, 0, &st);
  const std::time_t t2 = std::time(nullptr);
  if (rc != PHI_OK) {
    char buf[512];
    phi_gpu_last_error(ctx_, buf, sizeof buf);
    Fail(rc, buf);
    return;
  }
  steps_ = st.steps;
  accepted_ = st.accepted;
  WriteRestartIfAsked(st.final_dt);
  if (!out.is_open()) return;
  std::vector<Complex> rho((size_t)N * N);
  phi_gpu_get_rho0(ctx_, reinterpret_cast<double *>(rho.data()));
  if (p.verbose > -1) {
    out << "#Total number of integration steps = " << st.steps << "\n"
        << "#Total number of accepted integration steps = " << st.accepted << "\n"
        << "#Total integration time = " << std::difftime(t2, t1) / 60 << " mins.\n";
  }
  out << std::setw(20) << std::setprecision(6) << st.final_time << std::setw(6)
      << std::setprecision(4);
  for (int j = 0; j < N * N; ++j) out << " " << rho[j];
  out << std::endl;
}

// BiCGSTAB(ell), BiCGSTAB and the "unstable" variant of the reference
// (hierarchy_integrator.cc:3112, :3495, :3785) solve the same system.
// BICGSTABL runs the device BiCGSTAB(ell) with ell = bicgstab_ell and the
// reference's rule ||r|| <= BiCGSTABTolerance; BICGSTAB and BICGSTABU run
// ell = 1 with ||r||^2 <= BiCGSTABTolerance and at most 9999 steps.  Output
// follows :1595-1606 (initial guess) and :3730-3761 (closing lines and the
// final rho_0 row).
void HierarchyIntegrator::RunSteadyState(std::ofstream &out) {
  const PhiParameters &p = *parameters_;
  const int N = p.num_states;
  if (out.is_open()) {
    out << "#Initial rho:\n#";
    for (int i = 0; i < N * N; ++i) out << Complex(i % (N + 1) == 0 ? 1.0 / N : 0.0, 0.0) << " ";
    out << std::endl;
  }
  phi_solve_stats st{};
  const std::time_t t1 = std::time(nullptr);
  const bool ell_method = p.run_method == BICGSTABL;
  const int ell = ell_method ? std::min(std::max(p.bicgstab_ell, 1), 8) : 1;
  int rc = phi_gpu_steady_state(ctx_, ell, p.bicgstab_tolerance, ell_method ? PHI_TOL_ABSOLUTE : PHI_TOL_ABS_SQUARED,
                                ell_method ? 999999 : 9999, nullptr, &st);
  const std::time_t t2 = std::time(nullptr);
  if (rc != PHI_OK && rc != PHI_E_NO_CONVERGENCE) {
    char buf[512];
    phi_gpu_last_error(ctx_, buf, sizeof buf);
    Fail(rc, buf);
    return;
  }
  steps_ = st.iterations;
  accepted_ = st.iterations;
  residual_ = st.residual;
  if (rc == PHI_E_NO_CONVERGENCE) {
    status_ = rc;
    error_ = "BiCGSTAB did not converge";
    if (p.verbose > -2) std::cout << "Convergence failed! (steps = " << st.iterations << ", diff = " << st.residual << ")\n";
  } else if (p.verbose > -2) {
    std::cout << "Converged to diff = " << st.residual << " in " << st.iterations << " steps.\n";
  }
  if (!out.is_open()) return;
  if (rc == PHI_E_NO_CONVERGENCE)
    out << "#Info: Total steps = " << st.iterations << ". No convergence.\n";
  else
    out << "#Info: Converged to diff = " << st.residual << " in " << st.iterations << " steps.\n";
  out << "#Info: Total running time: " << std::difftime(t2, t1) / 60 / 60 / 24 << " days.\n";
  std::vector<Complex> rho((size_t)N * N);
  phi_gpu_get_rho0(ctx_, reinterpret_cast<double *>(rho.data()));
  out << st.iterations << " ";
  for (int j = 0; j < N * N; ++j) out << rho[j] << " ";
  out << std::endl;
}

// Memory block of PHI's header (PrintMemoryRequirements(true),
// hierarchy_integrator.cc:302-310), with this library's device buffers: the
// hierarchy state, and the state plus work buffers of RK4 (y, acc and two
// stage inputs), RKF45 (y, its ping-pong, five k, two stage inputs) and the
// BiCGSTAB(2) steady state (x, rhat, b, r_0..r_2, u_0..u_2).  Spectra are
// not provided (0).
void HierarchyIntegrator::WriteMemoryLines(std::ofstream &out, long long M) const {
  const int N = parameters_->num_states;
  const double E = (double)N * N, EP = E + ((N * N) & 1);
  const bool mixed = parameters_->precision == PHI_PREC_MIXED;
  const double mb = 1.0 / 1024 / 1024;
  const double state = 16.0 * E * M * mb, work = (mixed ? 8.0 * EP : 16.0 * E) * M * mb;
  const float hierarchy = (float)state;
  const float rk4 = (float)(2 * state + (mixed ? 3 : 2) * work);
  const float rkf45 = (float)(2 * state + 7 * work + (mixed ? 2 * work : 0));
  const float steady = (float)(state + 9 * state);
  out << "#Memory to store matrices for calculations:\n";
  out << "#hierarchy: " << hierarchy << " Mb.\n";
  out << "#rk4: " << rk4 << " Mb.\n";
  out << "#rkf45: " << rkf45 << " Mb.\n";
  out << "#rk4spectrum: " << 0 << " Mb.\n";
  out << "#rkf45spectrum: " << 0 << " Mb.\n";
  out << "#steadystate: " << steady << " Mb.\n";
}

// The closing restart file of Rk4Integrate / Rkf45Integrate
// (hierarchy_integrator.cc:2559-2563, :2925-2929): written when
// RestartOutputTimeSecs > 0.  The periodic wall-clock writes during a run are
// not made: a run is one device call.
void HierarchyIntegrator::WriteRestartIfAsked(double timestep) {
  const PhiParameters &p = *parameters_;
  if (!(p.restart_output_time > 0) || p.restart_output_filename.empty()) return;
  const int rc = phi_gpu_write_restart(ctx_, p.restart_output_filename.c_str(), timestep);
  if (rc != PHI_OK) {
    char buf[512];
    phi_restart_last_error(buf, sizeof buf);
    Fail(rc, std::string("RestartFile: ") + buf);
  }
}

Complex *HierarchyIntegrator::density_matrix() {
  // hilbert_space_size x hilbert_space_size, like PHI's (its truncated
  // systems return rho in the full space, hierarchy_integrator.cc:177-191).
  const int N = parameters_->num_states;
  const int H = std::max(N, parameters_->hilbert_space_size);
  Complex *rho = new Complex[(size_t)H * H];
  for (int i = 0; i < H * H; ++i) rho[i] = Complex(0, 0);
  if (has_result_) {
    const int R = std::min(result_size_, H);
    for (int j = 0; j < R; ++j)
      for (int i = 0; i < R; ++i) rho[i + (size_t)j * H] = result_[i + (size_t)j * result_size_];
  } else if (parameters_->initial_density_matrix) {
    for (int i = 0; i < H * H; ++i) rho[i] = parameters_->initial_density_matrix[i];
  }
  return rho;
}

extern "C" int phi_gpu_create_from_file(const char *path, const char *method, int32_t precision,
                                        int32_t device, phi_ctx **out) {
  if (!out || !path || !method) return PHI_E_INVALID;
  *out = nullptr;
  char prog[] = "phi_b200";
  std::string ps(path), ms(method);
  std::vector<char> a1(ps.begin(), ps.end()), a2(ms.begin(), ms.end());
  a1.push_back(0);
  a2.push_back(0);
  char *argv[3] = {prog, a1.data(), a2.data()};
  PhiParameters p;
  p.verbose = -2;
  std::streambuf *old = std::cout.rdbuf(nullptr);  // the reader echoes to stdout
  p.ReadCommandLine(3, argv);
  std::cout.rdbuf(old);
  p.precision = precision;
  p.device = device;
  if (p.run_method == NONE) {
    phi::set_create_error("unknown integration method '" + ms + "'");
    return PHI_E_INVALID;
  }
  phi_problem_desc d;
  std::string err;
  int rc = phi::descriptor_from_parameters(p, &d, &err);
  if (rc != PHI_OK) {
    phi::set_create_error(err);  // reported by phi_gpu_last_error(NULL, ...)
    return rc;
  }
  return phi_gpu_create(&d, out);
}
