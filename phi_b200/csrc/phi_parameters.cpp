// phi_parameters.cpp -- parameter-file reader of the drop-in PhiParameters.
//
// Reads PHI's format (PhiParameters::ReadInputFile, phi_parameters.cc:152-784):
//   * lines containing '#' are comments;
//   * `key=value` sets a scalar;
//   * `Key:` starts an array block whose first row is the next line; every
//     following line without '=' or ':' is another row of the same block;
//   * matrix rows are comma-separated reals or "(re,im)" pairs; row r of a
//     matrix fills column-major storage, element (r, c) at r + c*N
//     (parameter_input.cc:244-339 with j_skip = N);
//   * MatsubaraTerms=K is stored as K+1 (phi_parameters.cc:257-266).
// The value checks (positive / non-negative / 0-or-1) follow
// ParameterInput::ReadValue (parameter_input.cc:10-44).
#include "../../include/phi/phi_parameters.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <vector>

namespace {

enum Range { kAny, kPositive, kNonNegative };

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

bool range_ok(double v, Range r, const std::string &name) {
  if (r == kPositive && !(v > 0)) {
    std::cerr << "get() Error: " << name << " must be positive.\n";
    return false;
  }
  if (r == kNonNegative && !(v >= 0)) {
    std::cerr << "get() Error: " << name << " must be non-negative.\n";
    return false;
  }
  return true;
}

bool parse_int(const std::string &in, const std::string &name, int *out, Range r) {
  const std::string s = trim(in);
  if (s.empty() || s.find_first_not_of("+-0123456789") != std::string::npos) {
    std::cerr << "get() Error reading " << name << "\n";
    return false;
  }
  *out = std::atoi(s.c_str());
  return range_ok(*out, r, name);
}

bool parse_double(const std::string &in, const std::string &name, double *out, Range r) {
  const std::string s = trim(in);
  if (s.empty() || s.find_first_not_of("+-.0123456789eE") != std::string::npos) {
    std::cerr << "get() Error reading " << name << "\n";
    return false;
  }
  char *end = nullptr;
  *out = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) {
    std::cerr << "get() Error reading " << name << "\n";
    return false;
  }
  return range_ok(*out, r, name);
}

bool parse_bool(const std::string &in, const std::string &name, bool *out) {
  int v = 0;
  if (!parse_int(in, name, &v, kAny) || (v != 0 && v != 1)) {
    std::cerr << "get() Error reading " << name << ".\n"
              << "Boolean parameters must be 0 (for false) or 1 (for true).\n";
    return false;
  }
  *out = v == 1;
  return true;
}

std::vector<std::string> split_commas(const std::string &s) {
  std::vector<std::string> parts;
  std::string cur;
  for (char ch : s) {
    if (ch == ',') {
      parts.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(ch);
    }
  }
  parts.push_back(cur);
  return parts;
}

// Exactly n reals.
bool parse_real_row(const std::string &in, int n, std::vector<double> *out) {
  const std::string s = trim(in);
  if (s.empty() || s.back() == ',') return false;
  auto parts = split_commas(s);
  if ((int)parts.size() != n) {
    std::cerr << "get() Error: Expected to read " << n << " values but got " << parts.size()
              << " instead in line:\n\t" << s << "\n";
    return false;
  }
  out->resize(n);
  for (int i = 0; i < n; ++i) {
    double v;
    if (!parse_double(parts[i], "array element", &v, kAny)) return false;
    (*out)[i] = v;
  }
  return true;
}

// Exactly n complex values: all "(re,im)" or all reals.
bool parse_complex_row(const std::string &in, int n, std::vector<Complex> *out) {
  const std::string s = trim(in);
  if (s.empty() || s.back() == ',') return false;
  out->assign(n, Complex(0, 0));
  if (s.find('(') == std::string::npos) {
    std::vector<double> v;
    if (!parse_real_row(s, n, &v)) return false;
    for (int i = 0; i < n; ++i) (*out)[i] = Complex(v[i], 0.0);
    return true;
  }
  size_t pos = 0;
  int k = 0;
  while (k < n) {
    size_t l = s.find('(', pos), c = s.find(',', l), r = s.find(')', c);
    if (l == std::string::npos || c == std::string::npos || r == std::string::npos) break;
    double re, im;
    if (!parse_double(s.substr(l + 1, c - l - 1), "complex element", &re, kAny) ||
        !parse_double(s.substr(c + 1, r - c - 1), "complex element", &im, kAny))
      return false;
    (*out)[k++] = Complex(re, im);
    pos = r + 1;
  }
  if (k != n || s.find('(', pos) != std::string::npos) {
    std::cerr << "get() Error: Expected to read " << n << " values in:\n\t" << s << "\n";
    return false;
  }
  return true;
}

template <class T>
T *zeros(size_t n) {
  T *p = new T[n];
  for (size_t i = 0; i < n; ++i) p[i] = T(0);
  return p;
}

}  // namespace

long long GetHierarchyNodeCountEstimate(int truncation_level, int num_terms) {
  long double c = 1.0L;
  for (int i = 1; i <= truncation_level - 1; ++i) c = c * (num_terms + i) / i;
  return (long long)(c + 0.5L);
}

PhiParameters::PhiParameters() {
  time_indepenent_hamiltonian = nullptr;
  final_annealing_hamiltonian = nullptr;
  initial_annealing_hamiltonian = nullptr;
  initial_hamiltonian_field = nullptr;
  initial_hamiltonian_field_size = 0;
  final_hamiltonian_field = nullptr;
  final_hamiltonian_field_size = 0;
  minimum_field_change = 0.01;
  kappa = gamma = lambda = bath_coupling_op = nullptr;
  multiple_independent_bath_indices = nullptr;
  initial_density_matrix = nullptr;
  spectrum_initial_density_matrix = nullptr;
  hamiltonian_eigenvectors = hamiltonian_eigenvalues = nullptr;
  cpuaffinity = nullptr;
  SetDefaults();
}

PhiParameters::~PhiParameters() {
  delete[] time_indepenent_hamiltonian;
  delete[] final_annealing_hamiltonian;
  delete[] initial_annealing_hamiltonian;
  delete[] initial_hamiltonian_field;
  delete[] final_hamiltonian_field;
  delete[] kappa;
  delete[] gamma;
  delete[] lambda;
  delete[] bath_coupling_op;
  delete[] multiple_independent_bath_indices;
  delete[] initial_density_matrix;
  delete[] spectrum_initial_density_matrix;
}

// Defaults of PhiParameters::SetDefaults (phi_parameters.cc:9-88).
void PhiParameters::SetDefaults() {
  verbose = 1;
  hbar = HBAR;
  boltzmann_constant = K_B;
  num_states = 0;
  hilbert_space_size = 0;
  hilbert_space_num_elements = 0;
  num_bath_couplings = 0;
  num_matsubara_terms = 1;
  hierarchy_truncation_level = 1;
  matrix_count = 0;
  temperature = 300;
  integration_time = 0;
  timestep = 0.001;
  output_minimum_timestep = 0.01;
  start_time = 0;
  rkf45_minimum_timestep = 1e-6;
  rkf45_tolerance = 1e-6;
  bicgstab_tolerance = 1e-6;
  filter_tolerance = 0;
  use_time_local_truncation = false;
  is_multiple_independent_baths = false;
  is_truncated_system = false;
  is_spectrum_calculation = false;
  is_diagonal_bath_coupling = false;
  is_full_bath_coupling = false;
  is_rho_normalized = true;
  is_restarted = false;
  restart_output_time = 0;
  has_kappa = false;
  are_e_vecs_present = false;
  are_e_vals_present = false;
  bicgstab_ell = 2;
  num_threads = 1;
  num_cores = 1;
  stupid_hierarchy_partition = false;
  restart_input_filename.clear();
  restart_output_filename.clear();
  restart_backup_filename.clear();
  are_parameters_valid = true;
  run_method = NONE;
  precision = 0;
  device = 0;
}

bool PhiParameters::FileExists(const char *filename) {
  std::ifstream f(filename);
  return f.is_open();
}

// PhiParameters::ReadCommandLine (phi_parameters.cc:93-146).
void PhiParameters::ReadCommandLine(int num_args, char *argv[]) {
  if (num_args < 2) {
    std::cout << "Usage: \n\n  phi_b200 paramfile {integrator [threads],print}\n"
              << "  integrator  - One of rk4, rkf45, bicgstab.\n"
              << "  threads     - Accepted and ignored (one GPU)\n";
    are_parameters_valid = false;
    return;
  }
  std::cout << "Reading parameters from " << argv[1] << "\n\n";
  if (!FileExists(argv[1])) {
    are_parameters_valid = false;
    std::cout << "ERROR: No parameter file.\n";
    return;
  }
  if (num_args == 2) {
    std::cout << "No integration method specified.\n";
    return;
  }
  if (num_args == 4) num_threads = std::atoi(argv[3]);
  const std::string m = argv[2];
  if (m == "rk4spectrum") run_method = RK4SPECTRUM;
  else if (m == "rkf45spectrum") run_method = RKF45SPECTRUM;
  else if (m == "rk4") run_method = RK4;
  else if (m == "rkf45") run_method = RKF45;
  else if (m == "print") run_method = PRINTHIERARCHY;
  else if (m == "memory") run_method = PRINTMEMORY;
  else if (m == "bicgstabl" || m == "bicgstab") run_method = BICGSTABL;
  else if (m == "bicgstabu") run_method = BICGSTABU;
  ReadInputFile(argv[1]);
}

void PhiParameters::ReadInputFile(std::string parameter_file) {
  std::ifstream in(parameter_file.c_str());
  if (!in.is_open()) {
    std::cerr << "ERROR: cannot open " << parameter_file << "\n";
    are_parameters_valid = false;
    return;
  }
  std::vector<std::string> lines;
  for (std::string l; std::getline(in, l);) lines.push_back(l);
  std::string key;
  int row = 0;
  size_t li = 0;
  auto bad = [&](const std::string &msg) {
    std::cerr << msg;
    are_parameters_valid = false;
  };
  while (li < lines.size() && are_parameters_valid) {
    std::string line = lines[li++];
    if (line.find('#') != std::string::npos) continue;
    std::string val;
    if (line.find('=') != std::string::npos) {
      const size_t p = line.find('=');
      key = trim(line.substr(0, p));
      val = line.substr(p + 1);
    } else if (line.find(':') != std::string::npos) {
      key = trim(line.substr(0, line.find(':')));
      row = 0;
      val = li < lines.size() ? lines[li++] : "";
    } else if (!trim(line).empty()) {
      val = line;  // next row of the current array block
    } else {
      key.clear();
      continue;
    }
    const int N = num_states, HS = hilbert_space_size;
    if (key == "fout" || key == "Output" || key == "OutputFile") {
      output_filename = trim(val);
    } else if (key == "Ns" || key == "NumStates") {
      if (!parse_int(val, key, &num_states, kPositive)) { are_parameters_valid = false; break; }
      if (hilbert_space_size == 0) {
        hilbert_space_size = num_states;
        hilbert_space_num_elements = num_states * num_states;
      }
      if (num_bath_couplings == 0) num_bath_couplings = num_states;
      delete[] multiple_independent_bath_indices;
      multiple_independent_bath_indices = new int[num_bath_couplings];
      for (int i = 0; i < num_bath_couplings; ++i) multiple_independent_bath_indices[i] = i;
    } else if (key == "HilbertSpaceSize") {
      if (time_indepenent_hamiltonian || is_diagonal_bath_coupling || is_full_bath_coupling) {
        bad("ERROR: HilbertSpaceSize must be specified before the Hamiltonian and bath coupling operators.\n");
        break;
      }
      if (!parse_int(val, key, &hilbert_space_size, kPositive)) { are_parameters_valid = false; break; }
      hilbert_space_num_elements = hilbert_space_size * hilbert_space_size;
      if (hilbert_space_size < num_states) { bad("ERROR: HilbertSpaceSize cannot be less than NumStates.\n"); break; }
    } else if (key == "M" || key == "NumCouplingTerms") {
      if (!parse_int(val, key, &num_bath_couplings, kPositive)) { are_parameters_valid = false; break; }
      if (num_states != 0) {
        delete[] multiple_independent_bath_indices;
        multiple_independent_bath_indices = new int[num_bath_couplings];
        for (int i = 0; i < num_bath_couplings; ++i) multiple_independent_bath_indices[i] = i;
      }
    } else if (key == "Kt" || key == "MatsubaraTerms") {
      if (!parse_int(val, key, &num_matsubara_terms, kNonNegative)) { are_parameters_valid = false; break; }
      num_matsubara_terms += 1;
    } else if (key == "Lh" || key == "HierarchyTruncation") {
      if (!parse_int(val, key, &hierarchy_truncation_level, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "dt" || key == "Timestep") {
      if (!parse_double(val, key, &timestep, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "t" || key == "Time") {
      if (!parse_double(val, key, &integration_time, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "OutputMinimumTimestep") {
      if (!parse_double(val, key, &output_minimum_timestep, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "filter" || key == "filtered" || key == "FilterTolerance") {
      if (!parse_double(val, key, &filter_tolerance, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "TL" || key == "TimeLocal") {
      if (!parse_bool(val, key, &use_time_local_truncation)) { are_parameters_valid = false; break; }
    } else if (key == "rho_normalized" || key == "rho_normalised") {
      if (!parse_bool(val, key, &is_rho_normalized)) { are_parameters_valid = false; break; }
    } else if (key == "H" || key == "Hamiltonian" || key == "rho0" || key == "InitialDensityMatrix" ||
               key == "H_X" || key == "TransverseHamiltonian" || key == "H_Z" ||
               key == "LongitudinalHamiltonian") {
      if (N <= 0) { bad("ERROR: NumStates must be specified before " + key + ".\n"); break; }
      Complex **dst = (key == "H" || key == "Hamiltonian") ? &time_indepenent_hamiltonian
                      : (key == "rho0" || key == "InitialDensityMatrix") ? &initial_density_matrix
                      : (key == "H_X" || key == "TransverseHamiltonian") ? &initial_annealing_hamiltonian
                                                                         : &final_annealing_hamiltonian;
      if (row == 0) {
        if (*dst) { bad("ERROR: " + key + " already specified\n"); break; }
        *dst = zeros<Complex>((size_t)HS * HS);
      } else if (row >= HS) {
        bad("ERROR: Overflow in " + key + " input.\n");
        break;
      }
      std::vector<Complex> v;
      if (!parse_complex_row(val, HS, &v)) { bad("ERROR: incorrect " + key + " input format.\n"); break; }
      for (int c = 0; c < HS; ++c) (*dst)[row + (size_t)c * HS] = v[c];
      ++row;
    } else if (key == "Multibath" || key == "multiBath" || key == "DiagonalCouplingIndices") {
      if (num_bath_couplings <= 0) { bad("ERROR: NumCouplingTerms must be specified before " + key + ".\n"); break; }
      std::vector<double> v;
      if (!parse_real_row(val, num_bath_couplings, &v)) { bad("ERROR: incorrect " + key + " input format.\n"); break; }
      delete[] multiple_independent_bath_indices;
      multiple_independent_bath_indices = new int[num_bath_couplings];
      for (int i = 0; i < num_bath_couplings; ++i) multiple_independent_bath_indices[i] = (int)v[i];
      is_multiple_independent_baths = true;
    } else if (key == "Vbath" || key == "DiagonalCouplingTerms" || key == "CorrelatedCouplingTerms" ||
               key == "FullBathTerms") {
      if (num_bath_couplings <= 0 || N <= 0) {
        bad("ERROR: NumCouplingTerms and NumStates must be specified before " + key + ".\n");
        break;
      }
      const bool full = key == "FullBathTerms";
      const int width = full ? HS * HS : HS;
      if (row == 0) {
        if (bath_coupling_op) { bad("ERROR: Bath coupling operators already specified\n"); break; }
        bath_coupling_op = zeros<Float>((size_t)num_bath_couplings * width);
        if (full) is_full_bath_coupling = true;
        else is_diagonal_bath_coupling = true;
      } else if (row >= num_bath_couplings) {
        bad("ERROR: Overflow in " + key + " input.\n");
        break;
      }
      std::vector<double> v;
      if (!parse_real_row(val, width, &v)) { bad("ERROR: incorrect " + key + " input format.\n"); break; }
      for (int c = 0; c < width; ++c) bath_coupling_op[(size_t)row * width + c] = v[c];
      ++row;
    } else if (key == "RestartInput") {
      restart_input_filename = trim(val);
      is_restarted = true;
    } else if (key == "lambda" || key == "Lambda" || key == "gamma" || key == "Gamma") {
      if (num_bath_couplings <= 0) { bad("ERROR: NumCouplingTerms must be specified before " + key + ".\n"); break; }
      Float **dst = (key == "lambda" || key == "Lambda") ? &lambda : &gamma;
      if (*dst) { bad("ERROR: " + key + " already specified\n"); break; }
      std::vector<double> v;
      if (!parse_real_row(val, num_bath_couplings, &v)) { bad("ERROR: incorrect " + key + " input format.\n"); break; }
      *dst = zeros<Float>(num_bath_couplings);
      for (int i = 0; i < num_bath_couplings; ++i) (*dst)[i] = v[i];
    } else if (key == "TransverseField" || key == "LongitudinalField") {
      // Comma-separated samples (phi_parameters.cc:385-433).
      const int count = (int)std::count(val.begin(), val.end(), ',') + 1;
      std::vector<double> v;
      if (!parse_real_row(val, count, &v)) { bad("ERROR: incorrect " + key + " input format.\n"); break; }
      Float **dst = key == "TransverseField" ? &initial_hamiltonian_field : &final_hamiltonian_field;
      int *size = key == "TransverseField" ? &initial_hamiltonian_field_size : &final_hamiltonian_field_size;
      delete[] *dst;
      *dst = zeros<Float>(count);
      for (int i = 0; i < count; ++i) (*dst)[i] = v[i];
      *size = count;
    } else if (key == "MinimumFieldChange") {
      if (!parse_double(val, key, &minimum_field_change, kNonNegative)) { are_parameters_valid = false; break; }
    } else if (key == "kappa") {
      has_kappa = true;
    } else if (key == "T" || key == "Temperature") {
      if (!parse_double(val, key, &temperature, kNonNegative)) { are_parameters_valid = false; break; }
    } else if (key == "verbose") {
      verbose = std::atoi(trim(val).c_str());
    } else if (key == "RestartFile") {
      restart_output_filename = trim(val);
    } else if (key == "RestartOutputTimeSecs") {
      if (!parse_double(val, key, &restart_output_time, kNonNegative)) { are_parameters_valid = false; break; }
    } else if (key == "tol_low" || key == "RKF45mindt") {
      if (!parse_double(val, key, &rkf45_minimum_timestep, kPositive)) { are_parameters_valid = false; break; }
      if (key == "tol_low") bicgstab_tolerance = rkf45_minimum_timestep;
    } else if (key == "tol_high" || key == "RKF45tolerance") {
      if (!parse_double(val, key, &rkf45_tolerance, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "bicgstab_tolerance") {
      if (!parse_double(val, key, &bicgstab_tolerance, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "bicgstab") {
      if (!parse_int(val, key, &bicgstab_ell, kNonNegative)) { are_parameters_valid = false; break; }
    } else if (key == "hbar") {
      if (!parse_double(val, key, &hbar, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "kB" || key == "k_B") {
      if (!parse_double(val, key, &boltzmann_constant, kPositive)) { are_parameters_valid = false; break; }
    } else if (key == "Precision") {  // B200 addition: 0 = FP64, 1 = mixed
      if (!parse_int(val, key, &precision, kNonNegative)) { are_parameters_valid = false; break; }
    }
  }
  if (!are_parameters_valid) {
    std::cout << "Invalid parameters.\n";
    return;
  }
  if (run_method != PRINTMEMORY) FixIncompatibleCombinations();
  matrix_count = GetHierarchyNodeCountEstimate(hierarchy_truncation_level,
                                               num_bath_couplings * num_matsubara_terms);
}

// PhiParameters::FixIncompatibleCombinations (phi_parameters.cc:786-888).
void PhiParameters::CheckParameters() {
  const std::string e = "INPUT ERROR ";
  auto bad = [&](const char *msg) {
    std::cerr << e << msg << "\n";
    are_parameters_valid = false;
  };
  if (num_states <= 0) bad("NumStates must be > 0");
  if (hierarchy_truncation_level < 1) bad("HierarchyTruncation must be > 0");
  if (num_bath_couplings <= 0) bad("NumCouplingTerms must be > 0");
  if (num_matsubara_terms < 0) bad("NumMatsubaraTerms must be >= 0");
  // A static Hamiltonian, or both annealing Hamiltonians.  (PHI's test asks
  // for both kinds at once, which no valid input has.)
  if (time_indepenent_hamiltonian == nullptr &&
      (initial_annealing_hamiltonian == nullptr || final_annealing_hamiltonian == nullptr))
    bad("Hamiltonian must be specified");
  if (gamma == nullptr) bad("Gamma values must be specified");
  if (lambda == nullptr) bad("Lambda values must be specified");
  if (initial_density_matrix == nullptr && spectrum_initial_density_matrix == nullptr && is_spectrum_calculation)
    bad("Initial state must be specified");
  if (use_time_local_truncation && is_restarted)
    bad("Restarting time-local calculations truncation not implemented.");
}

void PhiParameters::FixIncompatibleCombinations() {
  are_parameters_valid = !(time_indepenent_hamiltonian == nullptr &&
                           (initial_annealing_hamiltonian == nullptr ||
                            final_annealing_hamiltonian == nullptr));
  if (!are_parameters_valid && run_method != NONE) {
    std::cout << "Invalid parameters, no Hamiltonian?.\n";
    run_method = BROKENINPUT;
    return;
  }
  // Annealing without field samples: the transverse field ramps 1 -> 0 and
  // the longitudinal one 0 -> 1 over the run (phi_parameters.cc:801-815).
  if (initial_annealing_hamiltonian != nullptr && initial_hamiltonian_field == nullptr) {
    initial_hamiltonian_field_size = 2;
    initial_hamiltonian_field = new Float[2]{1.0, 0.0};
  }
  if (initial_annealing_hamiltonian != nullptr && final_hamiltonian_field == nullptr) {
    final_hamiltonian_field_size = 2;
    final_hamiltonian_field = new Float[2]{0.0, 1.0};
  }
  if ((run_method == RKF45 || run_method == RKF45SPECTRUM || run_method == BICGSTAB ||
       run_method == BICGSTABL || run_method == BICGSTABU) &&
      !is_rho_normalized) {
    if (verbose > 0) std::cout << "Forcing rho hierarchy scaling.\n";
    is_rho_normalized = true;
  }
  if (run_method == BICGSTAB || run_method == BICGSTABL || run_method == BICGSTABU)
    use_time_local_truncation = false;
  if (run_method == BICGSTABL && bicgstab_ell < 1) run_method = BICGSTAB;
  if (filter_tolerance > 0 && (is_diagonal_bath_coupling || is_full_bath_coupling))
    filter_tolerance = 0;
  is_spectrum_calculation = run_method == RK4SPECTRUM || run_method == RKF45SPECTRUM;
  if (multiple_independent_bath_indices == nullptr && num_bath_couplings > 0) {
    multiple_independent_bath_indices = new int[num_bath_couplings];
    for (int i = 0; i < num_bath_couplings; ++i) multiple_independent_bath_indices[i] = i;
  }
  if (hilbert_space_size < num_states) {
    hilbert_space_size = num_states;
    hilbert_space_num_elements = num_states * num_states;
  } else if (hilbert_space_size > num_states) {
    is_truncated_system = true;
  }
}

// Header echo of PhiParameters::Write (phi_parameters.cc:934-1118), for the
// fields this library reads.
void PhiParameters::Write(std::ofstream *out, long long num_matrices) {
  if (!out || !out->is_open()) return;
  std::ostream &o = *out;
  o << "#PHI 1.1\n#Parameters:\n#-----------\n";
  if (hbar != HBAR) o << "#ReducedPlanckConstant=" << hbar << "\n";
  if (boltzmann_constant != K_B) o << "#BoltzmannConstant=" << boltzmann_constant << "\n";
  o << "#NumStates=" << num_states << "\n";
  o << "#MatsubaraTerms=" << num_matsubara_terms - 1 << "\n";
  o << "#CouplingTerms=" << num_bath_couplings << "\n";
  o << "#Temperature=" << temperature << "\n";
  o << "#HierarchyTruncation=" << hierarchy_truncation_level << "\n";
  o << "#TimeLocal=" << use_time_local_truncation << "\n";
  o << "#Timestep=" << timestep << "\n";
  o << "#Time=" << integration_time << "\n";
  o << "#filter=" << filter_tolerance << "\n";
  o << "#RKF45tolerance = " << rkf45_tolerance << "\n";
  o << "#RKF45mindt = " << rkf45_minimum_timestep << "\n";
  auto row = [&](const char *name, const Float *v, int n) {
    if (!v || n <= 0) return;
    o << "#" << name << ":\n#";
    for (int i = 0; i < n; ++i) o << v[i] << (i + 1 < n ? "," : "\n");
  };
  row("gamma", gamma, num_bath_couplings);
  row("lambda", lambda, num_bath_couplings);
  row("TransverseField", initial_hamiltonian_field, initial_hamiltonian_field_size);
  row("LongitudinalField", final_hamiltonian_field, final_hamiltonian_field_size);
  if (is_multiple_independent_baths && multiple_independent_bath_indices && num_bath_couplings > 0) {
    o << "#multiBath:\n#";
    for (int i = 0; i < num_bath_couplings; ++i)
      o << multiple_independent_bath_indices[i] << (i + 1 < num_bath_couplings ? "," : "\n");
  }
  if (bath_coupling_op) {
    const int width = is_full_bath_coupling ? num_states * num_states : num_states;
    o << (is_full_bath_coupling ? "#FullBathTerms:\n" : "#CorrelatedCouplingTerms:\n");
    for (int b = 0; b < num_bath_couplings; ++b) {
      o << "#";
      for (int i = 0; i < width; ++i) o << bath_coupling_op[(size_t)b * width + i] << (i + 1 < width ? "," : "\n");
    }
  }
  // Row r as PHI prints it (phi_parameters.cc:1054-1074): elements (r, c)
  // for c < N-1, then storage element (r+1)*N - 1 -- which is element
  // (N-1, r), not (r, N-1); kept so the header reads back the same.
  auto matrix = [&](const char *name, const Complex *m) {
    if (!m) return;
    o << "#" << name << ":\n";
    for (int r = 0; r < num_states; ++r) {
      o << "#";
      for (int c = 0; c + 1 < num_states; ++c) o << m[r + (size_t)c * num_states] << ",";
      o << m[(size_t)(r + 1) * num_states - 1] << "\n";
    }
  };
  matrix("TransverseHamiltonian", initial_annealing_hamiltonian);
  matrix("LongitudinalHamiltonian", final_annealing_hamiltonian);
  matrix("Hamiltonian", time_indepenent_hamiltonian);
  matrix("InitialDensityMatrix", initial_density_matrix);
  if (!restart_input_filename.empty()) o << "#RestartInput=" << restart_input_filename << "\n";
  if (restart_output_time > 0) {
    o << "#RestartOutputTime=" << restart_output_time << "\n";
    o << "#RestartFile=" << restart_output_filename << "\n";
  }
  o << "#Estimated Number of Matrices=" << num_matrices << "\n#-------------\n";
}
