// phi/phi_parameters.h -- drop-in PhiParameters for the B200 integrator.
//
// Same struct name, field names, units and conventions as PHI's
// phi_parameters.h:32-122 for everything the propagation and steady-state
// paths read, and the same parameter-file reader (ReadCommandLine /
// ReadInputFile / FixIncompatibleCombinations, phi_parameters.cc:93-888):
// `key=value` scalars, `Key:` matrix blocks read row by row into column-major
// storage, MatsubaraTerms stored as K+1, HierarchyTruncation counting tier 0.
// Inputs outside this library's scope (Hilbert-space truncation, spectra)
// are read and then rejected by HierarchyIntegrator with a message.
#ifndef PHI_B200_PHI_PARAMETERS_H_
#define PHI_B200_PHI_PARAMETERS_H_

#include <complex>
#include <fstream>
#include <string>

#include "../phi_b200.h"
#include "numeric_types.h"

// Reduced Planck constant in [cm-1*ps] and Boltzmann constant in [cm-1/K]
// (phi_parameters.h:13-16).
#define HBAR 5.3088354
#define K_B 0.6950344

enum RunMethod {
  BROKENINPUT,
  NONE,
  RK4,
  RKF45,
  RK4SPECTRUM,
  RKF45SPECTRUM,
  BICGSTABL,
  BICGSTAB,
  BICGSTABU,
  PRINTHIERARCHY,
  PRINTMEMORY
};

struct PHI_API PhiParameters {
  int verbose;

  Float hbar;
  Float boltzmann_constant;

  int num_states;
  int hilbert_space_num_elements;
  int hilbert_space_size;
  int num_bath_couplings;
  int num_matsubara_terms;  // K + 1

  int hierarchy_truncation_level;  // L + 1
  long long matrix_count;

  Complex *time_indepenent_hamiltonian;
  Complex *final_annealing_hamiltonian;
  Complex *initial_annealing_hamiltonian;
  // Annealing fields (TransverseField / LongitudinalField, sampled on
  // [0, 1] of the run) and MinimumFieldChange (phi_parameters.h:48-55).
  Float *initial_hamiltonian_field;
  int initial_hamiltonian_field_size;
  Float *final_hamiltonian_field;
  int final_hamiltonian_field_size;
  Float minimum_field_change;

  Float temperature;

  Float *kappa;  // accepted for compatibility (PHI declares it; no path reads it)
  Float *gamma;
  Float *lambda;
  Float *bath_coupling_op;
  int *multiple_independent_bath_indices;

  Complex *initial_density_matrix;
  Complex *spectrum_initial_density_matrix;  // spectra are out of scope; freed like PHI's

  Float integration_time;
  Float timestep;
  Float output_minimum_timestep;
  Float start_time;
  Float rkf45_minimum_timestep;
  Float rkf45_tolerance;
  Float bicgstab_tolerance;
  Float filter_tolerance;
  Float restart_output_time;  // RestartOutputTimeSecs: > 0 writes RestartFile at the end of a run

  std::string output_filename;
  std::string restart_input_filename;
  std::string restart_output_filename;
  std::string restart_backup_filename;  // accepted for compatibility

  bool is_truncated_system;
  bool use_time_local_truncation;
  bool is_multiple_independent_baths;
  bool is_spectrum_calculation;
  bool is_diagonal_bath_coupling;
  bool is_full_bath_coupling;
  bool is_rho_normalized;
  bool is_restarted;
  bool has_kappa;

  // Eigen data of the Hamiltonian (PHI's steady-state initial guess reads
  // them when present; accepted for compatibility, not owned).
  Complex *hamiltonian_eigenvectors, *hamiltonian_eigenvalues;
  bool are_e_vecs_present;
  bool are_e_vals_present;

  int bicgstab_ell;
  // CPU thread controls of PHI's pthread runtime: accepted for
  // compatibility, the GPU path ignores them.
  int num_threads;
  int num_cores;
  int *cpuaffinity;
  bool stupid_hierarchy_partition;
  bool are_parameters_valid;
  RunMethod run_method;

  // B200 additions: arithmetic of the Liouvillian (0 = FP64, 1 = mixed) and
  // the CUDA device.
  int precision;
  int device;

  PhiParameters();
  ~PhiParameters();
  PhiParameters(const PhiParameters &) = delete;
  PhiParameters &operator=(const PhiParameters &) = delete;

  void SetDefaults();
  bool FileExists(const char *filename);
  void FixIncompatibleCombinations();
  // Presence and range checks of phi_parameters.cc:890-932 (PHI itself never
  // calls it); clears are_parameters_valid with PHI's messages on stderr.
  void CheckParameters();
  void ReadCommandLine(int num_args, char *argv[]);
  void ReadInputFile(std::string parameter_file);
  void Write(std::ofstream *out, long long num_matrices);
};

// C(truncation - 1 + terms, terms): number of hierarchy nodes
// (phi_parameters.cc:1138-1147).
PHI_API long long GetHierarchyNodeCountEstimate(int truncation_level, int num_terms);

#endif  // PHI_B200_PHI_PARAMETERS_H_
