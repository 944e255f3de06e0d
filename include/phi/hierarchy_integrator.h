// phi/hierarchy_integrator.h -- drop-in HierarchyIntegrator for the B200
// integrator.
//
// Serves the call sequence of PHI's CLI (phi.cc:4-10) and of its tests
// (hierarchy_integrator_test.cc:38-44):
//
//   PhiParameters p;  ... fill fields or p.ReadCommandLine(argc, argv) ...
//   p.FixIncompatibleCombinations();
//   HierarchyIntegrator integrator(&p);
//   integrator.Launch();
//   Complex *rho = integrator.density_matrix();   // caller delete[]s
//
// Launch() blocks, runs p->run_method (RK4, RKF45, BICGSTAB*) on one GPU and
// writes PHI's output file (the `#` parameter echo, the rho_0 trajectory in
// storage order, the closing step counts).  As in the reference, invalid
// parameters or BROKENINPUT make Launch() a no-op; here status() and error()
// also report why.  num_threads is accepted and ignored.
#ifndef PHI_B200_HIERARCHY_INTEGRATOR_H_
#define PHI_B200_HIERARCHY_INTEGRATOR_H_

#include <string>

#include "../phi_b200.h"
#include "phi_parameters.h"

class PHI_API HierarchyIntegrator {
 public:
  explicit HierarchyIntegrator(PhiParameters *p);
  ~HierarchyIntegrator();
  HierarchyIntegrator(const HierarchyIntegrator &) = delete;
  HierarchyIntegrator &operator=(const HierarchyIntegrator &) = delete;

  // hierarchy_integrator.cc:113-175
  void Launch();
  // hierarchy_integrator.cc:816-868; id and num_threads are ignored.
  void Run(int id, int num_threads, RunMethod method);
  // hierarchy_integrator.cc:177-191: new Complex[N*N], column-major.
  Complex *density_matrix();

  // B200 additions.
  int status() const { return status_; }
  const std::string &error() const { return error_; }
  phi_ctx *context() { return ctx_; }
  long long steps() const { return steps_; }
  long long accepted_steps() const { return accepted_; }
  // Steady-state runs: BiCGSTAB iterations and final ||r||^2.
  double residual() const { return residual_; }

 private:
  PhiParameters *parameters_;
  phi_ctx *ctx_ = nullptr;
  int status_ = PHI_OK;
  std::string error_;
  long long steps_ = 0;
  long long accepted_ = 0;
  double residual_ = 0;
  bool has_result_ = false;
  Complex *result_ = nullptr;  // result_size_ x result_size_ (the full Hilbert space)
  int result_size_ = 0;

  bool Prepare();
  void RunRk4(std::ofstream &out);
  void RunRkf45(std::ofstream &out);
  void RunSteadyState(std::ofstream &out);
  void WriteRestartIfAsked(double timestep);
  void WriteMemoryLines(std::ofstream &out, long long M) const;
  void Fail(int code, const std::string &msg);
};

namespace phi {
// Checks that a PhiParameters lies inside this library's scope and fills a
// descriptor whose array pointers alias the parameters' arrays
// (std::complex<double> arrays are interleaved re/im doubles).
int descriptor_from_parameters(const PhiParameters &p, phi_problem_desc *d, std::string *err);
}

#endif  // PHI_B200_HIERARCHY_INTEGRATOR_H_
