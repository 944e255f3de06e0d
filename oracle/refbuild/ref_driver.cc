// Test-harness driver around the reference PHI sources (compiled unchanged
// from the reference tree by oracle/refbuild/Makefile).  It is part of the
// oracle: only tests/, the fixture generator and bench.py's CPU-baseline arm
// run it, and only as a checker or a timed reference, never as product code.
//
//   ref_driver run   <paramfile> <rk4|rkf45> <threads> <result-file>
//       PhiParameters::ReadCommandLine (phi_parameters.cc:93-146) ->
//       HierarchyIntegrator(PhiParameters*) -> Launch() -> density_matrix()
//       (hierarchy_integrator.cc:49-62, :113-175, :177-191); writes rho_0 in
//       storage (column-major) order with %.17g plus the wall time of Launch.
//   ref_driver order <paramfile> <result-file>
//       Hierarchy::ConstructI (hierarchy.cc:45-155) through a subclass that
//       reads the protected multi-index map; writes one multi-index per id.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <sys/time.h>

#include "hierarchy_integrator.h"
#include "phi_parameters.h"

namespace {

double WallSeconds() {
  timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

// Exposes the reference's node enumeration; Hierarchy's members are protected.
class OrderProbe : public Hierarchy {
 public:
  explicit OrderProbe(PhiParameters* p) : Hierarchy(p) {}
  int Dump(FILE* out) {
    ConstructI();
    for (int id = 0; id < matrix_count_; ++id) {
      const MultiIndex& mi = multi_index_map_[id];
      for (int t = 0; t < mi.size; ++t) {
        std::fprintf(out, t ? " %d" : "%d", mi.index_array[t]);
      }
      std::fprintf(out, "\n");
    }
    return matrix_count_;
  }
};

int RunIntegration(int argc, char** argv) {
  // argv: ref_driver run <paramfile> <method> <threads> <result-file>
  char* cl[4] = {argv[0], argv[2], argv[3], argv[4]};
  PhiParameters parameters;
  parameters.ReadCommandLine(4, cl);
  if (!parameters.are_parameters_valid) {
    std::fprintf(stderr, "ref_driver: invalid parameters\n");
    return 2;
  }
  // density_matrix() is hilbert_space_size^2 (UnTruncate under Hilbert-space
  // truncation; num_states^2 otherwise).
  const int n = parameters.hilbert_space_size > parameters.num_states ? parameters.hilbert_space_size
                                                                        : parameters.num_states;
  double t0 = WallSeconds();
  HierarchyIntegrator integrator(&parameters);
  integrator.Launch();
  double t1 = WallSeconds();
  Complex* rho = integrator.density_matrix();
  FILE* out = std::fopen(argv[5], "w");
  if (!out) return 3;
  std::fprintf(out, "launch_seconds %.9f\n", t1 - t0);
  std::fprintf(out, "num_states %d\n", n);
  for (int i = 0; i < n * n; ++i) {
    std::fprintf(out, "%.17g %.17g\n", rho[i].real(), rho[i].imag());
  }
  std::fclose(out);
  delete[] rho;
  return 0;
}

int RunOrder(int argc, char** argv) {
  // argv: ref_driver order <paramfile> <result-file>
  char* cl[3] = {argv[0], argv[2], const_cast<char*>("print")};
  PhiParameters parameters;
  parameters.ReadCommandLine(3, cl);
  parameters.verbose = -2;
  if (!parameters.are_parameters_valid) return 2;
  OrderProbe probe(&parameters);
  FILE* out = std::fopen(argv[3], "w");
  if (!out) return 3;
  probe.Dump(out);
  std::fclose(out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 6 && std::string(argv[1]) == "run") return RunIntegration(argc, argv);
  if (argc == 4 && std::string(argv[1]) == "order") return RunOrder(argc, argv);
  std::fprintf(stderr,
               "usage: ref_driver run <paramfile> <rk4|rkf45> <threads> <out>\n"
               "       ref_driver order <paramfile> <out>\n");
  return 1;
}
