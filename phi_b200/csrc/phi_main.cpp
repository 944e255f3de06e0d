// phi_main.cpp -- command-line driver with PHI's interface (phi.cc:4-10):
//   phi_b200 paramfile {rk4,rkf45} [threads]
#include "../../include/phi/hierarchy_integrator.h"
#include "../../include/phi/phi_parameters.h"

int main(int argc, char *argv[]) {
  PhiParameters parameters;
  parameters.ReadCommandLine(argc, argv);
  HierarchyIntegrator integrator(&parameters);
  integrator.Launch();
  return integrator.status() == PHI_OK || parameters.run_method == NONE ? 0 : 1;
}
