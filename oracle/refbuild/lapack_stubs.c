/* Stub LAPACK entry points for the -DNOBLAS oracle build of the reference.
 * They are only reached by Hilbert-space truncation and time-dependent
 * (annealing) Hamiltonians, which the oracle never runs; calling one is a
 * harness error, so each aborts loudly. */
#include <stdio.h>
#include <stdlib.h>

static void die(const char *name) {
  fprintf(stderr, "oracle reference build: LAPACK routine %s is stubbed out\n", name);
  abort();
}
double dlamch_(char *c) { (void)c; die("dlamch_"); return 0.0; }
void zheevr_(void) { die("zheevr_"); }
void dpttrf_(void) { die("dpttrf_"); }
void dpttrs_(void) { die("dpttrs_"); }
