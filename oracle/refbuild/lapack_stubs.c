/* LAPACK entry points for the -DNOBLAS oracle build of the reference.
 * zheevr / dlamch are only reached by Hilbert-space truncation, which the
 * oracle never runs; calling one is a harness error, so each aborts loudly.
 * dpttrf / dpttrs (CubicSpline::SolveTridiagonal, cubic_spline.cc:84-120, for
 * annealing Hamiltonians) are written here from the published algorithm: the
 * L D L^T factorisation of a symmetric positive definite tridiagonal matrix
 * and the forward / diagonal / backward solve, in LAPACK's operation order
 * (d(i+1) -= (e(i)/d(i)) e(i); b(i) -= b(i-1) e(i-1); b(i) = b(i)/d(i) -
 * b(i+1) e(i)). */
#include <stdio.h>
#include <stdlib.h>

static void die(const char *name) {
  fprintf(stderr, "oracle reference build: LAPACK routine %s is stubbed out\n", name);
  abort();
}
double dlamch_(char *c) { (void)c; die("dlamch_"); return 0.0; }
void zheevr_(void) { die("zheevr_"); }
void dpttrf_(int *n, double *d, double *e, int *info) {
  *info = 0;
  if (*n < 0) { *info = -1; return; }
  for (int i = 0; i < *n - 1; ++i) {
    if (!(d[i] > 0)) { *info = i + 1; return; }
    const double ei = e[i];
    e[i] = ei / d[i];
    d[i + 1] = d[i + 1] - e[i] * ei;
  }
  if (*n > 0 && !(d[*n - 1] > 0)) *info = *n;
}
void dpttrs_(int *n, int *nrhs, double *d, double *e, double *b, int *ldb, int *info) {
  *info = 0;
  if (*n < 0 || *nrhs < 0 || *ldb < (*n > 1 ? *n : 1)) { *info = -1; return; }
  for (int r = 0; r < *nrhs; ++r) {
    double *x = b + (long)r * *ldb;
    for (int i = 1; i < *n; ++i) x[i] = x[i] - x[i - 1] * e[i - 1];
    if (*n > 0) x[*n - 1] = x[*n - 1] / d[*n - 1];
    for (int i = *n - 2; i >= 0; --i) x[i] = x[i] / d[i] - x[i + 1] * e[i];
  }
}
