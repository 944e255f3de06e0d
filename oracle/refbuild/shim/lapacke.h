/* Self-written prototype shim so the reference PHI sources compile without a
 * LAPACKE installation.  Only declarations live here; the matching symbols are
 * defined in lapack_stubs.c and abort if called.  None of them is reached by
 * the in-scope paths (static Hamiltonian, untruncated Hilbert space). */
#ifndef PHI_ORACLE_SHIM_LAPACKE_H_
#define PHI_ORACLE_SHIM_LAPACKE_H_
#include <complex>
typedef int lapack_int;
extern "C" {
double dlamch_(char *cmach);
void zheevr_(char *jobz, char *range, char *uplo, lapack_int *n,
             std::complex<double> *a, lapack_int *lda, double *vl, double *vu,
             lapack_int *il, lapack_int *iu, double *abstol, lapack_int *m,
             double *w, std::complex<double> *z, lapack_int *ldz,
             lapack_int *isuppz, std::complex<double> *work, lapack_int *lwork,
             double *rwork, lapack_int *lrwork, lapack_int *iwork,
             lapack_int *liwork, lapack_int *info);
void dpttrf_(lapack_int *n, double *d, double *e, lapack_int *info);
void dpttrs_(lapack_int *n, lapack_int *nrhs, double *d, double *e, double *b,
             lapack_int *ldb, lapack_int *info);
}
#endif
