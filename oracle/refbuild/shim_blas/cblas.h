/* Self-written CBLAS prototype shim (names and argument order of the public
 * CBLAS interface) for the BLAS-mode build of the reference, linked against
 * an OpenBLAS shared library that exports these symbols.  Declarations only. */
#ifndef PHI_ORACLE_SHIM_CBLAS_H_
#define PHI_ORACLE_SHIM_CBLAS_H_
extern "C" {
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
#define PHI_CBLAS_PAIR(p, T)                                                                              \
  void cblas_##p##gemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int, int,       \
                       const void *, const void *, int, const void *, int, const void *, void *, int);    \
  void cblas_##p##hemm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, int, int, const void *,        \
                       const void *, int, const void *, int, const void *, void *, int);                  \
  void cblas_##p##symm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, int, int, const void *,        \
                       const void *, int, const void *, int, const void *, void *, int);                  \
  void cblas_##p##gemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, const void *, const void *, int, \
                       const void *, int, const void *, void *, int);                                     \
  void cblas_##p##her(enum CBLAS_ORDER, enum CBLAS_UPLO, int, T, const void *, int, void *, int);          \
  void cblas_##p##gerc(enum CBLAS_ORDER, int, int, const void *, const void *, int, const void *, int,    \
                       void *, int);                                                                      \
  void cblas_##p##copy(int, const void *, int, void *, int);                                              \
  void cblas_##p##axpy(int, const void *, const void *, int, void *, int);                                \
  void cblas_##p##dotc_sub(int, const void *, int, const void *, int, void *);                            \
  void cblas_##p##dotu_sub(int, const void *, int, const void *, int, void *);                            \
  void cblas_##p##scal(int, const void *, void *, int);
PHI_CBLAS_PAIR(c, float)
PHI_CBLAS_PAIR(z, double)
#undef PHI_CBLAS_PAIR
}
#endif
