// phi/numeric_types.h -- PHI's numeric type names, for code written against
// the reference's headers (numeric_types.h, and SetElementsToZero of
// complex_matrix.h:24-25, which the reference's hierarchy_integrator.h brings
// in).  The double-precision build only: PHI's SINGLEPRECISION build does
// not compile.
#ifndef PHI_B200_NUMERIC_TYPES_H_
#define PHI_B200_NUMERIC_TYPES_H_

#include <complex>

typedef double Float;
typedef std::complex<double> Complex;
typedef int phi_size_t;
typedef int phi_big_size_t;

const Complex kOne(1.0, 0.0);
const Complex kZero(0.0, 0.0);
const Complex kTwo(2.0, 0.0);
const Complex kNegativeOne(-1.0, 0.0);
const Complex kImaginary(0.0, 1.0);
const Complex kNegativeImaginary(0.0, -1.0);
const Float kZerof(0.0);

inline void SetElementsToZero(const phi_big_size_t size, Complex *matrix) {
  for (phi_big_size_t i = 0; i < size; ++i) matrix[i] = kZero;
}
inline void SetElementsToZero(const phi_big_size_t size, Float *matrix) {
  for (phi_big_size_t i = 0; i < size; ++i) matrix[i] = kZerof;
}

#endif  // PHI_B200_NUMERIC_TYPES_H_
