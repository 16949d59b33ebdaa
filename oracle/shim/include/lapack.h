#pragma once
// Project-written LAPACK declarations for the oracle build of the reference:
// the Fortran potrf entry points of scipy's bundled OpenBLAS ("scipy_"
// prefix), forwarded under the names the reference's LAPACK wrappers call.
#define LAPACK_H
#include <complex>
typedef int lapack_int;
typedef std::complex<float>  lapack_complex_float;
typedef std::complex<double> lapack_complex_double;
extern "C" {
void scipy_dpotrf_(const char* uplo, const lapack_int* n, double* A, const lapack_int* lda, lapack_int* info, unsigned long uplo_len);
void scipy_spotrf_(const char* uplo, const lapack_int* n, float*  A, const lapack_int* lda, lapack_int* info, unsigned long uplo_len);
}
inline void dpotrf_(const char* uplo, const lapack_int* n, double* A, const lapack_int* lda, lapack_int* info)
{ scipy_dpotrf_(uplo, n, A, lda, info, 1); }
inline void spotrf_(const char* uplo, const lapack_int* n, float* A, const lapack_int* lda, lapack_int* info)
{ scipy_spotrf_(uplo, n, A, lda, info, 1); }
