#pragma once
// Project-written CBLAS declarations for the oracle build of the reference.
// The only BLAS in this image is the OpenBLAS that scipy bundles, whose C
// entry points carry a "scipy_" prefix; the cblas_* names the reference's
// BLAS wrappers call are forwarded to those exports here.  Declarations
// follow the public CBLAS interface (netlib cblas.h).
#define CBLAS_H
typedef int blasint;
typedef enum CBLAS_ORDER     { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113, CblasConjNoTrans = 114 } CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO      { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG      { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum CBLAS_SIDE      { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;
typedef CBLAS_ORDER CBLAS_LAYOUT;

extern "C" {
#define TB_DECL_REAL(T, P) \
void scipy_cblas_##P##syrk(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, blasint, blasint, T, const T*, blasint, T, T*, blasint); \
void scipy_cblas_##P##trsm(CBLAS_ORDER, CBLAS_SIDE, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, blasint, blasint, T, const T*, blasint, T*, blasint); \
void scipy_cblas_##P##trsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, blasint, const T*, blasint, T*, blasint); \
void scipy_cblas_##P##gemv(CBLAS_ORDER, CBLAS_TRANSPOSE, blasint, blasint, T, const T*, blasint, const T*, blasint, T, T*, blasint); \
void scipy_cblas_##P##gemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, blasint, blasint, blasint, T, const T*, blasint, const T*, blasint, T, T*, blasint); \
void scipy_cblas_##P##ger(CBLAS_ORDER, blasint, blasint, T, const T*, blasint, const T*, blasint, T*, blasint); \
void scipy_cblas_##P##scal(blasint, T, T*, blasint); \
void scipy_cblas_##P##axpy(blasint, T, const T*, blasint, T*, blasint); \
T    scipy_cblas_##P##dot(blasint, const T*, blasint, const T*, blasint); \
void scipy_cblas_##P##copy(blasint, const T*, blasint, T*, blasint);
TB_DECL_REAL(double, d)
TB_DECL_REAL(float, s)
#undef TB_DECL_REAL
void scipy_openblas_set_num_threads(int);
int  scipy_openblas_get_num_threads(void);
}

#define TB_FWD_REAL(T, P) \
inline void cblas_##P##syrk(CBLAS_ORDER o, CBLAS_UPLO u, CBLAS_TRANSPOSE t, blasint n, blasint k, T a, const T* A, blasint lda, T b, T* C, blasint ldc) \
{ scipy_cblas_##P##syrk(o,u,t,n,k,a,A,lda,b,C,ldc); } \
inline void cblas_##P##trsm(CBLAS_ORDER o, CBLAS_SIDE s, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, blasint m, blasint n, T a, const T* A, blasint lda, T* B, blasint ldb) \
{ scipy_cblas_##P##trsm(o,s,u,t,d,m,n,a,A,lda,B,ldb); } \
inline void cblas_##P##trsv(CBLAS_ORDER o, CBLAS_UPLO u, CBLAS_TRANSPOSE t, CBLAS_DIAG d, blasint n, const T* A, blasint lda, T* x, blasint incx) \
{ scipy_cblas_##P##trsv(o,u,t,d,n,A,lda,x,incx); } \
inline void cblas_##P##gemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, blasint m, blasint n, T a, const T* A, blasint lda, const T* x, blasint incx, T b, T* y, blasint incy) \
{ scipy_cblas_##P##gemv(o,t,m,n,a,A,lda,x,incx,b,y,incy); } \
inline void cblas_##P##gemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, blasint m, blasint n, blasint k, T a, const T* A, blasint lda, const T* B, blasint ldb, T b, T* C, blasint ldc) \
{ scipy_cblas_##P##gemm(o,ta,tb,m,n,k,a,A,lda,B,ldb,b,C,ldc); } \
inline void cblas_##P##ger(CBLAS_ORDER o, blasint m, blasint n, T a, const T* x, blasint incx, const T* y, blasint incy, T* A, blasint lda) \
{ scipy_cblas_##P##ger(o,m,n,a,x,incx,y,incy,A,lda); } \
inline void cblas_##P##scal(blasint n, T a, T* x, blasint incx) { scipy_cblas_##P##scal(n,a,x,incx); } \
inline void cblas_##P##axpy(blasint n, T a, const T* x, blasint incx, T* y, blasint incy) { scipy_cblas_##P##axpy(n,a,x,incx,y,incy); } \
inline T    cblas_##P##dot(blasint n, const T* x, blasint incx, const T* y, blasint incy) { return scipy_cblas_##P##dot(n,x,incx,y,incy); } \
inline void cblas_##P##copy(blasint n, const T* x, blasint incx, T* y, blasint incy) { scipy_cblas_##P##copy(n,x,incx,y,incy); }
TB_FWD_REAL(double, d)
TB_FWD_REAL(float, s)
#undef TB_FWD_REAL
