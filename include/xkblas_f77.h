/* xkblas_f77.h -- the Fortran-77 BLAS level-3 names exported by
 * libxkblas_blas.so, the drop-in BLAS replacement (reference
 * blas/zlibxkblas_wrapper.c:46-392, blas/xkblas_f77.h).  Standard BLAS
 * calling convention: every argument by reference, option characters as
 * CHARACTER*1 (hidden length arguments, appended by Fortran compilers, are
 * not read).  Each call runs on the GPU through the synchronous form
 * xkblas_?xxx_sync (xkblas.h): on return the output is in host memory and
 * the library holds no device copy.  An invalid argument is reported on
 * stderr in the XERBLA format and the call returns without computing. */
#ifndef XKBLAS_F77_H
#define XKBLAS_F77_H
#include "xkblas.h"
#ifdef __cplusplus
extern "C" {
#endif

#define XKBLAS_DECL_F77(p, T, R)                                                    \
  void p##gemm_(const char* transa, const char* transb, const int* m, const int* n, \
                const int* k, const T* alpha, const T* A, const int* lda,           \
                const T* B, const int* ldb, const T* beta, T* C, const int* ldc);   \
  void p##gemmt_(const char* uplo, const char* transa, const char* transb,          \
                 const int* n, const int* k, const T* alpha, const T* A,            \
                 const int* lda, const T* B, const int* ldb, const T* beta, T* C,   \
                 const int* ldc);                                                   \
  void p##trsm_(const char* side, const char* uplo, const char* transa,             \
                const char* diag, const int* m, const int* n, const T* alpha,       \
                const T* A, const int* lda, T* B, const int* ldb);                  \
  void p##trmm_(const char* side, const char* uplo, const char* transa,             \
                const char* diag, const int* m, const int* n, const T* alpha,       \
                const T* A, const int* lda, T* B, const int* ldb);                  \
  void p##symm_(const char* side, const char* uplo, const int* m, const int* n,     \
                const T* alpha, const T* A, const int* lda, const T* B,             \
                const int* ldb, const T* beta, T* C, const int* ldc);               \
  void p##syrk_(const char* uplo, const char* trans, const int* n, const int* k,    \
                const T* alpha, const T* A, const int* lda, const T* beta, T* C,    \
                const int* ldc);                                                    \
  void p##syr2k_(const char* uplo, const char* trans, const int* n, const int* k,   \
                 const T* alpha, const T* A, const int* lda, const T* B,            \
                 const int* ldb, const T* beta, T* C, const int* ldc);
#define XKBLAS_DECL_F77_HE(p, T, R)                                                 \
  void p##hemm_(const char* side, const char* uplo, const int* m, const int* n,     \
                const T* alpha, const T* A, const int* lda, const T* B,             \
                const int* ldb, const T* beta, T* C, const int* ldc);               \
  void p##herk_(const char* uplo, const char* trans, const int* n, const int* k,    \
                const R* alpha, const T* A, const int* lda, const R* beta, T* C,    \
                const int* ldc);                                                    \
  void p##her2k_(const char* uplo, const char* trans, const int* n, const int* k,   \
                 const T* alpha, const T* A, const int* lda, const T* B,            \
                 const int* ldb, const R* beta, T* C, const int* ldc);

XKBLAS_DECL_F77(s, float, float)
XKBLAS_DECL_F77(d, double, double)
XKBLAS_DECL_F77(c, Complex32_t, float)
XKBLAS_DECL_F77(z, Complex64_t, double)
XKBLAS_DECL_F77_HE(c, Complex32_t, float)
XKBLAS_DECL_F77_HE(z, Complex64_t, double)

#ifdef __cplusplus
}
#endif
#endif
