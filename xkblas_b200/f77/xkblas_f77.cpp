// xkblas_f77.cpp -- libxkblas_blas.so: the Fortran-77 BLAS level-3 names
// (sgemm_ ... zher2k_) as a drop-in replacement BLAS, replacing the
// reference's wrapper library (blas/zlibxkblas_wrapper.c:46-392,
// blas/libxkblas_wrapper.c:88-170).  Each routine maps its option
// characters to the CBLAS codes (reference blas/xkblas.h:143-200) and calls
// the synchronous form xkblas_?xxx_sync of libxkblas.so (async call,
// coherence of the output, sync, cache release: the wrapper's sequence).
// The reference wrapper sends calls whose flops/data ratio is below
// XKBLAS_THRESHOLD[_<KERNEL>] to the CPU BLAS; this library has no CPU
// branch: every call runs on the GPU (the threshold variables are ignored).
// Argument errors are reported XERBLA-style on stderr and the call returns.
#include "xkblas_f77.h"

#include <cstdio>

namespace {

int trans_code(const char* c) {
  switch (c ? c[0] : 0) {
    case 'N': case 'n': return CblasNoTrans;
    case 'T': case 't': return CblasTrans;
    case 'C': case 'c': return CblasConjTrans;
  }
  return 0;  // rejected by the callee with its -i code
}
int uplo_code(const char* c) {
  switch (c ? c[0] : 0) {
    case 'U': case 'u': return CblasUpper;
    case 'L': case 'l': return CblasLower;
  }
  return 0;
}
int side_code(const char* c) {
  switch (c ? c[0] : 0) {
    case 'L': case 'l': return CblasLeft;
    case 'R': case 'r': return CblasRight;
  }
  return 0;
}
int diag_code(const char* c) {
  switch (c ? c[0] : 0) {
    case 'N': case 'n': return CblasNonUnit;
    case 'U': case 'u': return CblasUnit;
  }
  return 0;
}

void report(const char* name, int rc) {
  if (rc < 0)
    std::fprintf(stderr, " ** On entry to %s parameter number %d had an illegal value\n", name,
                 -rc);
  else if (rc > 0)
    std::fprintf(stderr, " ** %s: libxkblas runtime error %d\n", name, rc);
}

}  // namespace

#define XKB_F77(p, P, T, R)                                                                    \
  extern "C" void p##gemm_(const char* ta, const char* tb, const int* m, const int* n,         \
                           const int* k, const T* al, const T* A, const int* lda, const T* B,  \
                           const int* ldb, const T* be, T* C, const int* ldc) {                \
    report(#P "GEMM", xkblas_##p##gemm_sync(trans_code(ta), trans_code(tb), *m, *n, *k, al, A, \
                                            *lda, B, *ldb, be, C, *ldc));                      \
  }                                                                                            \
  extern "C" void p##gemmt_(const char* ul, const char* ta, const char* tb, const int* n,      \
                            const int* k, const T* al, const T* A, const int* lda,             \
                            const T* B, const int* ldb, const T* be, T* C, const int* ldc) {   \
    report(#P "GEMMT", xkblas_##p##gemmt_sync(uplo_code(ul), trans_code(ta), trans_code(tb),   \
                                              *n, *k, al, A, *lda, B, *ldb, be, C, *ldc));     \
  }                                                                                            \
  extern "C" void p##trsm_(const char* sd, const char* ul, const char* ta, const char* dg,     \
                           const int* m, const int* n, const T* al, const T* A,                \
                           const int* lda, T* B, const int* ldb) {                             \
    report(#P "TRSM", xkblas_##p##trsm_sync(side_code(sd), uplo_code(ul), trans_code(ta),      \
                                            diag_code(dg), *m, *n, al, A, *lda, B, *ldb));     \
  }                                                                                            \
  extern "C" void p##trmm_(const char* sd, const char* ul, const char* ta, const char* dg,     \
                           const int* m, const int* n, const T* al, const T* A,                \
                           const int* lda, T* B, const int* ldb) {                             \
    report(#P "TRMM", xkblas_##p##trmm_sync(side_code(sd), uplo_code(ul), trans_code(ta),      \
                                            diag_code(dg), *m, *n, al, A, *lda, B, *ldb));     \
  }                                                                                            \
  extern "C" void p##symm_(const char* sd, const char* ul, const int* m, const int* n,         \
                           const T* al, const T* A, const int* lda, const T* B,                \
                           const int* ldb, const T* be, T* C, const int* ldc) {                \
    report(#P "SYMM", xkblas_##p##symm_sync(side_code(sd), uplo_code(ul), *m, *n, al, A, *lda, \
                                            B, *ldb, be, C, *ldc));                            \
  }                                                                                            \
  extern "C" void p##syrk_(const char* ul, const char* tr, const int* n, const int* k,         \
                           const T* al, const T* A, const int* lda, const T* be, T* C,         \
                           const int* ldc) {                                                   \
    report(#P "SYRK", xkblas_##p##syrk_sync(uplo_code(ul), trans_code(tr), *n, *k, al, A,      \
                                            *lda, be, C, *ldc));                               \
  }                                                                                            \
  extern "C" void p##syr2k_(const char* ul, const char* tr, const int* n, const int* k,        \
                            const T* al, const T* A, const int* lda, const T* B,               \
                            const int* ldb, const T* be, T* C, const int* ldc) {               \
    report(#P "SYR2K", xkblas_##p##syr2k_sync(uplo_code(ul), trans_code(tr), *n, *k, al, A,    \
                                              *lda, B, *ldb, be, C, *ldc));                    \
  }

#define XKB_F77_HE(p, P, T, R)                                                                 \
  extern "C" void p##hemm_(const char* sd, const char* ul, const int* m, const int* n,         \
                           const T* al, const T* A, const int* lda, const T* B,                \
                           const int* ldb, const T* be, T* C, const int* ldc) {                \
    report(#P "HEMM", xkblas_##p##hemm_sync(side_code(sd), uplo_code(ul), *m, *n, al, A, *lda, \
                                            B, *ldb, be, C, *ldc));                            \
  }                                                                                            \
  extern "C" void p##herk_(const char* ul, const char* tr, const int* n, const int* k,         \
                           const R* al, const T* A, const int* lda, const R* be, T* C,         \
                           const int* ldc) {                                                   \
    report(#P "HERK", xkblas_##p##herk_sync(uplo_code(ul), trans_code(tr), *n, *k, al, A,      \
                                            *lda, be, C, *ldc));                               \
  }                                                                                            \
  extern "C" void p##her2k_(const char* ul, const char* tr, const int* n, const int* k,        \
                            const T* al, const T* A, const int* lda, const T* B,               \
                            const int* ldb, const R* be, T* C, const int* ldc) {               \
    report(#P "HER2K", xkblas_##p##her2k_sync(uplo_code(ul), trans_code(tr), *n, *k, al, A,    \
                                              *lda, B, *ldb, be, C, *ldc));                    \
  }

XKB_F77(s, S, float, float)
XKB_F77(d, D, double, double)
XKB_F77(c, C, Complex32_t, float)
XKB_F77(z, Z, Complex64_t, double)
XKB_F77_HE(c, C, Complex32_t, float)
XKB_F77_HE(z, Z, Complex64_t, double)
