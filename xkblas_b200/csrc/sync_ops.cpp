// sync_ops.cpp -- the synchronous forms xkblas_?xxx_sync: the _async call,
// memory_coherent_async on its output (the written triangle for the
// triangle-producing ops), xkblas_sync, xkblas_memory_invalidate_caches.
// That is the sequence the reference's F77 wrapper runs for every BLAS call
// (blas/zlibxkblas_wrapper.c:67-73), offered here as C entry points; the F77
// names themselves live in libxkblas_blas.so (f77/xkblas_f77.cpp).  Unlike
// that wrapper there is no CPU branch below an arithmetic-intensity
// threshold: every call runs on the GPU.
#include "xkblas.h"

namespace {

// rc: the _async result; on success make the output coherent and wait
int finish(int rc, int uplo, size_t M, size_t N, void* C, size_t ld, size_t es) {
  if (rc != 0) return rc;
  rc = xkblas_memory_coherent_async(uplo, 0, M, N, C, ld, es);
  const int rs = xkblas_sync();
  xkblas_memory_invalidate_caches();
  return rc ? rc : rs;
}

}  // namespace

#define XKB_DEFINE_SYNC_OPS(p, T, R)                                                            \
  extern "C" int xkblas_##p##gemm_sync(int tA, int tB, int M, int N, int K, const T* al,        \
                                       const T* A, int lda, const T* B, int ldb, const T* be,   \
                                       T* C, int ldc) {                                         \
    return finish(xkblas_##p##gemm_async(tA, tB, M, N, K, al, A, lda, B, ldb, be, C, ldc), 0,   \
                  M, N, C, ldc, sizeof(T));                                                     \
  }                                                                                             \
  extern "C" int xkblas_##p##gemmt_sync(int ul, int tA, int tB, int N, int K, const T* al,      \
                                        const T* A, int lda, const T* B, int ldb, const T* be,  \
                                        T* C, int ldc) {                                        \
    return finish(xkblas_##p##gemmt_async(ul, tA, tB, N, K, al, A, lda, B, ldb, be, C, ldc),   \
                  ul, N, N, C, ldc, sizeof(T));                                                 \
  }                                                                                             \
  extern "C" int xkblas_##p##trsm_sync(int sd, int ul, int tA, int dg, int M, int N,            \
                                       const T* al, const T* A, int lda, T* B, int ldb) {       \
    return finish(xkblas_##p##trsm_async(sd, ul, tA, dg, M, N, al, A, lda, B, ldb), 0, M, N, B, \
                  ldb, sizeof(T));                                                              \
  }                                                                                             \
  extern "C" int xkblas_##p##trmm_sync(int sd, int ul, int tA, int dg, int M, int N,            \
                                       const T* al, const T* A, int lda, T* B, int ldb) {       \
    return finish(xkblas_##p##trmm_async(sd, ul, tA, dg, M, N, al, A, lda, B, ldb), 0, M, N, B, \
                  ldb, sizeof(T));                                                              \
  }                                                                                             \
  extern "C" int xkblas_##p##symm_sync(int sd, int ul, int M, int N, const T* al, const T* A,   \
                                       int lda, const T* B, int ldb, const T* be, T* C,         \
                                       int ldc) {                                               \
    return finish(xkblas_##p##symm_async(sd, ul, M, N, al, A, lda, B, ldb, be, C, ldc), 0, M,   \
                  N, C, ldc, sizeof(T));                                                        \
  }                                                                                             \
  extern "C" int xkblas_##p##syrk_sync(int ul, int tr, int N, int K, const T* al, const T* A,   \
                                       int lda, const T* be, T* C, int ldc) {                   \
    return finish(xkblas_##p##syrk_async(ul, tr, N, K, al, A, lda, be, C, ldc), ul, N, N, C,    \
                  ldc, sizeof(T));                                                              \
  }                                                                                             \
  extern "C" int xkblas_##p##syr2k_sync(int ul, int tr, int N, int K, const T* al, const T* A,  \
                                        int lda, const T* B, int ldb, const T* be, T* C,        \
                                        int ldc) {                                              \
    return finish(xkblas_##p##syr2k_async(ul, tr, N, K, al, A, lda, B, ldb, be, C, ldc), ul, N, \
                  N, C, ldc, sizeof(T));                                                        \
  }

#define XKB_DEFINE_HE_SYNC_OPS(p, T, R)                                                         \
  extern "C" int xkblas_##p##hemm_sync(int sd, int ul, int M, int N, const T* al, const T* A,   \
                                       int lda, const T* B, int ldb, const T* be, T* C,         \
                                       int ldc) {                                               \
    return finish(xkblas_##p##hemm_async(sd, ul, M, N, al, A, lda, B, ldb, be, C, ldc), 0, M,   \
                  N, C, ldc, sizeof(T));                                                        \
  }                                                                                             \
  extern "C" int xkblas_##p##herk_sync(int ul, int tr, int N, int K, const R* al, const T* A,   \
                                       int lda, const R* be, T* C, int ldc) {                   \
    return finish(xkblas_##p##herk_async(ul, tr, N, K, al, A, lda, be, C, ldc), ul, N, N, C,    \
                  ldc, sizeof(T));                                                              \
  }                                                                                             \
  extern "C" int xkblas_##p##her2k_sync(int ul, int tr, int N, int K, const T* al, const T* A,  \
                                        int lda, const T* B, int ldb, const R* be, T* C,        \
                                        int ldc) {                                              \
    return finish(xkblas_##p##her2k_async(ul, tr, N, K, al, A, lda, B, ldb, be, C, ldc), ul, N, \
                  N, C, ldc, sizeof(T));                                                        \
  }

XKB_DEFINE_SYNC_OPS(s, float, float)
XKB_DEFINE_SYNC_OPS(d, double, double)
XKB_DEFINE_SYNC_OPS(c, Complex32_t, float)
XKB_DEFINE_SYNC_OPS(z, Complex64_t, double)
XKB_DEFINE_HE_SYNC_OPS(c, Complex32_t, float)
XKB_DEFINE_HE_SYNC_OPS(z, Complex64_t, double)
