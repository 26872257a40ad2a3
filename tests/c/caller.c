/* A C program written against include/xkblas.h the way the reference's
 * test programs call XKBlas (testing/ztesting_gemm.c:157-163: _async,
 * memory_coherent_async, sync, invalidate_caches), linked with
 * libxkblas.so.  It checks, on any machine: the header helpers, the -i
 * argument codes of the level-3 entry points, and that a valid call without
 * a usable GPU fails with ENODEV (no CPU path).  With a GPU it checks the
 * product instead.  Exit status 0 on success; prints the failed check. */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "xkblas.h"

#define CHECK(c)                                             \
  do {                                                       \
    if (!(c)) {                                              \
      fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                              \
    }                                                        \
  } while (0)

int main(int argc, char** argv) {
  const int want_gpu = argc > 1 && argv[1][0] == 'g';
  /* header helpers (Fortran characters -> CBLAS values) */
  CHECK(xkblas_blas2cblas_trans("n") == CblasNoTrans);
  CHECK(xkblas_blas2cblas_trans("T") == CblasTrans);
  CHECK(xkblas_blas2cblas_trans("conj") == CblasConjTrans);
  CHECK(xkblas_blas2cblas_side("R") == CblasRight);
  CHECK(xkblas_blas2cblas_fill("l") == CblasLower);
  CHECK(xkblas_blas2cblas_diag("U") == CblasUnit);
  CHECK(xkblas_blas2cblas_trans("x") == -1);

  enum { M = 64, N = 48, K = 40 };
  double* A = (double*)malloc(sizeof(double) * M * K);
  double* B = (double*)malloc(sizeof(double) * K * N);
  double* C = (double*)malloc(sizeof(double) * M * N);
  for (int i = 0; i < M * K; ++i) A[i] = (double)((i * 7) % 11) - 5.0;
  for (int i = 0; i < K * N; ++i) B[i] = (double)((i * 5) % 13) - 6.0;
  for (int i = 0; i < M * N; ++i) C[i] = 1.0;
  const double alpha = 2.0, beta = -1.0;
  const int ta = xkblas_blas2cblas_trans("N"), tb = xkblas_blas2cblas_trans("N");

  /* argument codes (reference blas/zgemm.c:132-181) */
  CHECK(xkblas_dgemm_async(-1, tb, M, N, K, &alpha, A, M, B, K, &beta, C, M) == -1);
  CHECK(xkblas_dgemm_async(ta, 7, M, N, K, &alpha, A, M, B, K, &beta, C, M) == -2);
  CHECK(xkblas_dgemm_async(ta, tb, -1, N, K, &alpha, A, M, B, K, &beta, C, M) == -3);
  CHECK(xkblas_dgemm_async(ta, tb, M, N, K, &alpha, A, M - 1, B, K, &beta, C, M) == -8);
  CHECK(xkblas_dgemm_async(ta, tb, M, N, K, &alpha, A, M, B, K, &beta, C, M - 1) == -13);
  CHECK(xkblas_dtrsm_async(xkblas_blas2cblas_side("x"), CblasLower, CblasNoTrans, CblasNonUnit,
                           M, N, &alpha, A, M, C, M) == -1);

  const int ir = xkblas_init();
  const int r = xkblas_dgemm_async(ta, tb, M, N, K, &alpha, A, M, B, K, &beta, C, M);
  if (!want_gpu) {
    CHECK(ir != 0);
    CHECK(r == ENODEV);
    CHECK(C[0] == 1.0);
  } else {
    CHECK(ir == 0 && r == 0);
    CHECK(xkblas_memory_coherent_async(0, 0, M, N, C, M, sizeof(double)) == 0);
    CHECK(xkblas_sync() == 0);
    CHECK(xkblas_memory_invalidate_caches() == 0);
    /* integer-valued products are exact in FP64 */
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < M; ++i) {
        double s = 0.0;
        for (int k = 0; k < K; ++k) s += A[i + k * M] * B[k + j * K];
        CHECK(C[i + j * M] == alpha * s + beta);
      }
    CHECK(xkblas_finalize() == 0);
  }
  free(A);
  free(B);
  free(C);
  printf("caller ok\n");
  return 0;
}
