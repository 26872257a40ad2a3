/*
 * Precision template for the CPU oracle (included by xkb_oracle.c once per
 * precision with OT = element type, OR = real type, OP(x) = name prefix,
 * OCPLX = 0/1).  TEST INFRASTRUCTURE ONLY: nothing in the library links it.
 *
 * Each tiled driver restates the loop nest of the reference driver named in
 * its comment (path:line in the XKBlas tree): the matrix is cut into NB x NB
 * tiles and the same tile tasks run in the same order, each tile task being
 * the plain BLAS definition that the reference hands to cuBLAS / CPU BLAS.
 */

/* ---- element access ----------------------------------------------------- */
static inline OT OP(opel)(int trans, const OT* A, long lda, long i, long p) {
  /* element (i,p) of op(A) */
  if (trans == XKO_NOTRANS) return A[i + p * lda];
  OT v = A[p + i * lda];
  return trans == XKO_CONJTRANS ? OCONJ(v) : v;
}

/* ---- tile bodies: plain BLAS definitions --------------------------------- */

/* C(m,n) = alpha*op(A)*op(B) + beta*C; uplo != 0 restricts the update to one
 * triangle of C (the BLAS gemmt contract).  Reference tile body:
 * blas/ztask_gemm.c:161-216 (CPU: zgemm_, GPU: cublasZgemm). */
static void OP(tile_gemm)(int uplo, int ta, int tb, long m, long n, long k,
                          OT alpha, const OT* A, long lda, const OT* B, long ldb,
                          OT beta, OT* C, long ldc, long ioff, long joff) {
  for (long j = 0; j < n; j++) {
    for (long i = 0; i < m; i++) {
      long gi = i + ioff, gj = j + joff;
      if (uplo == XKO_LOWER && gi < gj) continue;
      if (uplo == XKO_UPPER && gi > gj) continue;
      OT acc = 0;
      if (alpha != (OT)0)
        for (long p = 0; p < k; p++)
          acc += OP(opel)(ta, A, lda, i, p) * OP(opel)(tb, B, ldb, p, j);
      OT c = (beta == (OT)0) ? (OT)0 : beta * C[i + j * ldc];
      C[i + j * ldc] = alpha * acc + c;
    }
  }
}

/* B <- alpha * op(A)^-1 * B (side L) or alpha * B * op(A)^-1 (side R);
 * reference tile body blas/ztask_trsm.c:144-180 (dtrsm_ / cublasZtrsm). */
static void OP(tile_trsm)(int side, int uplo, int trans, int diag, long m,
                          long n, OT alpha, const OT* A, long lda, OT* B,
                          long ldb) {
  /* op(A) is lower triangular iff (uplo==L) xor (trans!=N) */
  int lower = (uplo == XKO_LOWER) ^ (trans != XKO_NOTRANS);
  if (side == XKO_LEFT) {
    for (long j = 0; j < n; j++) {
      OT* b = B + j * ldb;
      for (long i = 0; i < m; i++) b[i] *= alpha;
      if (lower) {
        for (long i = 0; i < m; i++) {
          OT s = b[i];
          for (long p = 0; p < i; p++) s -= OP(opel)(trans, A, lda, i, p) * b[p];
          b[i] = (diag == XKO_UNIT) ? s : s / OP(opel)(trans, A, lda, i, i);
        }
      } else {
        for (long i = m - 1; i >= 0; i--) {
          OT s = b[i];
          for (long p = i + 1; p < m; p++) s -= OP(opel)(trans, A, lda, i, p) * b[p];
          b[i] = (diag == XKO_UNIT) ? s : s / OP(opel)(trans, A, lda, i, i);
        }
      }
    }
  } else {
    /* X * op(A) = alpha*B, op(A) n x n */
    for (long i = 0; i < m; i++) {
      for (long j = 0; j < n; j++) B[i + j * ldb] *= alpha;
      if (!lower) {           /* upper: solve columns left to right */
        for (long j = 0; j < n; j++) {
          OT s = B[i + j * ldb];
          for (long p = 0; p < j; p++) s -= B[i + p * ldb] * OP(opel)(trans, A, lda, p, j);
          B[i + j * ldb] = (diag == XKO_UNIT) ? s : s / OP(opel)(trans, A, lda, j, j);
        }
      } else {                /* lower: right to left */
        for (long j = n - 1; j >= 0; j--) {
          OT s = B[i + j * ldb];
          for (long p = j + 1; p < n; p++) s -= B[i + p * ldb] * OP(opel)(trans, A, lda, p, j);
          B[i + j * ldb] = (diag == XKO_UNIT) ? s : s / OP(opel)(trans, A, lda, j, j);
        }
      }
    }
  }
}

/* one triangle of C <- alpha*op(A)*op(A)^T + beta*C  (herk: ^H, real scalars,
 * real diagonal).  Reference tile bodies blas/ztask_syrk.c:126-136,
 * blas/ztask_herk.c:126-136. */
static void OP(tile_syrk)(int herm, int uplo, int trans, long n, long k,
                          OT alpha, const OT* A, long lda, OT beta, OT* C,
                          long ldc) {
  for (long j = 0; j < n; j++) {
    long i0 = (uplo == XKO_LOWER) ? j : 0, i1 = (uplo == XKO_LOWER) ? n : j + 1;
    for (long i = i0; i < i1; i++) {
      OT acc = 0;
      for (long p = 0; p < k; p++) {
        OT a, b;
        if (trans == XKO_NOTRANS) {         /* A(i,p) * A(j,p) [conj for herk] */
          a = A[i + p * lda];
          b = herm ? OCONJ(A[j + p * lda]) : A[j + p * lda];
        } else {                            /* A(p,i) [conj for herk] * A(p,j) */
          a = herm ? OCONJ(A[p + i * lda]) : A[p + i * lda];
          b = A[p + j * lda];
        }
        acc += a * b;
      }
      OT c = (beta == (OT)0) ? (OT)0 : beta * C[i + j * ldc];
      OT r = alpha * acc + c;
#if OCPLX
      if (herm && i == j) r = OREAL(r);
#endif
      C[i + j * ldc] = r;
    }
  }
}

/* ---- drivers -------------------------------------------------------------- */

static long OP(ntiles)(long n, long nb) { return n <= 0 ? 0 : (n + nb - 1) / nb; }
static long OP(tsz)(long i, long nt, long n, long nb) { return i == nt - 1 ? n - i * nb : nb; }

/* Tile GEMM: blas/zgemm.c:279-367.  beta is applied on the first k tile only
 * (zgemm.c:298); the C tiles are independent so they run in parallel. */
void OP(xko_gemm)(int ta, int tb, int M, int N, int K, const OT* palpha,
                  const OT* A, int lda, const OT* B, int ldb, const OT* pbeta,
                  OT* C, int ldc, int NB) {
  OT alpha = *palpha, beta = *pbeta;
  if (M == 0 || N == 0) return;
  long mt = OP(ntiles)(M, NB), nt = OP(ntiles)(N, NB), kt = OP(ntiles)(K, NB);
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (long m = 0; m < mt; m++)
    for (long n = 0; n < nt; n++) {
      long mm = OP(tsz)(m, mt, M, NB), nn = OP(tsz)(n, nt, N, NB);
      OT* Ct = C + m * NB + n * NB * (long)ldc;
      if (kt == 0) {  /* K == 0: C = beta*C */
        OP(tile_gemm)(0, ta, tb, mm, nn, 0, alpha, A, lda, B, ldb, beta, Ct, ldc, 0, 0);
        continue;
      }
      for (long k = 0; k < kt; k++) {
        long kk = OP(tsz)(k, kt, K, NB);
        const OT* At = (ta == XKO_NOTRANS) ? A + m * NB + k * NB * (long)lda
                                           : A + k * NB + m * NB * (long)lda;
        const OT* Bt = (tb == XKO_NOTRANS) ? B + k * NB + n * NB * (long)ldb
                                           : B + n * NB + k * NB * (long)ldb;
        OP(tile_gemm)(0, ta, tb, mm, nn, kk, alpha, At, lda, Bt, ldb,
                      k == 0 ? beta : (OT)1, Ct, ldc, 0, 0);
      }
    }
}

/* Tile GEMMT: blas/zgemmt.c:252-390: C tiles of one triangle, diagonal tiles
 * restricted to the triangle (the reference's GPU body writes the whole
 * diagonal tile, blas/ztask_gemmt.c:213; the BLAS contract is kept here). */
void OP(xko_gemmt)(int uplo, int ta, int tb, int N, int K, const OT* palpha,
                   const OT* A, int lda, const OT* B, int ldb, const OT* pbeta,
                   OT* C, int ldc, int NB) {
  OT alpha = *palpha, beta = *pbeta;
  if (N == 0) return;
  long nt = OP(ntiles)(N, NB), kt = OP(ntiles)(K, NB);
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (long m = 0; m < nt; m++)
    for (long n = 0; n < nt; n++) {
      if (uplo == XKO_LOWER && n > m) continue;
      if (uplo == XKO_UPPER && n < m) continue;
      long mm = OP(tsz)(m, nt, N, NB), nn = OP(tsz)(n, nt, N, NB);
      int tu = (m == n) ? uplo : 0;
      OT* Ct = C + m * NB + n * NB * (long)ldc;
      if (kt == 0) { OP(tile_gemm)(tu, ta, tb, mm, nn, 0, alpha, A, lda, B, ldb, beta, Ct, ldc, 0, 0); continue; }
      for (long k = 0; k < kt; k++) {
        long kk = OP(tsz)(k, kt, K, NB);
        const OT* At = (ta == XKO_NOTRANS) ? A + m * NB + k * NB * (long)lda
                                           : A + k * NB + m * NB * (long)lda;
        const OT* Bt = (tb == XKO_NOTRANS) ? B + k * NB + n * NB * (long)ldb
                                           : B + n * NB + k * NB * (long)ldb;
        OP(tile_gemm)(tu, ta, tb, mm, nn, kk, alpha, At, lda, Bt, ldb,
                      k == 0 ? beta : (OT)1, Ct, ldc, 0, 0);
      }
    }
}

#define OA(i, j) (A + (long)(i) * NB + (long)(j) * NB * (long)lda)
#define OB(i, j) (B + (long)(i) * NB + (long)(j) * NB * (long)ldb)

/* Tile TRSM, all eight side/uplo/trans branches of blas/ztrsm.c:243-499:
 * diagonal solve on tile row/column k with lalpha (alpha on the first step
 * only, ztrsm.c:316), then the trailing GEMM updates with -1 (mzone) and
 * lalpha, or -1/alpha (minvalpha) in the Right/trans branches. */
void OP(xko_trsm)(int side, int uplo, int trans, int diag, int M, int N,
                  const OT* palpha, const OT* A, int lda, OT* B, int ldb,
                  int NB) {
  OT alpha = *palpha, zone = 1, mzone = -1;
  if (M == 0 || N == 0) return;
  long Bmt = OP(ntiles)(M, NB), Bnt = OP(ntiles)(N, NB);
  long Bm = M, Bn = N, Bmb = NB, Bnb = NB;
  if (side == XKO_LEFT) {
    if (uplo == XKO_UPPER) {
      if (trans == XKO_NOTRANS) {                               /* ztrsm.c:241-273 */
        for (long k = 0; k < Bmt; k++) {
          long km = k == 0 ? Bm - (Bmt - 1) * Bmb : Bmb;
          OT la = k == 0 ? alpha : zone;
          long kk = Bmt - 1 - k;
#pragma omp parallel for
          for (long n = 0; n < Bnt; n++)
            OP(tile_trsm)(side, uplo, trans, diag, km, OP(tsz)(n, Bnt, Bn, Bnb), la, OA(kk, kk), lda, OB(kk, n), ldb);
#pragma omp parallel for collapse(2)
          for (long m = k + 1; m < Bmt; m++)
            for (long n = 0; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, Bmb, OP(tsz)(n, Bnt, Bn, Bnb), km, mzone,
                            OA(Bmt - 1 - m, kk), lda, OB(kk, n), ldb, la, OB(Bmt - 1 - m, n), ldb, 0, 0);
        }
      } else {                                                  /* ztrsm.c:275-305 */
        for (long k = 0; k < Bmt; k++) {
          long km = OP(tsz)(k, Bmt, Bm, Bmb);
          OT la = k == 0 ? alpha : zone;
#pragma omp parallel for
          for (long n = 0; n < Bnt; n++)
            OP(tile_trsm)(side, uplo, trans, diag, km, OP(tsz)(n, Bnt, Bn, Bnb), la, OA(k, k), lda, OB(k, n), ldb);
#pragma omp parallel for collapse(2)
          for (long m = k + 1; m < Bmt; m++)
            for (long n = 0; n < Bnt; n++)
              OP(tile_gemm)(0, trans, XKO_NOTRANS, OP(tsz)(m, Bmt, Bm, Bmb), OP(tsz)(n, Bnt, Bn, Bnb), Bmb,
                            mzone, OA(k, m), lda, OB(k, n), ldb, la, OB(m, n), ldb, 0, 0);
        }
      }
    } else {
      if (trans == XKO_NOTRANS) {                               /* ztrsm.c:308-340 */
        for (long k = 0; k < Bmt; k++) {
          long km = OP(tsz)(k, Bmt, Bm, Bmb);
          OT la = k == 0 ? alpha : zone;
#pragma omp parallel for
          for (long n = 0; n < Bnt; n++)
            OP(tile_trsm)(side, uplo, trans, diag, km, OP(tsz)(n, Bnt, Bn, Bnb), la, OA(k, k), lda, OB(k, n), ldb);
#pragma omp parallel for collapse(2)
          for (long m = k + 1; m < Bmt; m++)
            for (long n = 0; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, OP(tsz)(m, Bmt, Bm, Bmb), OP(tsz)(n, Bnt, Bn, Bnb), Bmb,
                            mzone, OA(m, k), lda, OB(k, n), ldb, la, OB(m, n), ldb, 0, 0);
        }
      } else {                                                  /* ztrsm.c:342-372 */
        for (long k = 0; k < Bmt; k++) {
          long km = k == 0 ? Bm - (Bmt - 1) * Bmb : Bmb;
          OT la = k == 0 ? alpha : zone;
          long kk = Bmt - 1 - k;
#pragma omp parallel for
          for (long n = 0; n < Bnt; n++)
            OP(tile_trsm)(side, uplo, trans, diag, km, OP(tsz)(n, Bnt, Bn, Bnb), la, OA(kk, kk), lda, OB(kk, n), ldb);
#pragma omp parallel for collapse(2)
          for (long m = k + 1; m < Bmt; m++)
            for (long n = 0; n < Bnt; n++)
              OP(tile_gemm)(0, trans, XKO_NOTRANS, Bmb, OP(tsz)(n, Bnt, Bn, Bnb), km, mzone,
                            OA(kk, Bmt - 1 - m), lda, OB(kk, n), ldb, la, OB(Bmt - 1 - m, n), ldb, 0, 0);
        }
      }
    }
  } else {
    OT minvalpha = (OT)-1 / alpha;
    if (uplo == XKO_UPPER) {
      if (trans == XKO_NOTRANS) {                               /* ztrsm.c:375-407 */
        for (long k = 0; k < Bnt; k++) {
          long kn = OP(tsz)(k, Bnt, Bn, Bnb);
          OT la = k == 0 ? alpha : zone;
#pragma omp parallel for
          for (long m = 0; m < Bmt; m++)
            OP(tile_trsm)(side, uplo, trans, diag, OP(tsz)(m, Bmt, Bm, Bmb), kn, la, OA(k, k), lda, OB(m, k), ldb);
#pragma omp parallel for collapse(2)
          for (long m = 0; m < Bmt; m++)
            for (long n = k + 1; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, OP(tsz)(m, Bmt, Bm, Bmb), OP(tsz)(n, Bnt, Bn, Bnb), Bmb,
                            mzone, OB(m, k), ldb, OA(k, n), lda, la, OB(m, n), ldb, 0, 0);
        }
      } else {                                                  /* ztrsm.c:409-435 */
        for (long k = 0; k < Bnt; k++) {
          long kn = k == 0 ? Bn - (Bnt - 1) * Bnb : Bnb;
          long kk = Bnt - 1 - k;
#pragma omp parallel for
          for (long m = 0; m < Bmt; m++) {
            long mm = OP(tsz)(m, Bmt, Bm, Bmb);
            OP(tile_trsm)(side, uplo, trans, diag, mm, kn, alpha, OA(kk, kk), lda, OB(m, kk), ldb);
            for (long n = k + 1; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, trans, mm, Bnb, kn, minvalpha, OB(m, kk), ldb,
                            OA(Bnt - 1 - n, kk), lda, zone, OB(m, Bnt - 1 - n), ldb, 0, 0);
          }
        }
      }
    } else {
      if (trans == XKO_NOTRANS) {                               /* ztrsm.c:438-465 */
        for (long k = 0; k < Bnt; k++) {
          long kn = k == 0 ? Bn - (Bnt - 1) * Bnb : Bnb;
          OT la = k == 0 ? alpha : zone;
          long kk = Bnt - 1 - k;
#pragma omp parallel for
          for (long m = 0; m < Bmt; m++) {
            long mm = OP(tsz)(m, Bmt, Bm, Bmb);
            OP(tile_trsm)(side, uplo, trans, diag, mm, kn, la, OA(kk, kk), lda, OB(m, kk), ldb);
            for (long n = k + 1; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, mm, Bnb, kn, mzone, OB(m, kk), ldb,
                            OA(kk, Bnt - 1 - n), lda, la, OB(m, Bnt - 1 - n), ldb, 0, 0);
          }
        }
      } else {                                                  /* ztrsm.c:467-495 */
        for (long k = 0; k < Bnt; k++) {
          long kn = OP(tsz)(k, Bnt, Bn, Bnb);
#pragma omp parallel for
          for (long m = 0; m < Bmt; m++) {
            long mm = OP(tsz)(m, Bmt, Bm, Bmb);
            OP(tile_trsm)(side, uplo, trans, diag, mm, kn, alpha, OA(k, k), lda, OB(m, k), ldb);
            for (long n = k + 1; n < Bnt; n++)
              OP(tile_gemm)(0, XKO_NOTRANS, trans, mm, OP(tsz)(n, Bnt, Bn, Bnb), Bmb, minvalpha,
                            OB(m, k), ldb, OA(n, k), lda, zone, OB(m, n), ldb, 0, 0);
          }
        }
      }
    }
  }
}

/* Tile SYRK / HERK: blas/zsyrk.c:206-316 and blas/zherk.c:208-320: diagonal
 * tile by the rank-k kernel, off-diagonal tiles by GEMM(N,T) / GEMM(N,C)
 * (or (T,N)/(C,N) when trans != N), beta on k == 0 only. */
static void OP(xko_rk)(int herm, int uplo, int trans, int N, int K, OT alpha,
                       const OT* A, int lda, OT beta, OT* C, int ldc, int NB) {
  if (N == 0) return;
  long nt = OP(ntiles)(N, NB);
  long An = (trans == XKO_NOTRANS) ? K : N;   /* columns of A */
  long Am = (trans == XKO_NOTRANS) ? N : K;
  long kt = (trans == XKO_NOTRANS) ? OP(ntiles)(An, NB) : OP(ntiles)(Am, NB);
  long Ktot = K;
  int tcon = herm ? XKO_CONJTRANS : XKO_TRANS;
#pragma omp parallel for schedule(dynamic)
  for (long n = 0; n < nt; n++) {
    long nn = OP(tsz)(n, nt, N, NB);
    OT* Cnn = C + n * NB + n * NB * (long)ldc;
    if (kt == 0) { OP(tile_syrk)(herm, uplo, trans, nn, 0, alpha, A, lda, beta, Cnn, ldc); }
    for (long k = 0; k < kt; k++) {
      long kk = OP(tsz)(k, kt, Ktot, NB);
      const OT* Ank = (trans == XKO_NOTRANS) ? OA(n, k) : OA(k, n);
      OP(tile_syrk)(herm, uplo, trans, nn, kk, alpha, Ank, lda, k == 0 ? beta : (OT)1, Cnn, ldc);
    }
    for (long m = n + 1; m < nt; m++) {
      long mm = OP(tsz)(m, nt, N, NB);
      for (long k = 0; k < kt; k++) {
        long kk = OP(tsz)(k, kt, Ktot, NB);
        OT bk = k == 0 ? beta : (OT)1;
        if (trans == XKO_NOTRANS) {
          if (uplo == XKO_LOWER)
            OP(tile_gemm)(0, XKO_NOTRANS, tcon, mm, nn, kk, alpha, OA(m, k), lda, OA(n, k), lda,
                          bk, C + m * NB + n * NB * (long)ldc, ldc, 0, 0);
          else
            OP(tile_gemm)(0, XKO_NOTRANS, tcon, nn, mm, kk, alpha, OA(n, k), lda, OA(m, k), lda,
                          bk, C + n * NB + m * NB * (long)ldc, ldc, 0, 0);
        } else {
          if (uplo == XKO_LOWER)
            OP(tile_gemm)(0, tcon, XKO_NOTRANS, mm, nn, kk, alpha, OA(k, m), lda, OA(k, n), lda,
                          bk, C + m * NB + n * NB * (long)ldc, ldc, 0, 0);
          else
            OP(tile_gemm)(0, tcon, XKO_NOTRANS, nn, mm, kk, alpha, OA(k, n), lda, OA(k, m), lda,
                          bk, C + n * NB + m * NB * (long)ldc, ldc, 0, 0);
        }
      }
      if (kt == 0) {
        OT* Cmn = (uplo == XKO_LOWER) ? C + m * NB + n * NB * (long)ldc : C + n * NB + m * NB * (long)ldc;
        long r = (uplo == XKO_LOWER) ? mm : nn, c = (uplo == XKO_LOWER) ? nn : mm;
        OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, r, c, 0, alpha, A, lda, A, lda, beta, Cmn, ldc, 0, 0);
      }
    }
  }
}

void OP(xko_syrk)(int uplo, int trans, int N, int K, const OT* alpha,
                  const OT* A, int lda, const OT* beta, OT* C, int ldc, int NB) {
  OP(xko_rk)(0, uplo, trans, N, K, *alpha, A, lda, *beta, C, ldc, NB);
}

#if OCPLX
void OP(xko_herk)(int uplo, int trans, int N, int K, const OR* alpha,
                  const OT* A, int lda, const OR* beta, OT* C, int ldc, int NB) {
  OP(xko_rk)(1, uplo, trans, N, K, (OT)*alpha, A, lda, (OT)*beta, C, ldc, NB);
}
#endif

/* SYR2K / HER2K: C = alpha op(A) op(B)^T + alpha' op(B) op(A)^T + beta C on
 * one triangle, alpha' = alpha (syr2k) or conj(alpha) (her2k); restated at
 * the definition level -- the reference tile loop (blas/zsyr2k.c:234-325,
 * blas/zher2k.c:231-380) only reorders these sums per tile. */
static void OP(xko_r2k)(int herm, int uplo, int trans, int N, int K, OT alpha,
                        const OT* A, int lda, const OT* B, int ldb, OT beta,
                        OT* C, int ldc) {
  OT alpha2 = herm ? OCONJ(alpha) : alpha;
#pragma omp parallel for schedule(dynamic)
  for (long j = 0; j < N; j++) {
    long i0 = (uplo == XKO_LOWER) ? j : 0, i1 = (uplo == XKO_LOWER) ? N : j + 1;
    for (long i = i0; i < i1; i++) {
      OT s1 = 0, s2 = 0;
      for (long p = 0; p < K; p++) {
        OT ai, bj, bi, aj;
        if (trans == XKO_NOTRANS) {
          ai = A[i + p * lda]; bi = B[i + p * ldb]; aj = A[j + p * lda]; bj = B[j + p * ldb];
        } else {
          ai = A[p + i * lda]; bi = B[p + i * ldb]; aj = A[p + j * lda]; bj = B[p + j * ldb];
          if (herm) { ai = OCONJ(ai); bi = OCONJ(bi); aj = OCONJ(aj); bj = OCONJ(bj); }
        }
        if (herm) { s1 += ai * OCONJ(bj); s2 += bi * OCONJ(aj); }
        else { s1 += ai * bj; s2 += bi * aj; }
      }
      OT c = (beta == (OT)0) ? (OT)0 : beta * C[i + j * ldc];
      OT r = alpha * s1 + alpha2 * s2 + c;
#if OCPLX
      if (herm && i == j) r = OREAL(r);
#endif
      C[i + j * ldc] = r;
    }
  }
}

void OP(xko_syr2k)(int uplo, int trans, int N, int K, const OT* alpha,
                   const OT* A, int lda, const OT* B, int ldb, const OT* beta,
                   OT* C, int ldc, int NB) {
  (void)NB;
  OP(xko_r2k)(0, uplo, trans, N, K, *alpha, A, lda, B, ldb, *beta, C, ldc);
}

#if OCPLX
void OP(xko_her2k)(int uplo, int trans, int N, int K, const OT* alpha,
                   const OT* A, int lda, const OT* B, int ldb, const OR* beta,
                   OT* C, int ldc, int NB) {
  (void)NB;
  OP(xko_r2k)(1, uplo, trans, N, K, *alpha, A, lda, B, ldb, (OT)*beta, C, ldc);
}
#endif

/* SYMM / HEMM: C = alpha*A*B + beta*C (side L) or alpha*B*A + beta*C, A
 * symmetric / Hermitian stored in one triangle; definition-level restatement
 * of blas/zsymm.c:230-400 and blas/zhemm.c:234-390. */
static OT OP(symel)(int herm, int uplo, const OT* A, long lda, long i, long j) {
  int stored = (uplo == XKO_LOWER) ? (i >= j) : (i <= j);
  OT v = stored ? A[i + j * lda] : A[j + i * lda];
  if (!stored && herm) v = OCONJ(v);
#if OCPLX
  if (herm && i == j) v = OREAL(v);
#endif
  return v;
}

static void OP(xko_sm)(int herm, int side, int uplo, int M, int N, OT alpha,
                       const OT* A, int lda, const OT* B, int ldb, OT beta,
                       OT* C, int ldc) {
#pragma omp parallel for schedule(dynamic)
  for (long j = 0; j < N; j++)
    for (long i = 0; i < M; i++) {
      OT s = 0;
      if (side == XKO_LEFT)
        for (long p = 0; p < M; p++) s += OP(symel)(herm, uplo, A, lda, i, p) * B[p + j * ldb];
      else
        for (long p = 0; p < N; p++) s += B[i + p * ldb] * OP(symel)(herm, uplo, A, lda, p, j);
      OT c = (beta == (OT)0) ? (OT)0 : beta * C[i + j * ldc];
      C[i + j * ldc] = alpha * s + c;
    }
}

void OP(xko_symm)(int side, int uplo, int M, int N, const OT* alpha,
                  const OT* A, int lda, const OT* B, int ldb, const OT* beta,
                  OT* C, int ldc, int NB) {
  (void)NB;
  OP(xko_sm)(0, side, uplo, M, N, *alpha, A, lda, B, ldb, *beta, C, ldc);
}

#if OCPLX
void OP(xko_hemm)(int side, int uplo, int M, int N, const OT* alpha,
                  const OT* A, int lda, const OT* B, int ldb, const OT* beta,
                  OT* C, int ldc, int NB) {
  (void)NB;
  OP(xko_sm)(1, side, uplo, M, N, *alpha, A, lda, B, ldb, *beta, C, ldc);
}
#endif

/* TRMM: B = alpha*op(A)*B (side L) or alpha*B*op(A), A triangular;
 * definition-level restatement of blas/ztrmm.c:224-460. */
void OP(xko_trmm)(int side, int uplo, int trans, int diag, int M, int N,
                  const OT* palpha, const OT* A, int lda, OT* B, int ldb,
                  int NB) {
  (void)NB;
  OT alpha = *palpha;
  int lower = (uplo == XKO_LOWER) ^ (trans != XKO_NOTRANS);
  long na = (side == XKO_LEFT) ? M : N;
  OT* T = (OT*)malloc(sizeof(OT) * (size_t)na * (size_t)na);
  for (long j = 0; j < na; j++)
    for (long i = 0; i < na; i++) {
      OT v = 0;
      if (i == j) v = (diag == XKO_UNIT) ? (OT)1 : OP(opel)(trans, A, lda, i, j);
      else if ((lower && i > j) || (!lower && i < j)) v = OP(opel)(trans, A, lda, i, j);
      T[i + j * na] = v;
    }
  OT* R = (OT*)malloc(sizeof(OT) * (size_t)M * (size_t)N);
#pragma omp parallel for schedule(dynamic)
  for (long j = 0; j < N; j++)
    for (long i = 0; i < M; i++) {
      OT s = 0;
      if (side == XKO_LEFT) for (long p = 0; p < M; p++) s += T[i + p * na] * B[p + j * ldb];
      else for (long p = 0; p < N; p++) s += B[i + p * ldb] * T[p + j * na];
      R[i + j * M] = alpha * s;
    }
  for (long j = 0; j < N; j++)
    for (long i = 0; i < M; i++) B[i + j * ldb] = R[i + j * M];
  free(R);
  free(T);
}
/* LU factorization without pivoting, tile algorithm of
 * blas/zgetrf_nopiv.c:48-101 (Chameleon pzgetrf_nopiv): for each diagonal
 * tile k, the unblocked LU of A(k,k) (no pivoting), the column panel
 * A(m,k) <- A(m,k) U(k,k)^-1 (trsm Right/Upper/NoTrans/NonUnit), the row
 * panel A(k,n) <- L(k,k)^-1 A(k,n) (trsm Left/Lower/NoTrans/Unit), and the
 * trailing updates A(m,n) -= A(m,k) A(k,n).  Returns the first zero pivot,
 * 1-based (0 = none); the factorization continues past it. */
int OP(xko_getrf_nopiv)(int M, int N, OT* A, int lda, int NB) {
  long mt = OP(ntiles)(M, NB), nt = OP(ntiles)(N, NB);
  long kt = mt < nt ? mt : nt;
  int info = 0;
  OT zone = 1, mzone = -1;
  for (long k = 0; k < kt; k++) {
    long tkm = (k == mt - 1) ? M - k * NB : NB;
    long tkn = (k == nt - 1) ? N - k * NB : NB;
    OT* Akk = OA(k, k);
    long kmin = tkm < tkn ? tkm : tkn;
    for (long j = 0; j < kmin; j++) {  /* unblocked right-looking LU of the tile */
      OT d = Akk[j + j * lda];
      if (d == (OT)0 && info == 0) info = (int)(k * NB + j + 1);
      for (long i = j + 1; i < tkm; i++) Akk[i + j * lda] /= d;
      for (long c = j + 1; c < tkn; c++)
        for (long i = j + 1; i < tkm; i++) Akk[i + c * lda] -= Akk[i + j * lda] * Akk[j + c * lda];
    }
    for (long m = k + 1; m < mt; m++) {
      long tmm = (m == mt - 1) ? M - m * NB : NB;
      OP(tile_trsm)(XKO_RIGHT, XKO_UPPER, XKO_NOTRANS, XKO_NONUNIT, tmm, tkn, zone, Akk, lda,
                    OA(m, k), lda);
    }
    for (long n = k + 1; n < nt; n++) {
      long tnn = (n == nt - 1) ? N - n * NB : NB;
      OP(tile_trsm)(XKO_LEFT, XKO_LOWER, XKO_NOTRANS, XKO_UNIT, tkm, tnn, zone, Akk, lda,
                    OA(k, n), lda);
      for (long m = k + 1; m < mt; m++) {
        long tmm = (m == mt - 1) ? M - m * NB : NB;
        OP(tile_gemm)(0, XKO_NOTRANS, XKO_NOTRANS, tmm, tnn, NB, mzone, OA(m, k), lda,
                      OA(k, n), lda, zone, OA(m, n), lda, 0, 0);
      }
    }
  }
  return info;
}

#undef OA
#undef OB
