/*
 * xkb_oracle.c -- CPU oracle for the XKBlas level-3 tile path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, always as the checker.
 * The GPU library (libxkblas.so) neither links nor calls it.
 *
 * Contents
 *   - tiled drivers restating the reference tile algorithms for d and z
 *     (xkb_oracle_tmpl.h; s and c are checked through d and z on the same,
 *     exactly representable, inputs);
 *   - a double-double (Dekker/Knuth TwoProd via FMA + TwoSum) GEMM on chosen
 *     entries, the accuracy yardstick for the FP64 and Ozaki paths;
 *   - the seeded generators of the workloads: a PLASMA-zplrnt-style LCG
 *     (multiplier 6364136223846793005, increment 1 -- the constants of the
 *     reference's testing/zplgsy.c:37-39) scaled with a DOUBLE multiplier
 *     2^-64, the reference's zplgsy generator with its float multiplier kept
 *     (testing/zplgsy.c:69-101), and the exponent-spread generator;
 *   - the CPU reference path: dlopen of the system BLAS and its Fortran
 *     symbols, exactly what xkblas_?xxx_native does (reference
 *     blas/xkblas.c:2678-2696, blas/zgemm.c:383-414).
 */
#define _GNU_SOURCE
#include <complex.h>
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define XKO_NOTRANS 111
#define XKO_TRANS 112
#define XKO_CONJTRANS 113
#define XKO_UPPER 121
#define XKO_LOWER 122
#define XKO_NONUNIT 131
#define XKO_UNIT 132
#define XKO_LEFT 141
#define XKO_RIGHT 142

/* ---- real double instance ---- */
#define OT double
#define OR double
#define OP(x) d_##x
#define OCPLX 0
#define OCONJ(x) (x)
#define OREAL(x) (x)
#include "xkb_oracle_tmpl.h"
#undef OT
#undef OR
#undef OP
#undef OCPLX
#undef OCONJ
#undef OREAL

/* ---- complex double instance ---- */
#define OT double complex
#define OR double
#define OP(x) z_##x
#define OCPLX 1
#define OCONJ(x) conj(x)
#define OREAL(x) ((double complex)creal(x))
#include "xkb_oracle_tmpl.h"
#undef OT
#undef OR
#undef OP
#undef OCPLX
#undef OCONJ
#undef OREAL

/* ---- double-double accumulation ---------------------------------------- */
typedef struct { double hi, lo; } dd_t;

static inline dd_t dd_add_d(dd_t a, double b) {           /* Knuth TwoSum */
  double s = a.hi + b, bb = s - a.hi;
  double e = (a.hi - (s - bb)) + (b - bb) + a.lo;
  double h = s + e;
  dd_t r = {h, e - (h - s)};
  return r;
}
static inline dd_t dd_add_prod(dd_t a, double x, double y) { /* + x*y exactly split */
  double p = x * y, pe = fma(x, y, -p);                      /* Dekker TwoProd (FMA) */
  dd_t r = dd_add_d(a, p);
  return dd_add_d(r, pe);
}

static inline double d_opget(int t, const double* A, long lda, long i, long p) {
  return t == XKO_NOTRANS ? A[i + p * lda] : A[p + i * lda];
}

/* out[r + c*nr] = alpha*(op(A) op(B))(rows[r], cols[c]) + beta*C(...), the
 * dot products accumulated in double-double and the result rounded once.
 * out_lo (optional) receives the low word before the alpha/beta update. */
void xko_dgemm_dd(int ta, int tb, int K, double alpha, const double* A,
                  int lda, const double* B, int ldb, double beta,
                  const double* C, int ldc, const long* rows, int nr,
                  const long* cols, int nc, double* out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int c = 0; c < nc; c++)
    for (int r = 0; r < nr; r++) {
      long i = rows[r], j = cols[c];
      dd_t s = {0.0, 0.0};
      for (long p = 0; p < K; p++)
        s = dd_add_prod(s, d_opget(ta, A, lda, i, p), d_opget(tb, B, ldb, p, j));
      /* alpha*s + beta*c in double-double, rounded once */
      double ph = alpha * s.hi, pe = fma(alpha, s.hi, -ph);
      dd_t t = {ph, pe + alpha * s.lo};
      if (beta != 0.0 && C) t = dd_add_prod(t, beta, C[i + j * (long)ldc]);
      out[r + (long)c * nr] = t.hi + t.lo;
    }
}

/* complex version: 4 real products per complex product, each part in dd */
static inline double complex z_opget(int t, const double complex* A, long lda,
                                     long i, long p) {
  if (t == XKO_NOTRANS) return A[i + p * lda];
  double complex v = A[p + i * lda];
  return t == XKO_CONJTRANS ? conj(v) : v;
}
void xko_zgemm_dd(int ta, int tb, int K, const double complex* alpha,
                  const double complex* A, int lda, const double complex* B,
                  int ldb, const double complex* beta, const double complex* C,
                  int ldc, const long* rows, int nr, const long* cols, int nc,
                  double complex* out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int c = 0; c < nc; c++)
    for (int r = 0; r < nr; r++) {
      long i = rows[r], j = cols[c];
      dd_t sr = {0, 0}, si = {0, 0};
      for (long p = 0; p < K; p++) {
        double complex a = z_opget(ta, A, lda, i, p), b = z_opget(tb, B, ldb, p, j);
        sr = dd_add_prod(sr, creal(a), creal(b));
        sr = dd_add_prod(sr, -cimag(a), cimag(b));
        si = dd_add_prod(si, creal(a), cimag(b));
        si = dd_add_prod(si, cimag(a), creal(b));
      }
      double ar = creal(*alpha), ai = cimag(*alpha);
      dd_t tr = {0, 0}, ti = {0, 0};
      tr = dd_add_prod(tr, ar, sr.hi); tr = dd_add_prod(tr, -ai, si.hi);
      tr = dd_add_d(tr, ar * sr.lo - ai * si.lo);
      ti = dd_add_prod(ti, ar, si.hi); ti = dd_add_prod(ti, ai, sr.hi);
      ti = dd_add_d(ti, ar * si.lo + ai * sr.lo);
      if (C && (creal(*beta) != 0.0 || cimag(*beta) != 0.0)) {
        double complex cv = C[i + j * (long)ldc];
        double br = creal(*beta), bi = cimag(*beta);
        tr = dd_add_prod(tr, br, creal(cv)); tr = dd_add_prod(tr, -bi, cimag(cv));
        ti = dd_add_prod(ti, br, cimag(cv)); ti = dd_add_prod(ti, bi, creal(cv));
      }
      out[r + (long)c * nr] = (tr.hi + tr.lo) + I * (ti.hi + ti.lo);
    }
}

/* ---- generators ---------------------------------------------------------- */
#define XKO_RND_A 6364136223846793005ULL
#define XKO_RND_C 1ULL

/* LCG state after n steps from seed, by repeated squaring of the affine map
 * (the jump-ahead used by the reference generator, testing/zplgsy.c:43-62). */
static uint64_t xko_jump(uint64_t n, uint64_t seed) {
  uint64_t a = XKO_RND_A, c = XKO_RND_C, ran = seed;
  for (; n; n >>= 1) {
    if (n & 1) ran = a * ran + c;
    c *= (a + 1);
    a *= a;
  }
  return ran;
}

/* A(i,j) = 0.5 - ran*2^-64 for the element of linear index i + j*bigM in a
 * bigM-row matrix (so any tile can be generated independently), values in
 * (-0.5, 0.5] with 53-bit mantissas.  For complex (cplx=1) the imaginary part
 * takes the next number of the stream.  A is column major, leading dim lda. */
void xko_plrnt(int cplx, long M, long N, double* A, long lda, long bigM,
               long i0, long j0, uint64_t seed) {
  const double mul = 5.421010862427522170037264e-20; /* 2^-64 */
  long per = cplx ? 2 : 1;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < N; j++) {
    uint64_t ran = xko_jump((uint64_t)per * ((uint64_t)(i0) + (uint64_t)(j0 + j) * (uint64_t)bigM), seed);
    for (long i = 0; i < M; i++) {
      double re = 0.5 - (double)ran * mul;
      ran = XKO_RND_A * ran + XKO_RND_C;
      if (cplx) {
        double im = 0.5 - (double)ran * mul;
        ran = XKO_RND_A * ran + XKO_RND_C;
        A[2 * (i + j * lda)] = re;
        A[2 * (i + j * lda) + 1] = im;
      } else {
        A[i + j * lda] = re;
      }
    }
  }
}

/* The reference's symmetric/Hermitian test generator, testing/zplgsy.c:69-101,
 * restated with its quirks: float multiplier (24-bit mantissas), one jump of
 * NBELEM*N per column (NBELEM = 1 real, 2 complex), lower triangle
 * generated then mirrored (transpose, no conjugation), bump added to the
 * diagonal. */
void xko_plgsy(int cplx, double bump, long N, double* A, long lda,
               uint64_t seed) {
  const float fmul = 5.4210108624275222e-20f;
  long nbelem = cplx ? 2 : 1;
  for (long j = 0; j < N; j++) {
    uint64_t ran = xko_jump((uint64_t)(nbelem * N), seed);
    for (long i = j; i < N; i++) {
      double re = (double)(0.5f - (float)ran * fmul);
      ran = XKO_RND_A * ran + XKO_RND_C;
      if (cplx) {
        double im = (double)(0.5f - (float)ran * fmul);
        ran = XKO_RND_A * ran + XKO_RND_C;
        A[2 * (j * lda + i)] = re;
        A[2 * (j * lda + i) + 1] = im;
      } else {
        A[j * lda + i] = re;
      }
    }
  }
  for (long j = 0; j < N; j++) {
    A[(j + j * lda) * nbelem] += bump;
    for (long i = 0; i < j; i++) {
      if (cplx) {
        A[2 * (lda * j + i)] = A[2 * (lda * i + j)];
        A[2 * (lda * j + i) + 1] = A[2 * (lda * i + j) + 1];
      } else {
        A[lda * j + i] = A[lda * i + j];
      }
    }
  }
}

/* Wide exponent spread: a(i,j) = u*2^e, u uniform (-1,1] from the LCG,
 * e uniform integer in [-emax, emax]; e drawn per row (by_col = 0) or per
 * column (by_col = 1) from a second stream (seed + 0x9e3779b97f4a7c15). */
void xko_expspread(long M, long N, double* A, long lda, int emax, int by_col,
                   uint64_t seed) {
  const double mul = 5.421010862427522170037264e-20;
  long ne = by_col ? N : M;
  int* e = (int*)malloc(sizeof(int) * (size_t)(ne > 0 ? ne : 1));
  uint64_t r2 = seed + 0x9e3779b97f4a7c15ULL;
  for (long t = 0; t < ne; t++) {
    r2 = XKO_RND_A * r2 + XKO_RND_C;
    e[t] = (int)((r2 >> 11) % (uint64_t)(2 * emax + 1)) - emax;
  }
#pragma omp parallel for schedule(static)
  for (long j = 0; j < N; j++) {
    uint64_t ran = xko_jump((uint64_t)j * (uint64_t)M, seed);
    for (long i = 0; i < M; i++) {
      double u = 1.0 - 2.0 * ((double)ran * mul);
      ran = XKO_RND_A * ran + XKO_RND_C;
      A[i + j * lda] = ldexp(u, by_col ? e[j] : e[i]);
    }
  }
  free(e);
}

/* ---- CPU reference path: the system BLAS, loaded like xkblas_load_sym ---- */
static void* xko_blas = NULL;
static char xko_blas_path[4096];

/* Returns 0 on success.  path NULL: $XKBLAS_BLASLIB, else libopenblas.so. */
int xko_blas_open(const char* path) {
  if (xko_blas) return 0;
  if (!path) path = getenv("XKBLAS_BLASLIB");
  if (!path) path = "libopenblas.so";
  xko_blas = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!xko_blas) return -1;
  strncpy(xko_blas_path, path, sizeof(xko_blas_path) - 1);
  return 0;
}

void* xko_blas_sym(const char* name) {
  if (!xko_blas && xko_blas_open(NULL)) return NULL;
  return dlsym(xko_blas, name);
}

/* Thread count for OpenBLAS (openblas_set_num_threads when exported). */
int xko_blas_set_threads(int n) {
  void (*f)(int) = (void (*)(int))xko_blas_sym("openblas_set_num_threads");
  if (!f) return -1;
  f(n);
  return 0;
}

static char xko_op(int t) { return t == XKO_NOTRANS ? 'N' : (t == XKO_TRANS ? 'T' : 'C'); }
static char xko_ul(int u) { return u == XKO_UPPER ? 'U' : 'L'; }
static char xko_sd(int s) { return s == XKO_LEFT ? 'L' : 'R'; }
static char xko_dg(int d) { return d == XKO_UNIT ? 'U' : 'N'; }

typedef void (*gemm_f)(const char*, const char*, const int*, const int*, const int*,
                       const void*, const void*, const int*, const void*, const int*,
                       const void*, void*, const int*);
typedef void (*trsm_f)(const char*, const char*, const char*, const char*, const int*,
                       const int*, const void*, const void*, const int*, void*, const int*);
typedef void (*rk_f)(const char*, const char*, const int*, const int*, const void*,
                     const void*, const int*, const void*, void*, const int*);

/* p in {'s','d','c','z'}; returns -1 if the symbol is missing. */
int xko_native_gemm(char p, int ta, int tb, int M, int N, int K, const void* alpha,
                    const void* A, int lda, const void* B, int ldb, const void* beta,
                    void* C, int ldc) {
  char nm[16]; snprintf(nm, sizeof nm, "%cgemm_", p);
  gemm_f f = (gemm_f)xko_blas_sym(nm);
  if (!f) return -1;
  char a = xko_op(ta), b = xko_op(tb);
  f(&a, &b, &M, &N, &K, alpha, A, &lda, B, &ldb, beta, C, &ldc);
  return 0;
}

int xko_native_trsm(char p, int side, int uplo, int ta, int diag, int M, int N,
                    const void* alpha, const void* A, int lda, void* B, int ldb) {
  char nm[16]; snprintf(nm, sizeof nm, "%ctrsm_", p);
  trsm_f f = (trsm_f)xko_blas_sym(nm);
  if (!f) return -1;
  char s = xko_sd(side), u = xko_ul(uplo), t = xko_op(ta), d = xko_dg(diag);
  f(&s, &u, &t, &d, &M, &N, alpha, A, &lda, B, &ldb);
  return 0;
}

/* syrk (herk when name is "herk_") */
int xko_native_rk(char p, const char* kind, int uplo, int trans, int N, int K,
                  const void* alpha, const void* A, int lda, const void* beta,
                  void* C, int ldc) {
  char nm[16]; snprintf(nm, sizeof nm, "%c%s", p, kind);
  rk_f f = (rk_f)xko_blas_sym(nm);
  if (!f) return -1;
  char u = xko_ul(uplo), t = xko_op(trans);
  f(&u, &t, &N, &K, alpha, A, &lda, beta, C, &ldc);
  return 0;
}

const char* xko_blas_loaded(void) { return xko_blas ? xko_blas_path : ""; }
