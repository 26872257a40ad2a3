// native.cpp -- the xkblas_?xxx_native entry points of xkblas.h: direct calls
// of the system CPU BLAS through its Fortran symbols, loaded with dlopen
// exactly as the reference does (xkblas_load_sym, blas/xkblas.c:2678-2696;
// callers e.g. blas/zgemm.c:383-414).  They are part of the reference API
// (its tests use them as the reference result) and are never called by the
// *_async GPU path.  Library: $XKBLAS_BLASLIB, else "libopenblas.so".
// Divergence: a missing library or symbol returns ENOSYS instead of abort().
#include <dlfcn.h>

#include <cerrno>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "xkblas.h"

namespace {
std::mutex g_mu;
void* g_handle = nullptr;

void* blas_handle() {
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_handle) {
    const char* lib = getenv("XKBLAS_BLASLIB");
    g_handle = dlopen(lib ? lib : "libopenblas.so", RTLD_NOW | RTLD_LOCAL);
  }
  return g_handle;
}

char op(int t) { return t == CblasNoTrans ? 'N' : (t == CblasTrans ? 'T' : 'C'); }
char ul(int u) { return u == CblasUpper ? 'U' : 'L'; }
char sd(int s) { return s == CblasLeft ? 'L' : 'R'; }
char dg(int d) { return d == CblasUnit ? 'U' : 'N'; }

template <class F>
F sym(const char* name) {
  void* h = blas_handle();
  return h ? reinterpret_cast<F>(dlsym(h, name)) : nullptr;
}

typedef void (*gemm_t)(const char*, const char*, const int*, const int*, const int*, const void*,
                       const void*, const int*, const void*, const int*, const void*, void*,
                       const int*);
typedef void (*gemmt_t)(const char*, const char*, const char*, const int*, const int*,
                        const void*, const void*, const int*, const void*, const int*,
                        const void*, void*, const int*);
typedef void (*trxm_t)(const char*, const char*, const char*, const char*, const int*,
                       const int*, const void*, const void*, const int*, void*, const int*);
typedef void (*xymm_t)(const char*, const char*, const int*, const int*, const void*,
                       const void*, const int*, const void*, const int*, const void*, void*,
                       const int*);
typedef void (*xyrk_t)(const char*, const char*, const int*, const int*, const void*,
                       const void*, const int*, const void*, void*, const int*);
typedef void (*xyr2k_t)(const char*, const char*, const int*, const int*, const void*,
                        const void*, const int*, const void*, const int*, const void*, void*,
                        const int*);
}  // namespace

extern "C" void xkblas_load_sym(void** ptr, const char* name) {
  if (!ptr) return;
  void* h = blas_handle();
  *ptr = (h && name) ? dlsym(h, name) : nullptr;
}

#define XKB_NATIVE_OPS(p, T, R)                                                                 \
  extern "C" int xkblas_##p##gemm_native(int tA, int tB, int M, int N, int K, const T* al,      \
                                         const T* A, int lda, const T* B, int ldb, const T* be,  \
                                         T* C, int ldc) {                                        \
    gemm_t f = sym<gemm_t>(#p "gemm_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = op(tA), b = op(tB);                                                                \
    f(&a, &b, &M, &N, &K, al, A, &lda, B, &ldb, be, C, &ldc);                                   \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##gemmt_native(int u, int tA, int tB, int N, int K, const T* al,     \
                                          const T* A, int lda, const T* B, int ldb,             \
                                          const T* be, T* C, int ldc) {                         \
    gemmt_t f = sym<gemmt_t>(#p "gemmt_");                                                      \
    if (!f) return ENOSYS;                                                                      \
    char c = ul(u), a = op(tA), b = op(tB);                                                     \
    f(&c, &a, &b, &N, &K, al, A, &lda, B, &ldb, be, C, &ldc);                                   \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##trsm_native(int s, int u, int tA, int d, int M, int N,             \
                                         const T* al, const T* A, int lda, T* B, int ldb) {     \
    trxm_t f = sym<trxm_t>(#p "trsm_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = sd(s), b = ul(u), c = op(tA), e = dg(d);                                           \
    f(&a, &b, &c, &e, &M, &N, al, A, &lda, B, &ldb);                                            \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##trmm_native(int s, int u, int tA, int d, int M, int N,             \
                                         const T* al, const T* A, int lda, T* B, int ldb) {     \
    trxm_t f = sym<trxm_t>(#p "trmm_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = sd(s), b = ul(u), c = op(tA), e = dg(d);                                           \
    f(&a, &b, &c, &e, &M, &N, al, A, &lda, B, &ldb);                                            \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##symm_native(int s, int u, int M, int N, const T* al, const T* A,   \
                                         int lda, const T* B, int ldb, const T* be, T* C,       \
                                         int ldc) {                                             \
    xymm_t f = sym<xymm_t>(#p "symm_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = sd(s), b = ul(u);                                                                  \
    f(&a, &b, &M, &N, al, A, &lda, B, &ldb, be, C, &ldc);                                       \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##syrk_native(int u, int t, int N, int K, const T* al, const T* A,   \
                                         int lda, const T* be, T* C, int ldc) {                 \
    xyrk_t f = sym<xyrk_t>(#p "syrk_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = ul(u), b = op(t);                                                                  \
    f(&a, &b, &N, &K, al, A, &lda, be, C, &ldc);                                                \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##syr2k_native(int u, int t, int N, int K, const T* al, const T* A,  \
                                          int lda, const T* B, int ldb, const T* be, T* C,      \
                                          int ldc) {                                            \
    xyr2k_t f = sym<xyr2k_t>(#p "syr2k_");                                                      \
    if (!f) return ENOSYS;                                                                      \
    char a = ul(u), b = op(t);                                                                  \
    f(&a, &b, &N, &K, al, A, &lda, B, &ldb, be, C, &ldc);                                       \
    return 0;                                                                                   \
  }

#define XKB_NATIVE_HE_OPS(p, T, R)                                                              \
  extern "C" int xkblas_##p##hemm_native(int s, int u, int M, int N, const T* al, const T* A,   \
                                         int lda, const T* B, int ldb, const T* be, T* C,       \
                                         int ldc) {                                             \
    xymm_t f = sym<xymm_t>(#p "hemm_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = sd(s), b = ul(u);                                                                  \
    f(&a, &b, &M, &N, al, A, &lda, B, &ldb, be, C, &ldc);                                       \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##herk_native(int u, int t, int N, int K, const R* al, const T* A,   \
                                         int lda, const R* be, T* C, int ldc) {                 \
    xyrk_t f = sym<xyrk_t>(#p "herk_");                                                         \
    if (!f) return ENOSYS;                                                                      \
    char a = ul(u), b = op(t);                                                                  \
    f(&a, &b, &N, &K, al, A, &lda, be, C, &ldc);                                                \
    return 0;                                                                                   \
  }                                                                                             \
  extern "C" int xkblas_##p##her2k_native(int u, int t, int N, int K, const T* al, const T* A,  \
                                          int lda, const T* B, int ldb, const R* be, T* C,      \
                                          int ldc) {                                            \
    xyr2k_t f = sym<xyr2k_t>(#p "her2k_");                                                      \
    if (!f) return ENOSYS;                                                                      \
    char a = ul(u), b = op(t);                                                                  \
    f(&a, &b, &N, &K, al, A, &lda, B, &ldb, be, C, &ldc);                                       \
    return 0;                                                                                   \
  }

XKB_NATIVE_OPS(s, float, float)
XKB_NATIVE_OPS(d, double, double)
XKB_NATIVE_OPS(c, Complex32_t, float)
XKB_NATIVE_OPS(z, Complex64_t, double)
XKB_NATIVE_HE_OPS(c, Complex32_t, float)
XKB_NATIVE_HE_OPS(z, Complex64_t, double)
