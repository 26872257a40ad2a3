/*
 * xkblas.h -- public C interface of the B200 level-3 BLAS tile library.
 *
 * Drop-in for the XKBlas C API: the same symbol names, argument orders,
 * enum values and return conventions as XKBlas 0.6 (blas/xkblas.h:70-511 and
 * blas/zxkblas.h:45-151 of the reference).  Every declaration below names the
 * reference declaration it replaces.
 *
 * Semantics kept from the reference:
 *   - matrices are host resident, column major, owned by the caller;
 *   - xkblas_?xxx_async() enqueues work and returns 0, or -i when the i-th
 *     argument is invalid (reference e.g. blas/zgemm.c:132-181);
 *   - results are copied back to the host only on request:
 *     xkblas_memory_coherent_async() followed by xkblas_sync();
 *   - device copies stay cached (keyed by the host pointer) until
 *     xkblas_memory_invalidate*() or xkblas_memory_free().
 * Divergence: argument errors are reported by return code only; the library
 * never aborts the process (the reference prints and aborts).
 *
 * All compute runs on the GPU (FP64 DMMA tensor-core kernels, or the Ozaki
 * INT8 tensor-core form under XKBLAS_TENSOR_OP_MATH).  The *_native entry
 * points are the reference's CPU-BLAS pass-through and are never used by the
 * *_async path.
 */
#ifndef XKBLAS_B200_XKBLAS_H
#define XKBLAS_B200_XKBLAS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<float>  Complex32_t;
typedef std::complex<double> Complex64_t;
extern "C" {
#else
#include <complex.h>
typedef float _Complex  Complex32_t;
typedef double _Complex Complex64_t;
#endif
typedef double CFloat64_t;
typedef float  CFloat32_t;

#define __XKBLAS__ 0
#define __XKBLAS_MINOR__ 6
#define __XKBLAS_PATCHLEVEL__ 0

/* ---- enums: values identical to the reference (blas/xkblas.h:100-119) --- */
typedef enum { XKBLAS_DEFAULT_MATH, XKBLAS_TENSOR_OP_MATH } xkblas_mode_math_t;

#ifndef KAAPI_NO_DEFAULT_BLAS_ENUM
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113,
               CblasConjNoTrans = 114 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;
typedef CBLAS_ORDER CBLAS_LAYOUT;
#endif

/* Fortran-BLAS character arguments -> CBLAS enum values (reference
 * blas/xkblas.h:143-200, static inline there too).  First character only,
 * either case.  Divergence: an unknown character gives -1 (which every
 * entry point rejects with its -i argument code) instead of abort(). */
static inline int xkblas_blas2cblas_trans(const char* trans) {
  switch (trans[0]) {
    case 'n': case 'N': return CblasNoTrans;
    case 't': case 'T': return CblasTrans;
    case 'c': case 'C': return CblasConjTrans;
    default: return -1;
  }
}
static inline int xkblas_blas2cblas_side(const char* side) {
  switch (side[0]) {
    case 'l': case 'L': return CblasLeft;
    case 'r': case 'R': return CblasRight;
    default: return -1;
  }
}
static inline int xkblas_blas2cblas_fill(const char* uplo) {
  switch (uplo[0]) {
    case 'l': case 'L': return CblasLower;
    case 'u': case 'U': return CblasUpper;
    default: return -1;
  }
}
static inline int xkblas_blas2cblas_diag(const char* diag) {
  switch (diag[0]) {
    case 'n': case 'N': return CblasNonUnit;
    case 'u': case 'U': return CblasUnit;
    default: return -1;
  }
}

/* reference blas/xkblas.h:124-138 */
typedef enum {
  KERN_VOID, KERN_GEMM, KERN_GEMMT, KERN_TRMM, KERN_TRSM, KERN_SYMM,
  KERN_SYRK, KERN_SYR2K, KERN_HEMM, KERN_HERK, KERN_HER2K, KERN_SWAP,
  KERN_COPYSCALE
} xkblas_kernel_t;

/* reference blas/xkblas.h:221-243 */
typedef struct xkblas_dev_prop_t {
  int arch;
  int has_unified;
  int device_count;
} xkblas_dev_prop_t;

typedef enum xkblas_dev_arch_t {
  XKBLAS_ARCH_UNDEF = -1, XKBLAS_ARCH_UNKNOWN = 0, XKBLAS_ARCH_V100 = 1,
  XKBLAS_ARCH_A100 = 2, XKBLAS_ARCH_RESERVED0 = 3, XKBLAS_ARCH_GRACEHOPPER = 4,
  XKBLAS_ARCH_MI50 = 101, XKBLAS_ARCH_RESERVED1 = 102,
  XKBLAS_ARCH_RESERVED2 = 103, XKBLAS_ARCH_MI250 = 104,
  XKBLAS_ARCH_RESERVED3 = 105, XKBLAS_ARCH_MI300A = 106,
  /* added: Blackwell data-centre part this library is built for */
  XKBLAS_ARCH_B200 = 5
} xkblas_dev_arch_t;

struct xkblas_context;
typedef struct xkblas_context xkblas_context_t;
struct xkblas_matrix_descr;
typedef struct xkblas_matrix_descr xkblas_matrix_descr_t;

/* ---- lifecycle (reference blas/xkblas.h:95-498) ------------------------- */
int  xkblas_get_devicecount(void);                         /* :203 */
int  xkblas_init(void);                                    /* :207; ref-counted */
int  xkblas_finalize(void);                                /* :211 */
int  xkblas_get_device_count(int* count);                  /* :217 */
int  xkblas_get_device_properties(struct xkblas_dev_prop_t* prop); /* :256 */
int  xkblas_force_set_unified(void);                       /* :267; EINVAL here */
const char* xkblas_get_configuration(void);                /* :273 */
void xkblas_load_sym(void** ptr, const char* name);        /* :278 */
int  xkblas_sync(void);                                    /* :282; waits for the
                                                              work queued before it */
xkblas_context_t* xkblas_context_get(void);                /* :95; per thread */
void xkblas_set_modemath(xkblas_mode_math_t mode);         /* :107; per thread */
/* the calling thread's math mode (reference blas/xkblas.c:363-366, exported
 * there without a header declaration) */
xkblas_mode_math_t xkblas_get_modemath(void);
size_t xkblas_get_param(void);                             /* :470 */
void xkblas_set_param(size_t nb, size_t p);                /* :484 */
int  xkblas_get_ngpus(void);                               /* :476 */
int  xkblas_set_ngpus(int ngpus);                          /* :480 */
uint64_t xkblas_elapsedns(void);                           /* :492 */
double   xkblas_elapsedtime(void);                         /* :498 */

/* ---- matrix descriptors (reference blas/xkblas.h:287-312) --------------- */
xkblas_matrix_descr_t* xkblas_find(const void* A);
int xkblas_matrix_descr_isinit(xkblas_matrix_descr_t* Ah);
int xkblas_init_matrix_handle(xkblas_matrix_descr_t* Ah, void* A, size_t M,
                              size_t N, size_t LD, size_t eltsize, size_t MB,
                              size_t NB);
size_t xkblas_auto_tilesize(xkblas_context_t* ctx, xkblas_kernel_t kernel,
                            size_t M, size_t N, size_t K);

/* ---- host memory (reference blas/xkblas.h:70-85, 318-365, 500-511) ----- */
void*    xkblas_malloc(size_t sz);                 /* pinned host memory */
void     xkblas_free(void* ptr, size_t sz);
int      xkblas_malloc_unified(void** ptr, size_t size);
int      xkblas_free_unified(void* ptr);
void     xkblas_activate_custom_alloc(void);
void     xkblas_deactivate_custom_alloc(void);
uint64_t xkblas_register_memory_async(void* ptr, size_t sz);
uint64_t xkblas_unregister_memory_async(void* ptr, size_t sz);
int      xkblas_register_memory_test(uint64_t handle);
int      xkblas_register_memory_wait(uint64_t handle);
int      xkblas_register_memory_waitall(void);
int      xkblas_register_memory(void* ptr, size_t sz);
int      xkblas_unregister_memory(void* ptr, size_t sz);
void     xkblas_memset(void* ptr, int v, size_t sz);
void     xkblas_memcpy(void* dst, void* src, size_t sz);
void     xkblas_register_work_buffer(void* ptr, size_t sz);
void     xkblas_unregister_work_buffer(void* ptr);
void*    xkblas_get_work_pos(size_t sz);
void     xkblas_free_work_pos(void* ptr);
void     xkblas_bind_cpu(void* ptr, size_t sz);
void     xkblas_host_register_direct(void* ptr, size_t sz);
void     xkblas_host_unregister_direct(void* ptr);

/* ---- debug and multi-device placement (reference xkblas.h:371-430) -----
 * One GPU: placement calls validate their arguments and return 0. */
int  xkblas_dbg_setname(const char* name, xkblas_matrix_descr_t* Mh);
int  xkblas_dbg_setname_with_flags(const char* name, xkblas_matrix_descr_t* Mh,
                                   uint32_t flags);
void xkblas_dbg_dump_graph(const char* name);
int  xkblas_map_2Dblock_cyclic(xkblas_context_t* ctx, int hlevel, int storage,
                               size_t m, size_t n, const void* A, size_t ld,
                               size_t eltsize, size_t Bp, size_t Bq, size_t Gp,
                               size_t Gq, int force);
int  xkblas_map_1Dblock_cyclic(xkblas_context_t* ctx, int hlevel, int storage,
                               int colrow, size_t m, size_t n, const void* A,
                               size_t ld, size_t eltsize, size_t B, size_t G,
                               int force);
int  xkblas_distribute_2Dblock_cyclic_async(int hlevel, int storage, int uplo,
                               size_t NB, size_t m, size_t n, const void* A,
                               size_t ld, size_t eltsize, size_t Bp, size_t Bq,
                               size_t Gp, size_t Gq);
int  xkblas_distribute_1Dblock_cyclic_async(int hlevel, int storage, int uplo,
                               int colrow, size_t NB, size_t m, size_t n,
                               const void* A, size_t ld, size_t eltsize,
                               size_t B, size_t G);

/* ---- coherence (reference blas/xkblas.h:441-466) ------------------------
 * uplo 0: whole matrix; CblasUpper/CblasLower: that triangle (diagonal
 * tiles included).  memflag 1: the other triangle's device copy is dropped. */
int xkblas_memory_coherent_async(int uplo, int memflag, size_t M, size_t N,
                                 void* A, size_t ld, size_t elsize);
int xkblas_memory_syncall(void);
int xkblas_memory_invalidate(const void* A);
int xkblas_memory_invalidate_caches(void);
int xkblas_memory_free(void);

/* ---- level-3 operations (reference blas/zxkblas.h:45-151, generated for
 * s/d/c/z).  Scalars by pointer; CBLAS enum ints; int dims and ld. -------- */
#define XKBLAS_DECL_OPS(p, T, R)                                               \
  int xkblas_##p##gemm_async(int transA, int transB, int M, int N, int K,      \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##gemm_native(int transA, int transB, int M, int N, int K,     \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##gemmt_async(int uplo, int transA, int transB, int N, int K,  \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##gemmt_native(int uplo, int transA, int transB, int N, int K, \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##trsm_async(int side, int uplo, int transA, int diag, int N,  \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##trsm_native(int side, int uplo, int transA, int diag, int N, \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##trmm_async(int side, int uplo, int transA, int diag, int N,  \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##trmm_native(int side, int uplo, int transA, int diag, int N, \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##symm_async(int side, int uplo, int M, int N, const T* alpha, \
      const T* A, int LDA, const T* B, int LDB, const T* beta, T* C, int LDC); \
  int xkblas_##p##symm_native(int side, int uplo, int M, int N,                \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##syrk_async(int uplo, int trans, int N, int K,                \
      const T* alpha, const T* A, int LDA, const T* beta, T* C, int LDC);      \
  int xkblas_##p##syrk_native(int uplo, int trans, int N, int K,               \
      const T* alpha, const T* A, int LDA, const T* beta, T* C, int LDC);      \
  int xkblas_##p##syr2k_async(int uplo, int trans, int N, int K,               \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##syr2k_native(int uplo, int trans, int N, int K,              \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);

/* hemm/herk/her2k exist for c and z only (reference gen_internal_register.sh:10-20) */
#define XKBLAS_DECL_HE_OPS(p, T, R)                                            \
  int xkblas_##p##hemm_async(int side, int uplo, int M, int N, const T* alpha, \
      const T* A, int LDA, const T* B, int LDB, const T* beta, T* C, int LDC); \
  int xkblas_##p##hemm_native(int side, int uplo, int M, int N,                \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##herk_async(int uplo, int trans, int N, int K,                \
      const R* alpha, const T* A, int LDA, const R* beta, T* C, int LDC);      \
  int xkblas_##p##herk_native(int uplo, int trans, int N, int K,               \
      const R* alpha, const T* A, int LDA, const R* beta, T* C, int LDC);      \
  int xkblas_##p##her2k_async(int uplo, int trans, int N, int K,               \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const R* beta, T* C, int LDC);                                           \
  int xkblas_##p##her2k_native(int uplo, int trans, int N, int K,              \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const R* beta, T* C, int LDC);

XKBLAS_DECL_OPS(s, float, float)
XKBLAS_DECL_OPS(d, double, double)
XKBLAS_DECL_OPS(c, Complex32_t, float)
XKBLAS_DECL_OPS(z, Complex64_t, double)
XKBLAS_DECL_HE_OPS(c, Complex32_t, float)
XKBLAS_DECL_HE_OPS(z, Complex64_t, double)

/* ---- Cholesky factorization (reference blas/zpotrf.c:46, a tile driver
 * outside the reference's public headers): A = L L^H (CblasLower) or U^H U
 * (CblasUpper) in place on the host-resident matrix, asynchronous like the
 * level-3 calls (memory_coherent_async + sync make A final on the host).
 * Returns -2 (uplo), -5 (N), -8 (LDA) as the reference does.
 * xkblas_potrf_info: after the factorization, the first column (1-based)
 * whose pivot was not positive, 0 if A was positive definite (waits for the
 * device). ------------------------------------------------------------- */
int xkblas_spotrf_async(int uplo, int N, float* A, int LDA);
int xkblas_dpotrf_async(int uplo, int N, double* A, int LDA);
int xkblas_cpotrf_async(int uplo, int N, Complex32_t* A, int LDA);
int xkblas_zpotrf_async(int uplo, int N, Complex64_t* A, int LDA);
int xkblas_potrf_info(void);

/* ---- LU factorization without pivoting (reference blas/zgetrf_nopiv.c:
 * 48-101, a tile driver the reference builds but does not declare here).
 * A = L U in place, L unit lower, U upper; square matrices only (M == N,
 * else -2).  Stable for diagonally dominant or otherwise well-conditioned
 * leading blocks, as any LU without pivoting.  The factors become final on
 * the host after memory_coherent_async + sync; xkblas_getrf_info then gives
 * the first zero pivot (1-based, 0 = none). */
int xkblas_sgetrf_nopiv_async(int M, int N, float* A, int LDA);
int xkblas_dgetrf_nopiv_async(int M, int N, double* A, int LDA);
int xkblas_cgetrf_nopiv_async(int M, int N, Complex32_t* A, int LDA);
int xkblas_zgetrf_nopiv_async(int M, int N, Complex64_t* A, int LDA);
int xkblas_getrf_info(void);

/* ---- synchronous forms: _async + memory_coherent_async on the output
 * (its written triangle for gemmt/syrk/herk/syr2k/her2k) + xkblas_sync +
 * xkblas_memory_invalidate_caches -- the sequence the reference's F77
 * wrapper runs for every BLAS call (blas/zlibxkblas_wrapper.c:67-73), as C
 * entry points with the _async argument lists.  Return 0, -i for the i-th
 * bad argument, or a positive errno from the runtime. -------------------- */
#define XKBLAS_DECL_SYNC_OPS(p, T, R)                                          \
  int xkblas_##p##gemm_sync(int transA, int transB, int M, int N, int K,       \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##gemmt_sync(int uplo, int transA, int transB, int N, int K,   \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);                                           \
  int xkblas_##p##trsm_sync(int side, int uplo, int transA, int diag, int N,   \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##trmm_sync(int side, int uplo, int transA, int diag, int N,   \
      int NRHS, const T* alpha, const T* A, int LDA, T* B, int LDB);           \
  int xkblas_##p##symm_sync(int side, int uplo, int M, int N, const T* alpha,  \
      const T* A, int LDA, const T* B, int LDB, const T* beta, T* C, int LDC); \
  int xkblas_##p##syrk_sync(int uplo, int trans, int N, int K,                 \
      const T* alpha, const T* A, int LDA, const T* beta, T* C, int LDC);      \
  int xkblas_##p##syr2k_sync(int uplo, int trans, int N, int K,                \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const T* beta, T* C, int LDC);
#define XKBLAS_DECL_HE_SYNC_OPS(p, T, R)                                       \
  int xkblas_##p##hemm_sync(int side, int uplo, int M, int N, const T* alpha,  \
      const T* A, int LDA, const T* B, int LDB, const T* beta, T* C, int LDC); \
  int xkblas_##p##herk_sync(int uplo, int trans, int N, int K,                 \
      const R* alpha, const T* A, int LDA, const R* beta, T* C, int LDC);      \
  int xkblas_##p##her2k_sync(int uplo, int trans, int N, int K,                \
      const T* alpha, const T* A, int LDA, const T* B, int LDB,                \
      const R* beta, T* C, int LDC);

XKBLAS_DECL_SYNC_OPS(s, float, float)
XKBLAS_DECL_SYNC_OPS(d, double, double)
XKBLAS_DECL_SYNC_OPS(c, Complex32_t, float)
XKBLAS_DECL_SYNC_OPS(z, Complex64_t, double)
XKBLAS_DECL_HE_SYNC_OPS(c, Complex32_t, float)
XKBLAS_DECL_HE_SYNC_OPS(z, Complex64_t, double)

/* ---- added: per-call counters (reference XKBLAS_VERBOSE statistics,
 * blas/xkblas.c:1635-1700, as a queryable record) ------------------------ */
typedef struct xkblas_stats_t {
  uint64_t calls;          /* level-3 calls accepted */
  uint64_t kernels;        /* kernels launched by the library */
  uint64_t h2d_bytes;      /* bytes copied host -> device */
  uint64_t d2h_bytes;      /* bytes copied device -> host */
  uint64_t tile_hits;      /* tiles found valid on the device */
  uint64_t tile_misses;    /* tiles fetched from the host */
  uint64_t ozaki_calls;    /* contractions run in the Ozaki INT8 form (all of
                              the process's, counted on the device; reading
                              the statistics waits for the device) */
  uint64_t ozaki_moduli;   /* sum over those calls of the moduli used */
  double   flops;          /* algorithmic flops (reference blas/flops.h) */
  uint64_t batches;        /* deferred-call batches run as one executor launch */
  uint64_t batched_calls;  /* calls those batches held */
  uint64_t evictions;      /* matrices evicted under the cache limit */
} xkblas_stats_t;
int  xkblas_get_stats(xkblas_stats_t* st);
void xkblas_reset_stats(void);
/* Last device-side error word (0 = none; XKB_DEV_* of xkb_cuda.h), read and
 * cleared.  When a kernel recorded one, xkblas_sync() returns XKB_ETIMEDOUT
 * (-5) for a bounded wait that gave up, XKB_EFAULT (-7) for a refused
 * out-of-bounds access, XKB_ECUDA (-2) otherwise; the context stays usable. */
int  xkblas_last_device_error(void);

/* ---- added: event trace as the CSV tables of the reference's trace
 * converter (bin/ukilli.cpp:875-1115; the reference records with
 * KAAPI_RECORD_TRACE=1, kaapi/kaapi_trace_lib.c:754-840, and converts post
 * mortem).  Recording is off by default; XKBLAS_TRACE_DIR=<dir> turns it on
 * at initialisation and writes the tables into <dir> at the last
 * xkblas_finalize.  Tables (same headers and columns as the converter):
 *   kern.csv      kernel launches: Resource,Type,Stream,Push,Start,End,
 *                 Duration,Name ("<call>/<kernel>"),TaskId; an executor
 *                 launch ("batch/k_sched") is followed by one row per call
 *                 ("batch/<call>#<i>", ending at the call's completion)
 *   cpy.csv       host<->device copies: ...,Size (bytes),Dir (1 H2D, 2 D2H)
 *   call.csv      API calls: Resource,Level,Start,End (the xkblas_sync that
 *                 completed it),Duration,Name,NParam,Param0..Param15
 *   task.csv      API calls as host tasks (entry to return)
 *   parallel.csv  the host threads and the GPU over the recording
 * Times are seconds since recording started; device times come from CUDA
 * events on the launching stream.  Export drains what it wrote.  Record
 * eager execution only: inside a caller's CUDA-graph capture the recorder's
 * events and copies would become part of the graph. */
int      xkblas_trace_record(int on);           /* returns the previous state */
int      xkblas_trace_export(const char* dir);  /* 0, EINVAL or EIO */
uint64_t xkblas_trace_dropped(void);            /* events not recorded (table full) */

#ifdef __cplusplus
}
#endif
#endif /* XKBLAS_B200_XKBLAS_H */
