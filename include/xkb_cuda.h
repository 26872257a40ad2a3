/*
 * xkb_cuda.h -- the thin C ABI between the host runtime and the sm_100a
 * kernels of libxkblas.so.  Plain pointers (DEVICE addresses) and sizes; the
 * stream is a cudaStream_t passed as void* (NULL = the library's stream).
 *
 * It replaces the reference's per-tile GPU task bodies, which hand each tile
 * to cuBLAS:
 *   xkb_cuda_gemm       <- blas/ztask_gemm.c:176-216   (cublasZgemm, :206),
 *                          blas/ztask_gemmt.c:213, ztask_syrk.c:130,
 *                          ztask_herk.c:130, ztask_syr2k.c:138,
 *                          ztask_her2k.c:138 (triangle-masked variants)
 *   xkb_cuda_trsm       <- blas/ztask_trsm.c:162-180   (cublasZtrsm, :172)
 *   xkb_cuda_trmm       <- blas/ztask_trmm.c:156       (cublasZtrmm)
 *   xkb_cuda_symm       <- blas/ztask_symm.c:133, ztask_hemm.c:132
 *   xkb_cuda_ozaki_gemm: no counterpart in the
 *                          reference (FP64 contraction on INT8 tensor cores).
 * Every function returns 0 or a negative XKB_E* code; nothing aborts.
 */
#ifndef XKB_CUDA_H
#define XKB_CUDA_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* element types */
#define XKB_S 0   /* float            */
#define XKB_D 1   /* double           */
#define XKB_C 2   /* float complex    */
#define XKB_Z 3   /* double complex   */
/* op codes */
#define XKB_OP_N 0
#define XKB_OP_T 1
#define XKB_OP_C 2
/* triangle masks on C */
#define XKB_FULL 0
#define XKB_LOWER 1
#define XKB_UPPER 2

/* error codes */
#define XKB_OK 0
#define XKB_EINVAL -1     /* bad argument (size, alignment, op)         */
#define XKB_ECUDA -2      /* CUDA runtime error                          */
#define XKB_ENOMEM -3     /* device allocation failed                    */
#define XKB_ENODEV -4     /* no usable sm_100 device                     */
#define XKB_ETIMEDOUT -5  /* a bounded device-side wait gave up          */
#define XKB_ERANGE -6     /* size beyond a documented maximum            */
#define XKB_EFAULT -7     /* a device-side bounds check refused an access */

/* device error words (xkb_cuda_take_device_error, xkblas_last_device_error):
 * the first kernel problem recorded since the last read */
#define XKB_DEV_FULL_WAIT 1   /* a consumer gave up waiting for data / a task */
#define XKB_DEV_EMPTY_WAIT 2  /* a producer gave up waiting for a free stage  */
#define XKB_DEV_MMA_WAIT 3    /* a tensor-core completion wait gave up        */
#define XKB_DEV_ACC_WAIT 4    /* an epilogue gave up waiting for its results  */
#define XKB_DEV_BOUNDS 5      /* a bounds check refused an access             */

typedef struct xkb_gemm_args {
  int dtype;          /* XKB_S/D/C/Z                                          */
  int opA, opB;       /* XKB_OP_N/T/C                                         */
  int M, N, K;        /* C is M x N, op(A) M x K, op(B) K x N                 */
  const void* A; long lda;   /* column-major device matrices               */
  const void* B; long ldb;
  void* C; long ldc;
  double alpha[2];    /* (re, im); im ignored for real types                  */
  double beta[2];
  int uplo;           /* XKB_FULL / XKB_LOWER / XKB_UPPER: written part of C  */
  int herm_diag;      /* complex: force Im(C(i,i)) = 0 (herk/her2k contract)  */
  long diag;          /* C(i,j) lies on the diagonal when i + diag == j       */
} xkb_gemm_args;

/* C <- alpha*op(A)*op(B) + beta*C on the masked part of C, FP64 DMMA
 * tensor cores (float storage computed in double and rounded once). */
int xkb_cuda_gemm(const xkb_gemm_args* a, void* stream);

/* Triangular solve, all side/uplo/trans/diag cases:
 *   side L: B <- alpha * op(A)^-1 * B   (A is M x M)
 *   side R: B <- alpha * B * op(A)^-1   (A is N x N)
 * FP64 diagonal-block substitution + DMMA GEMM updates; when ozaki > 0 and
 * dtype is XKB_D/XKB_Z, updates whose three dimensions are all >= ozaki run
 * in the Ozaki INT8 form. */
int xkb_cuda_trsm(int dtype, int side, int uplo, int trans, int diag, int M,
                  int N, const double* alpha, const void* A, long lda, void* B,
                  long ldb, int ozaki, void* stream);

/* B <- alpha * op(A) * B (side L) or alpha * B * op(A) (side R): one
 * product with the triangle materialised; when ozaki > 0 and dtype is
 * XKB_D/XKB_Z, a product whose three dimensions are all >= ozaki runs in the
 * Ozaki INT8 form. */
int xkb_cuda_trmm(int dtype, int side, int uplo, int trans, int diag, int M,
                  int N, const double* alpha, const void* A, long lda, void* B,
                  long ldb, int ozaki, void* stream);

/* C <- alpha*A*B + beta*C (side L) or alpha*B*A + beta*C, A symmetric
 * (herm = 0) or Hermitian (herm = 1) stored in its uplo triangle; ozaki as
 * for xkb_cuda_trmm. */
int xkb_cuda_symm(int dtype, int herm, int side, int uplo, int M, int N,
                  const double* alpha, const void* A, long lda, const void* B,
                  long ldb, const double* beta, void* C, long ldc, int ozaki,
                  void* stream);

/* C <- beta*C on the masked part (used for K == 0 / alpha == 0). */
int xkb_cuda_scale(int dtype, int M, int N, const double* beta, void* C,
                   long ldc, int uplo, int herm_diag, long diag, void* stream);

/* Ozaki scheme II: FP64 (or complex128) C <- alpha*op(A)*op(B) + beta*C
 * computed as nmod INT8 tensor-core products modulo pairwise coprime
 * moduli (tcgen05, exact INT32 accumulation) and a Chinese-remainder
 * reconstruction.  nmod > 0 uses that many moduli (2..16).  nmod = 0
 * chooses the count on the device from the operands: with rho_i =
 * sqrt(nnz) ||row i of op(A)||_2 / ||row i||_1 and sigma_j the same for
 * column j of op(B), the smallest count (15 or 16, at least the tuning
 * table's count for K's band) whose exponent budget H meets
 * 53 + log2(2.31 max rho max sigma); when even 16 moduli cannot, the call
 * is computed by the plain FP64 kernel instead (the choice is made and
 * acted on on the device: no host synchronisation).
 * uplo/herm_diag/diag mask C as in xkb_gemm_args.  dtype XKB_D or XKB_Z. */
int xkb_cuda_ozaki_gemm(const xkb_gemm_args* a, int nmod, void* stream);

/* Column-panel form of the real Ozaki contraction (C full): op(A) converted
 * once; for each panel p of columns [bounds[p], bounds[p+1]) of op(B) and C
 * (bounds[0] = 0, bounds[npanel] = N) the stream waits on the CUDA event
 * wait_ev[p] (if not NULL), the panel is computed, and done_ev[p] (if not
 * NULL) is recorded.  Lets a caller overlap the panels' host<->device copies
 * with the arithmetic.  No counterpart in the reference. */
int xkb_cuda_ozaki_gemm_panels(const xkb_gemm_args* a, int nmod, void* stream, int npanel,
                               const long* bounds, void* const* wait_ev,
                               void* const* done_ev);

/* Row-block and column-panel form of the real Ozaki contraction (C full):
 * op(A) in row blocks [rb[i], rb[i+1]) (rb[0] = 0, rb[nr] = M), op(B) and C
 * in column panels [cb[j], cb[j+1]) (cb[0] = 0, cb[nc] = N); interior
 * bounds multiples of 256.  seq[0 .. nr+nc) is the order in which the
 * blocks land: seq[k] >= 0 is column panel seq[k] (the stream first waits on
 * b_ev[seq[k]], if not NULL), seq[k] < 0 row block -1-seq[k] (waits on
 * a_ev[-1-seq[k]]); row blocks in increasing order, panels too.  At the k-th
 * landing the block is converted and multiplied with every block of the
 * other operand landed before it, which completes the rectangle of C
 * [row block] x [0, columns landed) or [0, rows landed) x [panel];
 * done_ev[k] (if not NULL) is recorded once that rectangle is final (an
 * empty rectangle when nothing of the other operand has landed yet).  Lets
 * a caller start the arithmetic, and the copy-back of C, before all of
 * op(A) crossed the host link.  Results are those of
 * xkb_cuda_ozaki_gemm_panels with the same count.  No counterpart in the
 * reference. */
int xkb_cuda_ozaki_gemm_blocks(const xkb_gemm_args* a, int nmod, void* stream, int nr,
                               const long* rb, int nc, const long* cb, const int* seq,
                               void* const* a_ev, void* const* b_ev, void* const* done_ev);

/* The same real (XKB_D) Ozaki contraction as xkb_cuda_ozaki_gemm, for
 * callers that cannot allocate device memory at call time (a process whose
 * free GPU memory is held by its own caching allocator, a loop that must not
 * risk an allocation stalling or failing mid-step).  No counterpart in the
 * reference.  Allocates nothing: its scratch is one fixed device array
 * inside the library (about 12.6 MiB per GPU that loads it, held until the
 * process exits).  M, N, K <= 512, otherwise XKB_ERANGE; nmod as above.
 * Every call uses the same array, so calls that overlap on the GPU race:
 * serialise them.  The array and this path's kernels are placed in device
 * memory by xkblas_init() (for its device) or else by the first call on a
 * device, which looks the array up once per device (again after a
 * cudaDeviceReset); make that call, or xkblas_init(), before handing the
 * free device memory to another allocator and before any stream capture. */
int xkb_cuda_ozaki_gemm_noalloc(const xkb_gemm_args* a, int nmod, void* stream);

/* Number of moduli the Ozaki path uses for contraction length K when the
 * count is fixed by K alone (the column-panel form with nmod = 0): the
 * tuning table's count for K's band, else the smallest count keeping
 * H - log2(K)/2 >= 53 bits; 0 if K is beyond the exact-INT32 limit. */
int xkb_ozaki_default_moduli(long K);

/* Counters of the Ozaki contractions run on the device since the last reset:
 * out[0] calls, out[1] the moduli counts summed, out[2] calls the data rule
 * sent to the plain FP64 kernel; *last (if not NULL) the latest call's count
 * (0: plain kernel, -1: none yet).  reset != 0 clears them afterwards.
 * Waits for the device.  No counterpart in the reference. */
int xkb_ozaki_counts(unsigned long long* out, int* last, int reset);

/* Per-call trace (off by default): when enabled, contractions record CUDA
 * events around their phases on their own stream; xkb_trace_take() waits for
 * the recorded events and returns up to `max` completed records, oldest
 * first (a fixed ring of 256 records; older ones are overwritten). */
typedef struct xkb_trace_rec {
  char op[16];        /* "dmma_gemm", "ozaki_gemm"                         */
  int dtype, M, N, K; /* shape of the contraction                          */
  int nmod;           /* Ozaki moduli (0 for the plain path)               */
  float ms_total;     /* whole call on the device                          */
  float ms_convert;   /* Ozaki: scaling + residue planes of A and B        */
  float ms_gemm;      /* Ozaki: INT8 tensor-core products (all moduli);
                         plain: the DMMA kernel                            */
  float ms_crt;       /* Ozaki: CRT reconstruction + alpha/beta            */
} xkb_trace_rec;
int xkb_trace_enable(int on);
int xkb_trace_take(xkb_trace_rec* out, int max);

/* Failure-detection check of the executor's bounded waits (no counterpart
 * in the reference): launches one executor CTA on a ready queue whose only
 * queued task is never written (a dependency that never resolves).  The CTA
 * gives up after wait_ms (1..10000), records XKB_DEV_FULL_WAIT and ends;
 * the context stays usable.  Returns once launched. */
int xkb_cuda_sched_wait_test(int wait_ms, void* stream);

/* Batched execution: a list of independent GEMM / left-TRSM calls on device
 * operands run as ONE persistent launch of tile tasks (a DAG with device
 * dependency counters; replaces the reference's task runtime,
 * kaapi/kaapi_task.c:1277-1327 and kaapi/kaapi_offload_device.c:463-683).
 * dtype XKB_D or XKB_Z; any leading dimension >= the row count, 8-byte
 * aligned bases (operands not 16-byte aligned are staged with 8-byte
 * copies).  Calls of one batch must not write memory another call of the
 * batch reads or writes. */
#define XKB_BATCH_GEMM 0
#define XKB_BATCH_TRSM 1
typedef struct xkb_batch_op {
  int kind;                    /* XKB_BATCH_GEMM / XKB_BATCH_TRSM            */
  int dtype;                   /* XKB_D / XKB_Z                              */
  int opA, opB;                /* gemm: XKB_OP_N/T/C                         */
  int side, uplo, trans, diag; /* trsm: side 0 (left) only; uplo XKB_LOWER/
                                  XKB_UPPER; trans XKB_OP_*; diag 1 = unit   */
  int M, N, K;                 /* gemm: C is M x N, K inner; trsm: B is M x N */
  const void* A; long lda;
  const void* B; long ldb;     /* gemm only                                  */
  void* C; long ldc;           /* gemm: C; trsm: B (solved in place)         */
  double alpha[2], beta[2];
} xkb_batch_op;
/* schedule: 0 = gemm tiles first, 1 = solve steps interleaved with gemm
 * tiles (dependent steps far apart in the claim order). */
int xkb_cuda_batch(const xkb_batch_op* ops, int nops, int schedule, void* stream);
/* After a batch: ms[i] = completion time of call i after the batch's first
 * task started (synchronises the device). */
int xkb_cuda_batch_latency(double* ms, int n);
/* Repeated batches: when an op list identical to one submitted recently
 * (same calls, pointers, sizes, scalars and schedule) comes again, the
 * batch is kept as a CUDA graph with its task list resident on the device,
 * and later submissions replay the graph (no host-side task construction,
 * no task upload).  At most 8 graphs / 2 GiB are kept (least recently used
 * dropped); XKBLAS_BATCH_GRAPHS=0 disables.  xkb_cuda_batch_cached returns
 * how many are held; xkb_cuda_batch_release drops them (synchronises). */
int xkb_cuda_batch_cached(void);
int xkb_cuda_batch_release(void);

/* Tuning table: choices measured on the device by the autotuner
 * (python -m xkblas_b200.autotune --out FILE; the runtime loads
 * XKBLAS_TUNE_FILE at init).  Keys (built-in default):
 *   gemm_big_min_tiles      whole-matrix GEMM uses 128-wide tiles when it has
 *                           at least this many of them (SM count)
 *   ozaki_min_dim           tensor-op mode uses Ozaki when min(M,N,K) >= (2048;
 *                           read per call; XKBLAS_OZAKI_MIN_DIM overrides)
 *   ozaki_moduli_k<=<K>     moduli count for contractions with inner size <= K
 *                           (the smallest band covering K; else the K rule)
 *   batch_schedule          executor claim order, 0 solves first / 1 gemms (0)
 *   batch_tile128_min_rows  executor: real gemm calls this tall use 128-row
 *                           tiles (96)
 *   oz_group_m              Ozaki INT8 GEMM raster: M tiles per group of the
 *                           persistent tile walk (8)
 *   oz_2cta                 Ozaki INT8 GEMM on CTA pairs (tcgen05 cta_group::2,
 *                           256 x 256 tiles) instead of single CTAs (0)
 *   ozaki_panel_cols        public async API: column width of the panels a
 *                           large Ozaki DGEMM streams through (1024; 2..32
 *                           panels, multiples of 256 columns)
 *   batch_flush_mb          public async API: queued calls are launched once
 *                           their operands reach this many MiB (2048), so the
 *                           executor overlaps the uploads of later calls
 * xkb_tune_load returns the number of entries read or XKB_EINVAL. */
int xkb_tune_set(const char* key, double value);
double xkb_tune_get(const char* key, double dflt);
int xkb_tune_load(const char* path);
int xkb_tune_clear(void);

/* Cholesky factorization in place: A = L L^H (XKB_LOWER) or U^H U
 * (XKB_UPPER), s/d/c/z, only the stored triangle read and written
 * (replaces the reference's tile driver blas/zpotrf.c:46-220).  d_info: a
 * device int (may be NULL) that receives the first column, 1-based, whose
 * pivot is not positive; it is not cleared here.  ozaki > 0 (XKB_D/XKB_Z):
 * trailing updates and panel-solve updates whose dimensions are all
 * >= ozaki use the Ozaki INT8 form (tensor-op mode); 0: plain FP64. */
int xkb_cuda_potrf(int dtype, int uplo, int N, void* A, long lda, int* d_info, int ozaki,
                   void* stream);

/* LU factorization without pivoting in place, A = L U (L unit lower, U
 * upper), square N x N, s/d/c/z (replaces the reference's tile driver
 * blas/zgetrf_nopiv.c:48-101).  d_info: a device int (may be NULL) that
 * receives the first zero pivot, 1-based; it is not cleared here.  ozaki as
 * for xkb_cuda_potrf. */
int xkb_cuda_getrf_nopiv(int dtype, int N, void* A, long lda, int* d_info, int ozaki,
                         void* stream);

/* Device error word written by bounded waits (0 = none); clears it. */
int xkb_cuda_take_device_error(void);

/* Kernels launched by the library since load (for launch accounting). */
uint64_t xkb_cuda_kernel_count(void);

#ifdef __cplusplus
}
#endif
#endif
