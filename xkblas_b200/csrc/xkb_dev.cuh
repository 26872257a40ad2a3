// xkb_dev.cuh -- device-side primitives shared by the sm_100a kernels:
// mbarrier pipeline, TMA (cp.async.bulk.tensor), bounded waits, launch
// accounting and the device error word.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "evlog.hpp"
#include "xkb_cuda.h"

namespace xkb {

// A bounded wait gives up after this many nanoseconds of %globaltimer
// (no correct launch of this library waits that long on one barrier).
constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s

// Device error word, one per translation unit (no relocatable device code);
// each unit registers a reader so xkb_cuda_take_device_error() sees all.
static __device__ int g_dev_error;

enum DevErr : int {  // the XKB_DEV_* words of xkb_cuda.h
  kErrNone = 0,
  kErrFullWait = XKB_DEV_FULL_WAIT,    // consumer gave up waiting for a TMA stage / a task
  kErrEmptyWait = XKB_DEV_EMPTY_WAIT,  // producer gave up waiting for a free stage
  kErrMmaWait = XKB_DEV_MMA_WAIT,      // tensor-core completion wait gave up
  kErrAccWait = XKB_DEV_ACC_WAIT,      // epilogue gave up waiting for the accumulator
  kErrBounds = XKB_DEV_BOUNDS,         // a bounds check refused an access
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void dev_error(int code) {
  atomicCAS(&g_dev_error, 0, code);
}

__device__ __forceinline__ bool dev_error_set() {
  return *reinterpret_cast<volatile int*>(&g_dev_error) != 0;
}

// ---- mbarrier ---------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on phase `parity`.  Returns false (and records `code`) when
// the time limit passes or another thread already recorded an error.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  uint64_t t0 = globaltimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0) {
      if (dev_error_set()) return false;
      if (globaltimer() - t0 > kWaitLimitNs) {
        dev_error(code);
        return false;
      }
    }
  }
}

// ---- TMA --------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch(const CUtensorMap* m) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}
// 2D tiled load into shared memory, completion counted on `bar` (bytes).
// The caller guarantees x * element size is a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* m, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace xkb

// Host-side helpers shared by the launch code (defined in runtime_cuda.cu).
namespace xkb {
typedef int (*ErrReader)();
int register_error_reader(ErrReader r);
// Reads and clears this unit's error word.
static int take_unit_error() {
  int v = 0, z = 0;
  if (cudaMemcpyFromSymbol(&v, g_dev_error, sizeof v) != cudaSuccess) return 0;
  if (v) cudaMemcpyToSymbol(g_dev_error, &z, sizeof z);
  return v;
}
static int g_unit_reader_registered = register_error_reader(&take_unit_error);
// Encode a 2-D tiled tensor map: rows x cols column-major with leading
// dimension ld (elements of `elem_bytes`), box bx (along rows) x by.
// Returns false if the driver entry point is missing or encoding fails.
bool encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes,
                    const void* base, uint64_t rows, uint64_t cols, uint64_t ld,
                    uint32_t bx, uint32_t by, CUtensorMapSwizzle swz);
// 3-D byte tensor (planes of rows x inner bytes), 128-byte swizzle, box
// (box_inner x box_rows x 1): the layout tcgen05 K-major operands use.
// planes of `rows` x `inner` bytes (inner contiguous), consecutive planes
// plane_rows * inner bytes apart (0: rows; a view of rows of larger planes)
bool encode_tmap_3d_u8(CUtensorMap* map, const void* base, uint64_t inner, uint64_t rows,
                       uint64_t planes, uint32_t box_inner, uint32_t box_rows,
                       uint64_t plane_rows = 0);
cudaStream_t resolve_stream(void* s);
// trace: begin a record (returns a slot or -1 when tracing is off) and mark
// phase boundaries 1..3 (3 = end) on the launching stream.
int trace_begin(const char* op, int dtype, int M, int N, int K, int nmod, cudaStream_t st);
void trace_mark(int slot, int k, cudaStream_t st);
void count_launch(int n = 1);
// A lazily created non-blocking stream with a fork and a join event, for
// work that is independent of what the caller's stream runs meanwhile
// (slot 0: the LU's column-panel solves, slots 1-3: the TRSM's groups of
// right-hand sides after the first, slots kHiStream and kHiStream2: the
// critical path of the blocked factorizations and the panel work beside it,
// slot kTrsmInvStream: the TRSM's inverses of pairs of diagonal blocks;
// slots from kHiStream on are created with the device's greatest stream
// priority so that their small launches are scheduled ahead of the trailing
// updates that run meanwhile).  s is nullptr if CUDA could not create it.
constexpr int kSideStreams = 7;
constexpr int kHiStream = 4, kHiStream2 = 5, kTrsmInvStream = 6;
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
const SideStream& side_stream(int slot);
// Fork: `side` waits for what `st` queued so far; returns `side`'s stream,
// or `st` itself (run in order) when there is no side stream.
cudaStream_t side_fork(const SideStream& side, cudaStream_t st);
// Join: `st` waits for what the forked stream queued; false on a CUDA error.
bool side_join(const SideStream& side, cudaStream_t forked, cudaStream_t st);
// n <= 8 reusable timing-free events of the calling library (created once),
// for dependencies between the side streams; nullptr if creation failed.
cudaEvent_t* dep_events();
// xkb_cuda_trsm with the choice to split many right-hand sides into two
// concurrent halves (off where the caller already runs solves side by side)
int trsm_entry(int dtype, int side, int uplo, int trans, int diag, int M, int N,
               const double* alpha, const void* A, long lda, void* B, long ldb, int ozaki,
               cudaStream_t st, bool split_rhs);
// xkb_cuda_gemm whose kernel runs only where the device word *run_if is
// non-zero (gemm_dmma.cu): the plain fallback of a data-chosen Ozaki call.
int gemm_if(const xkb_gemm_args* a, const int* run_if, cudaStream_t st);
double tune(const char* key, double dflt);   // tuning table (runtime_cuda.cu)
int tune_band(const char* prefix, long K);
int sm_count();
}  // namespace xkb
