// runtime.hpp -- host runtime of libxkblas.so: the device-resident tile
// directory (replacing the reference's XKaapi software DSM,
// kaapi/kaapi_memory.c:2553-2778), streams, and the per-call statistics.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "evlog.hpp"
#include "xkb_cuda.h"
#include "xkblas.h"

namespace xkbrt {

// Per-tile state bits of the directory.
enum : uint8_t {
  kDevValid = 1,   // device copy holds the current value
  kHostStale = 2,  // device copy is newer than the host copy
};

// One user matrix known to the library (reference: xkblas_matrix_descr,
// blas/common.gen:167-187; created on first touch like
// xkblas_init_matrix_handle, blas/xkblas.c:458-510).  Unlike the reference,
// the device copy is ONE column-major buffer for the whole matrix; tiles are
// the unit of coherence (valid / dirty bits) and of host<->device copies.
// A CUDA event held by every descriptor whose results it marks; destroyed
// with its last holder (CUDA releases a recorded event once it completed).
struct SharedEvent {
  cudaEvent_t e = nullptr;
  ~SharedEvent() {
    if (e) cudaEventDestroy(e);
  }
};
using EventRef = std::shared_ptr<SharedEvent>;
// A fresh event (nullptr if CUDA cannot create one).
EventRef new_event_ref();

struct Desc {
  void* host = nullptr;
  size_t M = 0, N = 0, ld = 0, esz = 0;   // host view
  void* dev = nullptr;
  size_t dld = 0;                         // device leading dimension (elements)
  size_t mb = 0, nb = 0, mt = 0, nt = 0;  // tile grid
  std::vector<uint8_t> st;                // mt*nt tile states, column major
  bool registered_init = false;           // handle initialised (isinit)
  uint8_t pend = 0;                       // deferred calls: 1 read, 2 written
  bool managed = false;                   // CUDA managed memory: used in place, never copied
  size_t bytes = 0;                       // device buffer size (counted against the cache limit)
  uint64_t last_use = 0;                  // LRU stamp: the runtime's use clock at the last touch
  uint64_t epoch = 0;                     // API call that last touched it (never evicted by it)
  // rectangles finished on the compute stream, in the order they finish:
  // rows [r0, r1) x columns [c0, c1) are final once `ev` fired.  Together
  // they cover [0, max r1) x [0, max c1) once.  Set by the panel
  // contraction (one column panel each), the row-block / column-panel
  // contraction (one rectangle per landed block) and an executor batch (the
  // whole matrix); lets coherence copy results back as soon as their
  // producer is done instead of after all queued work.  Cleared by any write
  // that does not set it.
  struct Ready {
    size_t r0, r1, c0, c1;
    std::shared_ptr<struct SharedEvent> ev;
  };
  std::vector<Ready> ready;
  std::string name;
  uint8_t& tile(size_t i, size_t j) { return st[i + j * mt]; }
};

// Per-operation counters ("dgemm", "ztrsm", ...): accepted calls and their
// algorithmic flops (reference per-task-type statistics printed at
// finalize under XKBLAS_VERBOSE, blas/xkblas.c:1635-1700).
struct OpCount {
  uint64_t calls = 0;
  double flops = 0;
};

struct Stats {
  uint64_t calls = 0, h2d = 0, d2h = 0, hits = 0, misses = 0, evictions = 0;
  uint64_t ozaki_calls = 0, ozaki_moduli = 0;  // the device counters at the last reset
  double flops = 0;
};

struct Runtime {
  std::recursive_mutex mu;
  int refcount = 0;
  bool ready = false;
  int device = 0;
  cudaStream_t s_comp = nullptr, s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t ev_pool[64];
  bool alloc_unsynced = false;  // device buffers allocated since the last host->device copy
  bool h2d_unsynced = false;    // copies the compute stream does not wait for yet
  int ev_next = 0;
  std::unordered_map<const void*, Desc*> descs;
  size_t nb_param = 0;        // preset tile size (0 = automatic)
  size_t prec_param = 8;
  int math = XKBLAS_DEFAULT_MATH;  // process default (XKBLAS_DEFAULT_MATH); per thread: ThreadCtx
  std::vector<cudaEvent_t> ev_free;  // sync events of ended threads, reused
  int ozaki_moduli = 0;       // 0 = automatic
  bool unified = false;       // xkblas_malloc_unified returns managed memory (XKBLAS_UNIFIED)
  // contractions smaller than this stay plain: XKBLAS_OZAKI_MIN_DIM, else the
  // tuning key ozaki_min_dim (read per call), else 2048; see ozaki_min_dim()
  long ozaki_min_env = -1;
                              // (measured crossover on a B200, autotune.py)
  Stats stats;
  std::map<std::string, OpCount> per_op;  // since init (XKBLAS_VERBOSE report)
  int verbose = 0;                        // XKBLAS_VERBOSE level
  int sticky_error = 0;
  // Deferred calls: async GEMM / left-TRSM calls queued as one batch for the
  // persistent tile-task executor (XKBLAS_BATCH=0 disables).  The queue is
  // launched at the next coherence point (memory_coherent_async, sync, a
  // buffer release), before any call that is not deferred, and before a call
  // that touches what a queued call writes or writes what one reads.
  bool batch_on = true;
  size_t batch_max = 8192;
  // queued calls are launched once their operands reach batch_flush_mb
  // (tuning key, default 2048) MiB, so that the executor starts while later
  // calls' operands are still uploading; XKBLAS_BATCH_FLUSH_MB overrides
  size_t batch_flush_env = 0;
  size_t pend_bytes = 0;  // operand bytes of the queued calls
  std::vector<xkb_batch_op> pending;
  std::vector<Desc*> pend_descs;  // buffers the queued calls touch (Desc::pend set)
  uint64_t batches = 0, batched_calls = 0;
  int* d_potrf_info = nullptr;  // device word for the last factorization
  // Device cache limit (reference: XKBLAS_CACHE_LIMIT -> KAAPI_CUDA_CACHE_LIMIT,
  // percent of device memory, default 98, clamped to [1, 100],
  // kaapi/kaapi_impl.c:208,311-316; kaapi_plugin_cuda.c:2306).  Matrix
  // buffers beyond it evict the least recently used matrices not touched by
  // the current call (dirty tiles written back first).
  size_t cache_limit = 0, dev_bytes = 0;
  uint64_t use_clock = 0, call_epoch = 0;
};

Runtime& rt();
int ensure_init();  // lazily initialises (returns XKB_* code)

// One context per calling thread (reference: an xkblas_context_t per
// pthread, blas/xkblas.c:224-243): its math mode (the process default until
// the thread sets one, blas/xkblas.c:356-365) and the events its
// xkblas_sync waits for.  The events return to a pool when the thread ends.
struct ThreadCtx {
  int math = -1;                    // -1: the process default (Runtime::math)
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // compute, h2d, d2h
  ~ThreadCtx();
};
ThreadCtx& tctx();
int thread_math();  // the calling thread's mode
cudaEvent_t next_event();

// Directory operations (caller holds rt().mu).
Desc* get_desc(const void* host, size_t M, size_t N, size_t ld, size_t esz, size_t NB,
               int* err);
// Make the tiles covering rows [r0,r1) x cols [c0,c1) valid on the device
// (H2D on the copy stream; the compute stream then waits).
// wait = false: the compute stream is not yet made to wait for the copies;
// the caller calls comp_wait_h2d() before its next launch.
int make_valid(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1, bool wait = true);
// Make the compute stream wait for the copies issued by make_valid(.., false).
int comp_wait_h2d();
// Mark a region as written by the compute stream (device newer than host).
void mark_written(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1, int uplo);
// Mark a region as produced on the device without reading the host copy.
void mark_full_overwrite(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1);
int coherent(Desc* d, int uplo, int memflag);
// Column-panel upload: for each panel [bounds[p], bounds[p+1]) and every
// (matrix, row count) in `ds`, copy the panel's columns of the tiles (covering
// rows [0, row count)) that are not valid on the device, in panel order, and
// record ev[p] on the copy stream after panel p.  The compute stream is NOT
// made to wait: the caller waits per panel.  The tiles become valid.
int make_valid_panels(const std::vector<std::pair<Desc*, size_t>>& ds,
                      const std::vector<long>& bounds, std::vector<cudaEvent_t>& ev);
// Row-block / column-panel upload for a contraction with inner dimension K:
// row block i = rows [rb[i], rb[i+1]) of op(A) (rows of the stored `da`, or
// its columns when a_trans), column panel j = columns [cb[j], cb[j+1]) of
// the stored `db` (K rows).  The parts of those blocks whose tiles are not
// valid on the device are copied in the order `seq` names (>= 0: panel,
// < 0: row block -1 - seq), and ev_a[i] / ev_b[j] recorded on the copy
// stream once the block has landed.  The compute stream is NOT made to wait.
// The tiles become valid.
int make_valid_blocks(Desc* da, bool a_trans, size_t K, const std::vector<long>& rb, Desc* db,
                      const std::vector<long>& cb, const std::vector<int>& seq,
                      std::vector<cudaEvent_t>& ev_a, std::vector<cudaEvent_t>& ev_b);
// The Ozaki crossover in effect (min(M, N, K) at or above it: tensor-op mode
// uses the Ozaki form).
long ozaki_min_dim();
// Launch the deferred calls (caller holds rt().mu); returns an XKB_* code.
int flush_pending();
// Launch a list of calls on the compute stream: one call through the
// whole-matrix kernels, more as one executor batch.
int launch_ops(const std::vector<xkb_batch_op>& ops);
// Queue a call for the executor; reads: the buffers it reads (nullptr
// entries ignored), w: the buffer it writes.  Flushes first on a conflict.
int defer_op(const xkb_batch_op& o, Desc* r0, Desc* r1, Desc* r2, Desc* w);
void drop_desc(Desc* d);
void* dev_ptr(const Desc* d, size_t r, size_t c);

size_t auto_tilesize(xkblas_kernel_t kernel, size_t M, size_t N, size_t K);

// Statistics of an accepted level-3 call (caller holds rt().mu).
void count_call(const char* op);
void add_flops(const char* op, double flops);

// Scratch device memory for a call, stream-ordered on the compute stream.
void* scratch_alloc(size_t bytes);
void scratch_free(void* p);

}  // namespace xkbrt
