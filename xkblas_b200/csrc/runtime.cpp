// runtime.cpp -- lifecycle, device-resident tile directory, coherence and the
// host-memory part of the xkblas.h API.
//
// The reference runs an XKaapi data-flow runtime with one host thread per
// GPU and an MSI-like software DSM (kaapi/kaapi_memory.c).  On one B200 the
// same contract is kept with much less machinery:
//   * every matrix has one device buffer (allocated stream-ordered from the
//     CUDA memory pool) and a tile directory of valid / dirty bits;
//   * missing tiles are fetched by pinned asynchronous 2-D copies on a copy
//     stream, coalesced into column panels; the compute stream waits on an
//     event, so transfers of later calls overlap earlier compute;
//   * xkblas_memory_coherent_async() queues device->host copies of the dirty
//     tiles on a second copy stream after the producing kernels;
//   * xkblas_sync() drains the three streams and reports device errors.
#include "runtime.hpp"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

namespace xkb {
void set_library_stream(cudaStream_t s);
int noalloc_prepare();  // ozaki.cu: places the scratch-free path's array and kernels
}

namespace xkbrt {

Runtime& rt() {
  static Runtime* r = new Runtime();  // never destroyed: safe at exit
  return *r;
}

static int cuda_ok(cudaError_t e) { return e == cudaSuccess ? XKB_OK : XKB_ECUDA; }
static void print_configuration(const cudaDeviceProp& prop);
static void print_statistics();

int ensure_init() {
  Runtime& R = rt();
  if (R.ready) return XKB_OK;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return XKB_ENODEV;
  }
  int dev = 0;
  if (const char* g = getenv("XKBLAS_GPUSET")) dev = atoi(g);
  if (dev < 0 || dev >= n) dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return XKB_ENODEV;
  if (prop.major != 10) return XKB_ENODEV;  // kernels are built for sm_100a only
  if (cudaSetDevice(dev) != cudaSuccess) return XKB_ENODEV;
  R.device = dev;
  // the fixed scratch array of xkb_cuda_ozaki_gemm_noalloc and that path's
  // kernels are placed in device memory now, while memory is free, not at
  // their first use (lazy module loading); a failure here is reported by
  // that entry point's first call instead
  if (xkb::noalloc_prepare() != XKB_OK) cudaGetLastError();
  {
    size_t fr = 0, total = 0;
    if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
      cudaGetLastError();
      total = prop.totalGlobalMem;
    }
    double pct = 98.0;
    if (const char* s = getenv("XKBLAS_CACHE_LIMIT")) pct = std::min(100.0, std::max(1.0, atof(s)));
    R.cache_limit = (size_t)((double)total * pct / 100.0);
    // extension: an absolute limit in MiB
    if (const char* s = getenv("XKBLAS_CACHE_LIMIT_MB"))
      if (atof(s) > 0) R.cache_limit = (size_t)(atof(s) * 1048576.0);
  }
  if (const char* dir = getenv("XKBLAS_TRACE_DIR"))
    if (*dir) xkblas_trace_record(1);
  if (cudaStreamCreateWithFlags(&R.s_comp, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&R.s_h2d, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&R.s_d2h, cudaStreamNonBlocking) != cudaSuccess)
    return XKB_ECUDA;
  for (auto& e : R.ev_pool)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return XKB_ECUDA;
  // keep freed pool memory cached: the directory allocates and frees often
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  xkb::set_library_stream(R.s_comp);
  if (const char* b = getenv("XKBLAS_BATCH")) R.batch_on = atoi(b) != 0;
  if (const char* u = getenv("XKBLAS_UNIFIED")) R.unified = R.unified || atoi(u) != 0;
  if (const char* t = getenv("XKBLAS_TILE_SIZE")) R.nb_param = (size_t)atol(t);
  else if (const char* b = getenv("XKBLAS_BLOC_SIZE")) R.nb_param = (size_t)atol(b);
  // element size the tile-size rule assumes (reference blas/xkblas.c:1483-1497;
  // an unknown value is reported and ignored instead of exiting)
  if (const char* p = getenv("XKBLAS_PRECISION")) {
    if (!strcmp(p, "float") || !strcmp(p, "real*4")) R.prec_param = 4;
    else if (!strcmp(p, "double") || !strcmp(p, "real*8")) R.prec_param = 8;
    else if (!strcmp(p, "complex32") || !strcmp(p, "complex*4")) R.prec_param = 8;
    else if (!strcmp(p, "complex64") || !strcmp(p, "complex*8")) R.prec_param = 16;
    else
      fprintf(stderr, "[XKBlas] XKBLAS_PRECISION must be float|real*4|double|real*8|"
                      "complex32|complex*4|complex64|complex*8; '%s' ignored\n", p);
  }
  if (const char* v = getenv("XKBLAS_VERBOSE")) R.verbose = std::max(0, atoi(v));
  if (const char* m = getenv("XKBLAS_DEFAULT_MATH")) {
    if (!strcmp(m, "TC") || !strcmp(m, "tensorcore")) R.math = XKBLAS_TENSOR_OP_MATH;
    else R.math = XKBLAS_DEFAULT_MATH;
  }
  // autotuner output (python -m xkblas_b200.autotune), then explicit settings
  if (const char* f = getenv("XKBLAS_TUNE_FILE")) xkb_tune_load(f);

  if (const char* s = getenv("XKBLAS_OZAKI_SLICES")) R.ozaki_moduli = atoi(s);
  if (const char* s = getenv("XKBLAS_OZAKI_MIN_DIM")) R.ozaki_min_env = atol(s);
  if (const char* s = getenv("XKBLAS_BATCH_FLUSH_MB")) R.batch_flush_env = (size_t)atol(s) << 20;
  R.ready = true;
  if (R.verbose) print_configuration(prop);
  return XKB_OK;
}

// XKBLAS_VERBOSE at initialisation: the configuration in effect (reference
// blas/xkblas.c:1578-1604 prints its runtime's description there).
static void print_configuration(const cudaDeviceProp& prop) {
  const Runtime& R = rt();
  const char* tf = getenv("XKBLAS_TUNE_FILE");
  printf("[XKBlas info]\n%s\n", xkblas_get_configuration());
  printf("device %d: %s, sm_%d%d, %d SMs, %.1f GiB, L2 %.0f MiB\n", R.device, prop.name,
         prop.major, prop.minor, prop.multiProcessorCount,
         (double)prop.totalGlobalMem / 1073741824.0, (double)prop.l2CacheSize / 1048576.0);
  printf("tile size: %s%zu, precision: %zu bytes\n", R.nb_param ? "" : "auto ",
         R.nb_param, R.prec_param);
  printf("math: %s; Ozaki moduli: %s%d, below %ld: plain\n",
         R.math == XKBLAS_TENSOR_OP_MATH ? "tensor-op (Ozaki INT8)" : "default (FP64 DMMA)",
         R.ozaki_moduli ? "fixed " : "data rule, 0 = ", R.ozaki_moduli, ozaki_min_dim());
  printf("deferred-call batches: %s, cache limit: %.0f MiB, unified: %s, tuning file: %s\n",
         R.batch_on ? "on" : "off", (double)R.cache_limit / 1048576.0, R.unified ? "on" : "off",
         tf && *tf ? tf : "none");
  printf("[XKBlas info]\n");
  fflush(stdout);
}

// XKBLAS_VERBOSE at finalisation: per-operation counts and flops, then the
// totals (reference blas/xkblas.c:1635-1700 prints per task type).
static void print_statistics() {
  Runtime& R = rt();
  unsigned long long oz[3] = {0, 0, 0};
  xkb_ozaki_counts(oz, nullptr, 0);
  printf("[XKBlas stats]\n");
  uint64_t calls = 0;
  double flops = 0;
  for (const auto& kv : R.per_op) {
    printf("\t[%12s]: count=%12llu, flops=%10e\n", kv.first.c_str(),
           (unsigned long long)kv.second.calls, kv.second.flops);
    calls += kv.second.calls;
    flops += kv.second.flops;
  }
  printf("\t[%12s]: count=%12llu, flops=%10e\n", "sum -->", (unsigned long long)calls, flops);
  if (R.verbose >= 2) {
    printf("\tkernels=%llu h2d_bytes=%llu d2h_bytes=%llu tile_hits=%llu tile_misses=%llu "
           "evictions=%llu batches=%llu batched_calls=%llu\n",
           (unsigned long long)xkb_cuda_kernel_count(), (unsigned long long)R.stats.h2d,
           (unsigned long long)R.stats.d2h, (unsigned long long)R.stats.hits,
           (unsigned long long)R.stats.misses, (unsigned long long)R.stats.evictions,
           (unsigned long long)R.batches, (unsigned long long)R.batched_calls);
    printf("\tozaki: contractions=%llu moduli=%llu plain_fallbacks=%llu\n", oz[0], oz[1], oz[2]);
  }
  fflush(stdout);
}

void count_call(const char* op) {
  Runtime& R = rt();
  R.stats.calls++;
  R.per_op[op].calls++;
}

void add_flops(const char* op, double flops) {
  Runtime& R = rt();
  R.stats.flops += flops;
  R.per_op[op].flops += flops;
}

ThreadCtx& tctx() {
  static thread_local ThreadCtx t;
  return t;
}

ThreadCtx::~ThreadCtx() {
  // no CUDA call at thread exit: the events go back to the runtime's pool
  if (!ev[0]) return;
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  for (cudaEvent_t e : ev) R.ev_free.push_back(e);
}

int thread_math() {
  const int m = tctx().math;
  return m < 0 ? rt().math : m;
}

// Events are recycled round-robin; 64 in flight is far more than any call
// sequence keeps outstanding between two stream waits.
EventRef new_event_ref() {
  auto r = std::make_shared<SharedEvent>();
  if (cudaEventCreateWithFlags(&r->e, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return r;
}

long ozaki_min_dim() {
  const Runtime& R = rt();
  return R.ozaki_min_env >= 0 ? R.ozaki_min_env : (long)xkb_tune_get("ozaki_min_dim", 2048.0);
}

cudaEvent_t next_event() {
  Runtime& R = rt();
  cudaEvent_t e = R.ev_pool[R.ev_next];
  R.ev_next = (R.ev_next + 1) % 64;
  return e;
}

static size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void* dev_ptr(const Desc* d, size_t r, size_t c) {
  return static_cast<char*>(d->dev) + (r + c * d->dld) * d->esz;
}

void* scratch_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocAsync(&p, std::max<size_t>(bytes, 256), rt().s_comp) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void scratch_free(void* p) {
  if (p) cudaFreeAsync(p, rt().s_comp);
}

static void free_desc_memory(Desc* d) {
  Runtime& R = rt();
  if (d->managed) {  // the caller's memory: only queued calls must run first
    flush_pending();
    d->dev = nullptr;
    return;
  }
  if (d->dev) {
    flush_pending();  // queued calls may use the buffer
    // D2H copies and kernels may still read the buffer: order the free
    // after both streams.
    cudaEvent_t e = next_event();
    cudaEventRecord(e, R.s_d2h);
    cudaStreamWaitEvent(R.s_comp, e, 0);
    cudaEvent_t e2 = next_event();
    cudaEventRecord(e2, R.s_h2d);
    cudaStreamWaitEvent(R.s_comp, e2, 0);
    cudaFreeAsync(d->dev, R.s_comp);
    d->dev = nullptr;
    R.dev_bytes -= std::min(R.dev_bytes, d->bytes);
    d->bytes = 0;
  }
}

void drop_desc(Desc* d) {
  Runtime& R = rt();
  free_desc_memory(d);
  R.descs.erase(d->host);
  delete d;
}

// Copy back every dirty tile of d synchronously (used before a descriptor
// must be rebuilt because a call reuses its pointer with another shape).
static int flush_sync(Desc* d) {
  int e = coherent(d, 0, 0);
  if (e) return e;
  return cuda_ok(cudaStreamSynchronize(rt().s_d2h));
}

// Evict one matrix: its dirty tiles go back to the host, later uploads of it
// wait for that copy, and its device buffer is released (stream ordered).
static void evict(Desc* d) {
  Runtime& R = rt();
  coherent(d, 0, 0);
  cudaEvent_t e = next_event();
  cudaEventRecord(e, R.s_d2h);
  cudaStreamWaitEvent(R.s_h2d, e, 0);
  R.stats.evictions++;
  drop_desc(d);
}

// Evict least recently used matrices not touched by the current call until
// `need` more bytes fit under the cache limit; false if that cannot be
// reached (the allocation then goes ahead above the limit if it can).
static bool evict_for(size_t need) {
  Runtime& R = rt();
  while (R.dev_bytes + need > R.cache_limit) {
    Desc* v = nullptr;
    for (auto& kv : R.descs) {
      Desc* d = kv.second;
      if (d->managed || !d->dev || d->epoch == R.call_epoch) continue;
      if (!v || d->last_use < v->last_use) v = d;
    }
    if (!v) return false;
    evict(v);
  }
  return true;
}

static int alloc_desc(Desc* d) {
  Runtime& R = rt();
  // a host matrix with contiguous columns keeps its layout on the device, so
  // that every transfer of it is one contiguous copy; otherwise columns are
  // padded to 128 bytes (the kernels take any leading dimension and repack
  // for TMA where they need to)
  const size_t align = std::max<size_t>(1, 128 / d->esz);
  d->dld = d->ld == d->M ? std::max<size_t>(d->M, 1) : round_up(std::max<size_t>(d->M, 1), align);
  const size_t bytes = d->dld * std::max<size_t>(d->N, 1) * d->esz;
  if (R.cache_limit) evict_for(bytes);
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, R.s_comp) != cudaSuccess) {
    cudaGetLastError();
    // out of device memory below the limit: evict what the call does not use
    // and try once more
    evict_for(R.cache_limit);
    if (cudaMallocAsync(&p, bytes, R.s_comp) != cudaSuccess) {
      cudaGetLastError();
      return XKB_ENOMEM;
    }
  }
  d->dev = p;
  d->bytes = bytes;
  R.dev_bytes += bytes;
  R.alloc_unsynced = true;  // the copy stream waits for it before its next copy
  return XKB_OK;
}

Desc* get_desc(const void* host, size_t M, size_t N, size_t ld, size_t esz, size_t NB,
               int* err) {
  Runtime& R = rt();
  *err = XKB_OK;
  auto it = R.descs.find(host);
  if (it != R.descs.end()) {
    Desc* d = it->second;
    if (d->ld == ld && d->esz == esz && M <= d->M && N <= d->N) {
      d->last_use = ++R.use_clock;
      d->epoch = R.call_epoch;
      return d;
    }
    // Same pointer, different geometry: write back, rebuild.
    if ((*err = flush_sync(d)) != XKB_OK) return nullptr;
    drop_desc(d);
  }
  Desc* d = new Desc();
  d->host = const_cast<void*>(host);
  d->M = M;
  d->N = N;
  d->ld = ld;
  d->esz = esz;
  d->mb = d->nb = std::max<size_t>(NB, 1);
  d->mt = std::max<size_t>(1, (M + d->mb - 1) / d->mb);
  d->nt = std::max<size_t>(1, (N + d->nb - 1) / d->nb);
  d->st.assign(d->mt * d->nt, 0);
  d->registered_init = true;
  d->last_use = ++R.use_clock;
  d->epoch = R.call_epoch;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, host) == cudaSuccess && pa.type == cudaMemoryTypeManaged) {
    // managed memory (xkblas_malloc_unified): the kernels use it in place;
    // its pages are moved to the device ahead of the first kernel
    d->managed = true;
    d->dev = const_cast<void*>(host);
    d->dld = ld;
    d->st.assign(d->mt * d->nt, kDevValid);
    if (cudaMemPrefetchAsync(host, ((N ? N - 1 : 0) * ld + M) * esz, R.device, R.s_comp) !=
        cudaSuccess)
      cudaGetLastError();  // advisory only
  } else {
    cudaGetLastError();
    if ((*err = alloc_desc(d)) != XKB_OK) {
      delete d;
      return nullptr;
    }
  }
  R.descs[host] = d;
  return d;
}

// Host <-> device copies of rows [r0,r1) x cols [c0,c1).  The device copy
// has a padded leading dimension; when the host block is contiguous (whole
// columns of a matrix with ld == M) and its columns are short, the transfer
// crosses the host link as one contiguous copy through a stream-ordered
// staging buffer and is re-pitched on the device: pitched copies of short
// rows move far below the link's bandwidth.
static int copy_h2d(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1) {
  Runtime& R = rt();
  if (r1 <= r0 || c1 <= c0) return XKB_OK;
  if (R.alloc_unsynced) {  // buffers allocated on the compute stream since the last copy
    cudaEvent_t e = next_event();
    cudaEventRecord(e, R.s_comp);
    cudaStreamWaitEvent(R.s_h2d, e, 0);
    R.alloc_unsynced = false;
  }
  const char* src = static_cast<const char*>(d->host) + (r0 + c0 * d->ld) * d->esz;
  char* dst = static_cast<char*>(dev_ptr(d, r0, c0));
  const size_t w = (r1 - r0) * d->esz;
  R.stats.h2d += w * (c1 - c0);
  const long long tv = xkb::evlog_copy_begin(R.s_h2d, w * (c1 - c0), 1);
  cudaError_t e;
  if (d->ld == d->dld && (r1 - r0 == d->M || c1 - c0 == 1))  // one contiguous range
    e = cudaMemcpyAsync(dst, src, ((c1 - c0 - 1) * d->ld + (r1 - r0)) * d->esz,
                        cudaMemcpyHostToDevice, R.s_h2d);
  else
    e = cudaMemcpy2DAsync(dst, d->dld * d->esz, src, d->ld * d->esz, w, c1 - c0,
                          cudaMemcpyHostToDevice, R.s_h2d);
  xkb::evlog_copy_end(tv, R.s_h2d);
  return cuda_ok(e);
}

static int copy_d2h(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1) {
  Runtime& R = rt();
  if (r1 <= r0 || c1 <= c0) return XKB_OK;
  char* dst = static_cast<char*>(d->host) + (r0 + c0 * d->ld) * d->esz;
  const char* src = static_cast<const char*>(dev_ptr(d, r0, c0));
  const size_t w = (r1 - r0) * d->esz;
  R.stats.d2h += w * (c1 - c0);
  const long long tv = xkb::evlog_copy_begin(R.s_d2h, w * (c1 - c0), 2);
  cudaError_t e;
  if (d->ld == d->dld && (r1 - r0 == d->M || c1 - c0 == 1))
    e = cudaMemcpyAsync(dst, src, ((c1 - c0 - 1) * d->ld + (r1 - r0)) * d->esz,
                        cudaMemcpyDeviceToHost, R.s_d2h);
  else
    e = cudaMemcpy2DAsync(dst, d->ld * d->esz, src, d->dld * d->esz, w, c1 - c0,
                          cudaMemcpyDeviceToHost, R.s_d2h);
  xkb::evlog_copy_end(tv, R.s_d2h);
  return cuda_ok(e);
}

// For each tile column in [tc0, tc1) find runs of tiles whose state
// satisfies `want`; whole-height runs of consecutive tile columns merge into
// one 2-D copy.  `fn(r0, r1, c0, c1)` issues the copy.
template <class Pred, class Fn>
static int for_runs(Desc* d, size_t tr0, size_t tr1, size_t tc0, size_t tc1, Pred want,
                    Fn fn) {
  size_t pend_c0 = 0, pend_c1 = 0;  // pending full-height column range
  bool pend = false;
  auto flush = [&]() -> int {
    if (!pend) return XKB_OK;
    pend = false;
    return fn(tr0 * d->mb, std::min(tr1 * d->mb, d->M), pend_c0 * d->nb,
              std::min(pend_c1 * d->nb, d->N));
  };
  for (size_t j = tc0; j < tc1; ++j) {
    bool all = true;
    for (size_t i = tr0; i < tr1 && all; ++i) all = want(d->tile(i, j), i, j);
    if (all) {
      if (pend && pend_c1 == j) pend_c1 = j + 1;
      else {
        int e = flush();
        if (e) return e;
        pend = true;
        pend_c0 = j;
        pend_c1 = j + 1;
      }
      continue;
    }
    int e = flush();
    if (e) return e;
    size_t i = tr0;
    while (i < tr1) {
      if (!want(d->tile(i, j), i, j)) {
        ++i;
        continue;
      }
      size_t i1 = i;
      while (i1 < tr1 && want(d->tile(i1, j), i1, j)) ++i1;
      e = fn(i * d->mb, std::min(i1 * d->mb, d->M), j * d->nb, std::min((j + 1) * d->nb, d->N));
      if (e) return e;
      i = i1;
    }
  }
  return flush();
}

int make_valid(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1, bool wait) {
  Runtime& R = rt();
  if (r1 <= r0 || c1 <= c0) return XKB_OK;
  const size_t tr0 = r0 / d->mb, tr1 = (r1 + d->mb - 1) / d->mb;
  const size_t tc0 = c0 / d->nb, tc1 = (c1 + d->nb - 1) / d->nb;
  uint64_t miss = 0, hit = 0;
  for (size_t j = tc0; j < tc1; ++j)
    for (size_t i = tr0; i < tr1; ++i) (d->tile(i, j) & kDevValid) ? ++hit : ++miss;
  R.stats.hits += hit;
  R.stats.misses += miss;
  if (miss == 0) return XKB_OK;
  int e = for_runs(
      d, tr0, tr1, tc0, tc1, [](uint8_t s, size_t, size_t) { return !(s & kDevValid); },
      [&](size_t a, size_t b, size_t c, size_t dd) { return copy_h2d(d, a, b, c, dd); });
  if (e) return e;
  for (size_t j = tc0; j < tc1; ++j)
    for (size_t i = tr0; i < tr1; ++i) d->tile(i, j) |= kDevValid;
  R.h2d_unsynced = true;
  return wait ? comp_wait_h2d() : XKB_OK;
}

int comp_wait_h2d() {
  Runtime& R = rt();
  if (!R.h2d_unsynced) return XKB_OK;
  R.h2d_unsynced = false;
  cudaEvent_t ev = next_event();
  cudaEventRecord(ev, R.s_h2d);
  return cuda_ok(cudaStreamWaitEvent(R.s_comp, ev, 0));
}

static bool tile_in_uplo(const Desc* d, size_t i, size_t j, int uplo) {
  // tile (i,j) intersects the uplo triangle of the matrix
  const size_t r0 = i * d->mb, r1 = std::min((i + 1) * d->mb, d->M);
  const size_t c0 = j * d->nb, c1 = std::min((j + 1) * d->nb, d->N);
  if (uplo == CblasLower) return r1 > c0;   // some row >= some col
  if (uplo == CblasUpper) return c1 > r0;
  (void)r0;
  return true;
}

void mark_written(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1, int uplo) {
  if (r1 <= r0 || c1 <= c0) return;
  d->ready.clear();  // this write is ordered by the compute stream only
  const size_t tr0 = r0 / d->mb, tr1 = (r1 + d->mb - 1) / d->mb;
  const size_t tc0 = c0 / d->nb, tc1 = (c1 + d->nb - 1) / d->nb;
  for (size_t j = tc0; j < tc1; ++j)
    for (size_t i = tr0; i < tr1; ++i)
      if (!uplo || tile_in_uplo(d, i, j, uplo))
        d->tile(i, j) |= d->managed ? kDevValid : (kDevValid | kHostStale);
}

void mark_full_overwrite(Desc* d, size_t r0, size_t r1, size_t c0, size_t c1) {
  mark_written(d, r0, r1, c0, c1, 0);
}

int flush_pending() {
  Runtime& R = rt();
  if (R.pending.empty()) return XKB_OK;
  std::vector<xkb_batch_op> ops;
  ops.swap(R.pending);
  std::vector<Desc*> written;
  for (Desc* d : R.pend_descs) {
    if (d->pend & 2) written.push_back(d);
    d->pend = 0;
  }
  R.pend_descs.clear();
  R.pend_bytes = 0;
  const int e = launch_ops(ops);
  if (e) return e;
  // the outputs are final once this launch is: coherence need not wait for
  // work queued after it
  if (EventRef ev = new_event_ref()) {
    cudaEventRecord(ev->e, R.s_comp);
    for (Desc* d : written) d->ready.assign(1, {0, d->M, 0, d->N, ev});
  }
  return XKB_OK;
}

int launch_ops(const std::vector<xkb_batch_op>& ops) {
  Runtime& R = rt();
  // trace name of the launched work: the deferred call, not the call whose
  // flush launches it
  static const char* const kNames[2][2] = {{"dgemm", "zgemm"}, {"dtrsm", "ztrsm"}};
  const xkb_batch_op& o0 = ops[0];
  xkb::EvName ev_name(ops.size() > 1 ? "batch"
                                     : kNames[o0.kind == XKB_BATCH_TRSM][o0.dtype == XKB_Z]);
  if (ops.size() == 1) {  // a lone call: the whole-matrix kernels
    const xkb_batch_op& o = ops[0];
    if (o.kind == XKB_BATCH_TRSM)
      return xkb_cuda_trsm(o.dtype, 0, o.uplo, o.trans, o.diag, o.M, o.N, o.alpha, o.A, o.lda,
                           o.C, o.ldc, 0, R.s_comp);
    xkb_gemm_args a{};
    a.dtype = o.dtype;
    a.opA = o.opA;
    a.opB = o.opB;
    a.M = o.M;
    a.N = o.N;
    a.K = o.K;
    a.A = o.A;
    a.lda = o.lda;
    a.B = o.B;
    a.ldb = o.ldb;
    a.C = o.C;
    a.ldc = o.ldc;
    a.alpha[0] = o.alpha[0];
    a.alpha[1] = o.alpha[1];
    a.beta[0] = o.beta[0];
    a.beta[1] = o.beta[1];
    a.uplo = XKB_FULL;
    return xkb_cuda_gemm(&a, R.s_comp);
  }
  R.batches++;
  R.batched_calls += ops.size();
  return xkb_cuda_batch(ops.data(), (int)ops.size(), (int)xkb_tune_get("batch_schedule", 0.0),
                        R.s_comp);
}

int defer_op(const xkb_batch_op& o, Desc* r0, Desc* r1, Desc* r2, Desc* w) {
  Runtime& R = rt();
  auto has = [](const Desc* d, uint8_t bits) { return d && (d->pend & bits); };
  // read-after-write, write-after-read, write-after-write on a queued buffer
  const bool conflict = has(r0, 2) || has(r1, 2) || has(r2, 2) || has(w, 3);
  if (conflict || R.pending.size() >= R.batch_max) {
    if (int e = flush_pending()) return e;
  }
  R.pending.push_back(o);
  const size_t es = (o.dtype == XKB_S ? 4 : (o.dtype == XKB_Z ? 16 : 8));
  R.pend_bytes += es * (o.kind == XKB_BATCH_TRSM
                            ? (size_t)o.M * o.M + (size_t)o.M * o.N
                            : (size_t)o.M * o.K + (size_t)o.K * o.N + (size_t)o.M * o.N);
  auto mark = [&](Desc* d, uint8_t bit) {
    if (!d) return;
    if (!d->pend) R.pend_descs.push_back(d);
    d->pend |= bit;
  };
  mark(r0, 1);
  mark(r1, 1);
  mark(r2, 1);
  mark(w, 2);
  if (w) w->ready.clear();  // set again when this call is launched
  const size_t lim = R.batch_flush_env
                         ? R.batch_flush_env
                         : (size_t)(xkb_tune_get("batch_flush_mb", 2048.0) * 1048576.0);
  if (R.pend_bytes >= lim) return flush_pending();
  return XKB_OK;
}

int make_valid_panels(const std::vector<std::pair<Desc*, size_t>>& ds,
                      const std::vector<long>& bounds, std::vector<cudaEvent_t>& ev) {
  Runtime& R = rt();
  const size_t np = bounds.size() - 1, ncol = (size_t)bounds.back();
  ev.assign(np, nullptr);
  // snapshot of the tiles that need a copy: tile rows covering [0, rows),
  // tile columns covering [0, ncol); whole tiles are copied, as make_valid does
  std::vector<std::vector<uint8_t>> need(ds.size());
  std::vector<size_t> tr1(ds.size()), tc1(ds.size());
  for (size_t m = 0; m < ds.size(); ++m) {
    Desc* d = ds[m].first;
    tr1[m] = std::min(d->mt, (ds[m].second + d->mb - 1) / d->mb);
    tc1[m] = std::min(d->nt, (ncol + d->nb - 1) / d->nb);
    need[m].assign(d->mt * d->nt, 0);
    for (size_t j = 0; j < tc1[m]; ++j)
      for (size_t i = 0; i < tr1[m]; ++i) {
        const bool miss = !(d->tile(i, j) & kDevValid);
        need[m][i + j * d->mt] = miss;
        miss ? ++R.stats.misses : ++R.stats.hits;
      }
  }
  for (size_t p = 0; p < np; ++p) {
    for (size_t m = 0; m < ds.size(); ++m) {
      Desc* d = ds[m].first;
      // the last panel also takes the rest of its last tile column
      const size_t c0 = std::min((size_t)bounds[p], d->N);
      const size_t c1 = p + 1 == np ? std::min(tc1[m] * d->nb, d->N)
                                    : std::min((size_t)bounds[p + 1], d->N);
      for (size_t tj = c0 / d->nb; tj * d->nb < c1; ++tj) {
        const size_t a = std::max(c0, tj * d->nb), b = std::min(c1, (tj + 1) * d->nb);
        size_t i = 0;
        while (i < tr1[m]) {  // runs of tile rows needing a copy in this tile column
          if (!need[m][i + tj * d->mt]) {
            ++i;
            continue;
          }
          size_t i1 = i;
          while (i1 < tr1[m] && need[m][i1 + tj * d->mt]) ++i1;
          if (int e = copy_h2d(d, i * d->mb, std::min(i1 * d->mb, d->M), a, b)) return e;
          i = i1;
        }
      }
    }
    ev[p] = next_event();
    cudaEventRecord(ev[p], R.s_h2d);
  }
  for (size_t m = 0; m < ds.size(); ++m)
    for (size_t j = 0; j < tc1[m]; ++j)
      for (size_t i = 0; i < tr1[m]; ++i) ds[m].first->tile(i, j) |= kDevValid;
  return XKB_OK;
}

int make_valid_blocks(Desc* da, bool a_trans, size_t K, const std::vector<long>& rb, Desc* db,
                      const std::vector<long>& cb, const std::vector<int>& seq,
                      std::vector<cudaEvent_t>& ev_a, std::vector<cudaEvent_t>& ev_b) {
  Runtime& R = rt();
  const size_t nr = rb.size() - 1, nc = cb.size() - 1;
  ev_a.assign(nr, nullptr);
  ev_b.assign(nc, nullptr);
  // the stored region of a block: rows [r0, r1) x columns [c0, c1)
  struct Reg {
    size_t r0, r1, c0, c1;
  };
  auto region = [&](int s) -> Reg {
    if (s >= 0) return {0, K, (size_t)cb[s], (size_t)cb[s + 1]};
    const size_t i = (size_t)(-1 - s);
    return a_trans ? Reg{0, K, (size_t)rb[i], (size_t)rb[i + 1]}
                   : Reg{(size_t)rb[i], (size_t)rb[i + 1], 0, K};
  };
  // snapshot of the tiles that need a copy (whole matrices as used)
  auto snapshot = [&](Desc* d, size_t rows, size_t cols) {
    std::vector<uint8_t> need(d->mt * d->nt, 0);
    const size_t tr1 = std::min(d->mt, (rows + d->mb - 1) / d->mb);
    const size_t tc1 = std::min(d->nt, (cols + d->nb - 1) / d->nb);
    for (size_t j = 0; j < tc1; ++j)
      for (size_t i = 0; i < tr1; ++i) {
        const bool miss = !(d->tile(i, j) & kDevValid);
        need[i + j * d->mt] = miss;
        miss ? ++R.stats.misses : ++R.stats.hits;
      }
    return need;
  };
  const size_t a_rows = a_trans ? K : (size_t)rb.back(), a_cols = a_trans ? (size_t)rb.back() : K;
  std::vector<uint8_t> need_a = snapshot(da, a_rows, a_cols);
  std::vector<uint8_t> need_b = snapshot(db, K, (size_t)cb.back());
  for (int s : seq) {
    Desc* d = s >= 0 ? db : da;
    const std::vector<uint8_t>& need = s >= 0 ? need_b : need_a;
    const Reg g = region(s);
    // runs of tile rows needing a copy in each tile column, clipped to the block
    for (size_t tj = g.c0 / d->nb; tj * d->nb < g.c1 && tj < d->nt; ++tj) {
      const size_t c0 = std::max(g.c0, tj * d->nb), c1 = std::min(g.c1, (tj + 1) * d->nb);
      const size_t ti1 = std::min(d->mt, (g.r1 + d->mb - 1) / d->mb);
      size_t i = g.r0 / d->mb;
      while (i < ti1) {
        if (!need[i + tj * d->mt]) {
          ++i;
          continue;
        }
        size_t i1 = i;
        while (i1 < ti1 && need[i1 + tj * d->mt]) ++i1;
        if (int e = copy_h2d(d, std::max(g.r0, i * d->mb), std::min(g.r1, i1 * d->mb), c0, c1))
          return e;
        i = i1;
      }
    }
    cudaEvent_t ev = next_event();
    cudaEventRecord(ev, R.s_h2d);
    (s >= 0 ? ev_b[(size_t)s] : ev_a[(size_t)(-1 - s)]) = ev;
  }
  auto mark = [&](Desc* d, size_t rows, size_t cols) {
    const size_t tr1 = std::min(d->mt, (rows + d->mb - 1) / d->mb);
    const size_t tc1 = std::min(d->nt, (cols + d->nb - 1) / d->nb);
    for (size_t j = 0; j < tc1; ++j)
      for (size_t i = 0; i < tr1; ++i) d->tile(i, j) |= kDevValid;
  };
  mark(da, a_rows, a_cols);
  mark(db, K, (size_t)cb.back());
  return XKB_OK;
}

int coherent(Desc* d, int uplo, int memflag) {
  Runtime& R = rt();
  if (int e = flush_pending()) return e;
  if (d->managed) {
    // nothing to copy (the reference's unified mode returns here too,
    // blas/xkblas.c:1959); move the pages back to the host once the queued
    // work is done, so that host reads after xkblas_sync do not fault
    cudaEvent_t ev = next_event();
    cudaEventRecord(ev, R.s_comp);
    cudaStreamWaitEvent(R.s_d2h, ev, 0);
    if (cudaMemPrefetchAsync(d->host, ((d->N ? d->N - 1 : 0) * d->ld + d->M) * d->esz,
                             cudaCpuDeviceId, R.s_d2h) != cudaSuccess)
      cudaGetLastError();
    d->ready.clear();
    return XKB_OK;
  }
  int e = XKB_OK;
  if (uplo == 0 && !d->ready.empty()) {
    // written rectangle by rectangle: copy each back once its event fired, in
    // the order they finish; what lies outside them after all work queued
    // so far
    const auto stale = [&](uint8_t s, size_t, size_t) { return (s & kHostStale) != 0; };
    size_t Mc = 0, Nc = 0;
    for (const auto& r : d->ready) {
      Mc = std::max(Mc, r.r1);
      Nc = std::max(Nc, r.c1);
      bool waited = false;
      e = for_runs(d, r.r0 / d->mb, std::min(d->mt, (r.r1 + d->mb - 1) / d->mb), r.c0 / d->nb,
                   std::min(d->nt, (r.c1 + d->nb - 1) / d->nb), stale,
                   [&](size_t a, size_t b, size_t c, size_t dd) {
                     const size_t ra = std::max(a, r.r0), rz = std::min(b, r.r1);
                     const size_t ca = std::max(c, r.c0), cz = std::min(dd, r.c1);
                     if (ra >= rz || ca >= cz) return XKB_OK;
                     if (!waited) {
                       cudaStreamWaitEvent(R.s_d2h, r.ev->e, 0);
                       waited = true;
                     }
                     return copy_d2h(d, ra, rz, ca, cz);
                   });
      if (e) break;
    }
    cudaEvent_t tail = nullptr;
    auto after_all = [&](size_t a, size_t b, size_t c, size_t dd) {
      if (a >= b || c >= dd) return XKB_OK;
      if (!tail) {
        tail = next_event();
        cudaEventRecord(tail, R.s_comp);
        cudaStreamWaitEvent(R.s_d2h, tail, 0);
      }
      return copy_d2h(d, a, b, c, dd);
    };
    if (!e)
      e = for_runs(d, 0, d->mt, 0, d->nt, stale, [&](size_t a, size_t b, size_t c, size_t dd) {
        // the parts of the run outside [0, Mc) x [0, Nc)
        if (int r = after_all(std::max(a, Mc), b, c, dd)) return r;
        return after_all(a, std::min(b, Mc), std::max(c, Nc), dd);
      });
  } else {
    // D2H after everything already queued on the compute stream
    cudaEvent_t ev = next_event();
    cudaEventRecord(ev, R.s_comp);
    cudaStreamWaitEvent(R.s_d2h, ev, 0);
    e = for_runs(
        d, 0, d->mt, 0, d->nt,
        [&](uint8_t s, size_t i, size_t j) {
          return (s & kHostStale) && (uplo == 0 || tile_in_uplo(d, i, j, uplo));
        },
        [&](size_t a, size_t b, size_t c, size_t dd) { return copy_d2h(d, a, b, c, dd); });
  }
  if (e) return e;
  d->ready.clear();
  for (size_t j = 0; j < d->nt; ++j)
    for (size_t i = 0; i < d->mt; ++i) {
      uint8_t& s = d->tile(i, j);
      const bool in = uplo == 0 || tile_in_uplo(d, i, j, uplo);
      if (in) s &= (uint8_t)~kHostStale;
      else if (memflag == 1) s = 0;  // strict mode: the other part is dropped
    }
  return XKB_OK;
}

size_t auto_tilesize(xkblas_kernel_t kernel, size_t M, size_t N, size_t K) {
  // reference blas/xkblas.c:2239-2533 with one GPU; a preset NB wins.
  (void)N;
  (void)K;
  Runtime& R = rt();
  if (R.nb_param) return R.nb_param;
  const size_t ng = 1;
  size_t NB = 0, fact = 1;
  switch (kernel) {
    case KERN_GEMM:
    case KERN_GEMMT:
      NB = M / ng;
      if (M > 16384 && NB < 2048) NB = 2048;
      if (NB > 4096) NB = M / (2 * ng);
      if (NB < 512) NB = 512;
      NB = (NB + 63) & ~size_t(63);
      break;
    case KERN_HERK:
    case KERN_SYRK:
      fact = 2;
      for (;;) {
        NB = M / (fact * ng);
        if (NB >= 2048) NB &= ~size_t(2047);
        if (NB <= 1024 && fact == 2) {
          fact = 1;
          continue;
        }
        break;
      }
      if (NB > 4096) NB = M / (2 * fact * ng);
      if (NB < 512) NB = 512;
      break;
    case KERN_HER2K:
    case KERN_SYR2K:
      fact = 4;
      for (;;) {
        NB = (M / (fact * ng) + 63) & ~size_t(63);
        if (NB <= 2048 && fact > 2) {
          --fact;
          continue;
        }
        break;
      }
      if (NB > 4096) NB = M / (2 * fact * ng);
      if (NB < 512) NB = 512;
      break;
    case KERN_HEMM:
    case KERN_SYMM:
      NB = (M / ng) & ~size_t(1023);
      if (NB < 1024) NB = 1024;
      if (NB < 4096) NB *= 2;
      break;
    case KERN_TRMM:
    case KERN_TRSM:
      NB = (M / (2 * ng) + 63) & ~size_t(63);
      if (NB < 2048) NB = 2048;
      break;
    default:
      NB = M / ng;
      if (NB >= 4096) NB = M / (2 * ng);
      if (NB < 1024) NB = 1024;
      NB = (NB + 63) & ~size_t(63);
      break;
  }
  return std::max<size_t>(NB, 64);
}

}  // namespace xkbrt

using namespace xkbrt;

// ============================================================================
// C API: lifecycle, parameters, memory, coherence
// ============================================================================
extern "C" {

int xkblas_get_devicecount(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int xkblas_init(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (R.refcount++ != 0) return 0;
  int e = ensure_init();
  return e == XKB_OK ? 0 : e;
}

int xkblas_finalize(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (R.refcount == 0) return 0;
  if (--R.refcount != 0) return 0;
  if (!R.ready) return 0;
  cudaStreamSynchronize(R.s_comp);
  cudaStreamSynchronize(R.s_h2d);
  cudaStreamSynchronize(R.s_d2h);
  std::vector<Desc*> all;
  for (auto& kv : R.descs) all.push_back(kv.second);
  for (Desc* d : all) drop_desc(d);
  cudaStreamSynchronize(R.s_comp);
  xkb_cuda_batch_release();
  if (const char* dir = getenv("XKBLAS_TRACE_DIR"))
    if (*dir) xkblas_trace_export(dir);
  if (R.verbose) print_statistics();
  return 0;
}

int xkblas_get_device_count(int* count) {
  if (!count) return EINVAL;
  *count = xkblas_get_devicecount() > 0 ? 1 : 0;
  return 0;
}

int xkblas_get_device_properties(struct xkblas_dev_prop_t* prop) {
  if (!prop) return EINVAL;
  prop->device_count = xkblas_get_devicecount() > 0 ? 1 : 0;
  prop->has_unified = 0;
  if (prop->device_count) {
    int m = 0;
    if (cudaDeviceGetAttribute(&m, cudaDevAttrConcurrentManagedAccess, rt().device) == cudaSuccess)
      prop->has_unified = m ? 1 : 0;
    else
      cudaGetLastError();
  }
  prop->arch = XKBLAS_ARCH_UNKNOWN;
  if (prop->device_count) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, rt().device) == cudaSuccess && p.major == 10)
      prop->arch = XKBLAS_ARCH_B200;
  }
  return 0;
}

int xkblas_force_set_unified(void) {
  int dev = 0, managed = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&managed, cudaDevAttrManagedMemory, dev) != cudaSuccess || !managed) {
    cudaGetLastError();
    return EINVAL;
  }
  rt().unified = true;
  return 0;
}

const char* xkblas_get_configuration(void) {
  return "xkblas-b200 0.6: sm_100a; FP64 DMMA (TMA+mbarrier) tile GEMM; Ozaki-II INT8 "
         "tcgen05/TMEM; device tile directory; 1 GPU";
}

void xkblas_load_sym(void** ptr, const char* name);  // native.cpp

int xkblas_sync(void) {
  // Waits for the work queued before this call -- all of the calling
  // thread's own calls -- without holding the runtime lock while waiting, so
  // other threads keep submitting (reference: each thread synchronises its
  // own task list, blas/xkblas.c:1773-1850).  Deferred calls are launched
  // first (the queue is shared by the threads).
  Runtime& R = rt();
  ThreadCtx& T = tctx();
  int e = 0;
  {
    std::lock_guard<std::recursive_mutex> g(R.mu);
    if (!R.ready) {
      xkb::evlog_sync_done();
      return 0;
    }
    e = flush_pending();
    if (!T.ev[0]) {
      for (auto& ev : T.ev) {
        if (!R.ev_free.empty()) {
          ev = R.ev_free.back();
          R.ev_free.pop_back();
        } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
          cudaGetLastError();
          ev = nullptr;
        }
      }
    }
    const cudaStream_t ss[3] = {R.s_comp, R.s_h2d, R.s_d2h};
    for (int i = 0; i < 3; ++i)
      if (!T.ev[i] || cudaEventRecord(T.ev[i], ss[i]) != cudaSuccess) {
        cudaGetLastError();
        if (cudaStreamSynchronize(ss[i]) != cudaSuccess) e = XKB_ECUDA;  // no event: drain
      }
  }
  for (cudaEvent_t ev : T.ev)
    if (ev && cudaEventSynchronize(ev) != cudaSuccess) e = XKB_ECUDA;
  std::lock_guard<std::recursive_mutex> g(R.mu);
  int de = xkb_cuda_take_device_error();
  if (de) {
    // a bounded device wait that gave up, or a bounds check that refused an
    // access; xkblas_last_device_error() gives the exact word
    R.sticky_error = de;
    e = (de >= XKB_DEV_FULL_WAIT && de <= XKB_DEV_ACC_WAIT) ? XKB_ETIMEDOUT
        : de == XKB_DEV_BOUNDS                              ? XKB_EFAULT
                                                            : XKB_ECUDA;
  }
  xkb::evlog_sync_done();
  return e;
}

int xkblas_last_device_error(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  int v = R.sticky_error;
  R.sticky_error = 0;
  return v;
}

xkblas_context_t* xkblas_context_get(void) {
  // the calling thread's context (an opaque, non-null handle per thread)
  return reinterpret_cast<xkblas_context_t*>(&tctx());
}

void xkblas_set_modemath(xkblas_mode_math_t mode) {
  // the calling thread's mode only (reference blas/xkblas.c:356-359)
  tctx().math = (mode == XKBLAS_TENSOR_OP_MATH) ? XKBLAS_TENSOR_OP_MATH : XKBLAS_DEFAULT_MATH;
}

xkblas_mode_math_t xkblas_get_modemath(void) {
  return thread_math() == XKBLAS_TENSOR_OP_MATH ? XKBLAS_TENSOR_OP_MATH : XKBLAS_DEFAULT_MATH;
}

size_t xkblas_get_param(void) { return rt().nb_param; }
void xkblas_set_param(size_t nb, size_t p) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  R.nb_param = nb;
  R.prec_param = p ? p : 8;
}
int xkblas_get_ngpus(void) { return xkblas_get_devicecount() > 0 ? 1 : 0; }
int xkblas_set_ngpus(int ngpus) { return (ngpus == 1 || ngpus == 0) ? 0 : EINVAL; }

uint64_t xkblas_elapsedns(void) {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
double xkblas_elapsedtime(void) { return 1e-9 * (double)xkblas_elapsedns(); }

size_t xkblas_auto_tilesize(xkblas_context_t* ctx, xkblas_kernel_t kernel, size_t M,
                            size_t N, size_t K) {
  (void)ctx;
  return auto_tilesize(kernel, M, N, K);
}

// ---- descriptors -----------------------------------------------------------
xkblas_matrix_descr_t* xkblas_find(const void* A) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  auto it = R.descs.find(A);
  return it == R.descs.end() ? nullptr : reinterpret_cast<xkblas_matrix_descr_t*>(it->second);
}

int xkblas_matrix_descr_isinit(xkblas_matrix_descr_t* Ah) {
  return Ah && reinterpret_cast<Desc*>(Ah)->registered_init;
}

int xkblas_init_matrix_handle(xkblas_matrix_descr_t* Ah, void* A, size_t M, size_t N,
                              size_t LD, size_t eltsize, size_t MB, size_t NB) {
  // Descriptors are created by the library on first touch; this entry point
  // (re)creates the one of A with the given geometry.
  (void)Ah;
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (!A || LD < std::max<size_t>(M, 1) || eltsize == 0) return EINVAL;
  if (ensure_init() != XKB_OK) return ENODEV;
  int err;
  Desc* d = get_desc(A, M, N, LD, eltsize, std::max(MB, NB), &err);
  return d ? 0 : EINVAL;
}

// ---- host memory -----------------------------------------------------------
void* xkblas_malloc(size_t sz) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, std::max<size_t>(sz, 1), cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return malloc(std::max<size_t>(sz, 1));  // no driver: plain host memory
  }
  return p;
}

void xkblas_free(void* ptr, size_t sz) {
  (void)sz;
  if (!ptr) return;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) == cudaSuccess && a.type == cudaMemoryTypeHost) {
    cudaFreeHost(ptr);
    return;
  }
  cudaGetLastError();
  free(ptr);
}

// Unified mode (reference blas/xkblas.c:155-220): managed memory when the
// mode is on (xkblas_force_set_unified or XKBLAS_UNIFIED=1), else malloc.
// Managed matrices are used in place by the kernels (no tile copies).
int xkblas_malloc_unified(void** ptr, size_t size) {
  if (!ptr) return EINVAL;
  Runtime& R = rt();
  if (R.unified) {
    if (cudaMallocManaged(ptr, std::max<size_t>(size, 1), cudaMemAttachGlobal) != cudaSuccess) {
      cudaGetLastError();
      *ptr = nullptr;
      return ENOMEM;
    }
    return 0;
  }
  *ptr = malloc(std::max<size_t>(size, 1));
  return *ptr ? 0 : ENOMEM;
}
int xkblas_free_unified(void* ptr) {
  if (!ptr) return 0;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) == cudaSuccess && a.type == cudaMemoryTypeManaged) {
    Runtime& R = rt();
    {
      std::lock_guard<std::recursive_mutex> g(R.mu);
      auto it = R.descs.find(ptr);  // a directory entry must not outlive the memory
      if (it != R.descs.end()) drop_desc(it->second);
      if (R.ready) cudaDeviceSynchronize();
    }
    cudaFree(ptr);
    return 0;
  }
  cudaGetLastError();
  free(ptr);
  return 0;
}
void xkblas_activate_custom_alloc(void) {}
void xkblas_deactivate_custom_alloc(void) {}

// Host registration is synchronous here (cudaHostRegister is fast on this
// platform); the async forms return a handle that is already complete.
uint64_t xkblas_register_memory_async(void* ptr, size_t sz) {
  return xkblas_register_memory(ptr, sz) == 0 ? (uint64_t)(uintptr_t)ptr : 0;
}
uint64_t xkblas_unregister_memory_async(void* ptr, size_t sz) {
  return xkblas_unregister_memory(ptr, sz) == 0 ? (uint64_t)(uintptr_t)ptr : 0;
}
int xkblas_register_memory_test(uint64_t h) { return h != 0; }
int xkblas_register_memory_wait(uint64_t h) { return h ? 0 : EINVAL; }
int xkblas_register_memory_waitall(void) { return 0; }
int xkblas_register_memory(void* ptr, size_t sz) {
  if (!ptr || !sz) return EINVAL;
  cudaError_t e = cudaHostRegister(ptr, sz, cudaHostRegisterPortable);
  if (e == cudaErrorHostMemoryAlreadyRegistered || e == cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaGetLastError();
  return EINVAL;
}
int xkblas_unregister_memory(void* ptr, size_t sz) {
  (void)sz;
  if (!ptr) return EINVAL;
  cudaError_t e = cudaHostUnregister(ptr);
  cudaGetLastError();
  return (e == cudaSuccess || e == cudaErrorHostMemoryNotRegistered) ? 0 : EINVAL;
}
void xkblas_memset(void* ptr, int v, size_t sz) {
  if (ptr) memset(ptr, v, sz);
}
void xkblas_memcpy(void* dst, void* src, size_t sz) {
  if (dst && src) memcpy(dst, src, sz);
}
void xkblas_register_work_buffer(void* ptr, size_t sz) { xkblas_register_memory(ptr, sz); }
void xkblas_unregister_work_buffer(void* ptr) { xkblas_unregister_memory(ptr, 0); }
void* xkblas_get_work_pos(size_t sz) { return xkblas_malloc(sz); }
void xkblas_free_work_pos(void* ptr) { xkblas_free(ptr, 0); }
void xkblas_bind_cpu(void* ptr, size_t sz) {
  (void)ptr;
  (void)sz;
}
void xkblas_host_register_direct(void* ptr, size_t sz) { xkblas_register_memory(ptr, sz); }
void xkblas_host_unregister_direct(void* ptr) { xkblas_unregister_memory(ptr, 0); }

// ---- debug / placement: one GPU ------------------------------------------
int xkblas_dbg_setname(const char* name, xkblas_matrix_descr_t* Mh) {
  return xkblas_dbg_setname_with_flags(name, Mh, 0);
}
int xkblas_dbg_setname_with_flags(const char* name, xkblas_matrix_descr_t* Mh,
                                  uint32_t flags) {
  (void)flags;
  if (!Mh || !name) return EINVAL;
  reinterpret_cast<Desc*>(Mh)->name = name;
  return 0;
}
void xkblas_dbg_dump_graph(const char* name) { (void)name; }
int xkblas_map_2Dblock_cyclic(xkblas_context_t* ctx, int hlevel, int storage, size_t m,
                              size_t n, const void* A, size_t ld, size_t eltsize, size_t Bp,
                              size_t Bq, size_t Gp, size_t Gq, int force) {
  (void)ctx; (void)hlevel; (void)storage; (void)m; (void)n; (void)ld; (void)eltsize;
  (void)Bp; (void)Bq; (void)force;
  if (!A || Gp == 0 || Gq == 0) return EINVAL;
  return 0;
}
int xkblas_map_1Dblock_cyclic(xkblas_context_t* ctx, int hlevel, int storage, int colrow,
                              size_t m, size_t n, const void* A, size_t ld, size_t eltsize,
                              size_t B, size_t G, int force) {
  (void)ctx; (void)hlevel; (void)storage; (void)colrow; (void)m; (void)n; (void)ld;
  (void)eltsize; (void)B; (void)force;
  if (!A || G == 0) return EINVAL;
  return 0;
}
int xkblas_distribute_2Dblock_cyclic_async(int hlevel, int storage, int uplo, size_t NB,
                                           size_t m, size_t n, const void* A, size_t ld,
                                           size_t eltsize, size_t Bp, size_t Bq, size_t Gp,
                                           size_t Gq) {
  (void)hlevel; (void)storage; (void)Bp; (void)Bq; (void)Gp; (void)Gq;
  // one GPU: "distribute" = upload the tiles now
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (!A || ld < m || eltsize == 0) return EINVAL;
  if (ensure_init() != XKB_OK) return ENODEV;
  int err;
  Desc* d = get_desc(A, m, n, ld, eltsize, NB ? NB : auto_tilesize(KERN_GEMM, m, n, 0), &err);
  if (!d) return EINVAL;
  (void)uplo;
  return make_valid(d, 0, m, 0, n) ? EINVAL : 0;
}
int xkblas_distribute_1Dblock_cyclic_async(int hlevel, int storage, int uplo, int colrow,
                                           size_t NB, size_t m, size_t n, const void* A,
                                           size_t ld, size_t eltsize, size_t B, size_t G) {
  (void)colrow; (void)B; (void)G;
  return xkblas_distribute_2Dblock_cyclic_async(hlevel, storage, uplo, NB, m, n, A, ld, eltsize,
                                                1, 1, 1, 1);
}

// ---- coherence ---------------------------------------------------------------
int xkblas_memory_coherent_async(int uplo, int memflag, size_t M, size_t N, void* A, size_t ld,
                                 size_t elsize) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (!R.ready) return 0;
  if (uplo != 0 && uplo != CblasUpper && uplo != CblasLower) return EINVAL;
  auto it = R.descs.find(A);
  if (it == R.descs.end()) return 0;  // never used on the device: host is current
  Desc* d = it->second;
  (void)M; (void)N; (void)ld; (void)elsize;
  return coherent(d, uplo, memflag) ? EINVAL : 0;
}

int xkblas_memory_syncall(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (!R.ready) return 0;
  for (auto& kv : R.descs)
    if (coherent(kv.second, 0, 0)) return EINVAL;
  return xkblas_sync() ? EINVAL : 0;
}

int xkblas_memory_invalidate(const void* A) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  auto it = R.descs.find(A);
  if (it == R.descs.end()) return 0;
  drop_desc(it->second);
  return 0;
}

int xkblas_memory_invalidate_caches(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  std::vector<Desc*> all;
  for (auto& kv : R.descs) all.push_back(kv.second);
  for (Desc* d : all) drop_desc(d);
  return 0;
}

int xkblas_memory_free(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  xkblas_memory_invalidate_caches();
  if (!R.ready) return 0;
  cudaStreamSynchronize(R.s_comp);
  xkb_cuda_batch_release();  // cached batch graphs hold device memory
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, R.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  return 0;
}

int xkblas_get_stats(xkblas_stats_t* st) {
  if (!st) return EINVAL;
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  st->calls = R.stats.calls;
  st->kernels = xkb_cuda_kernel_count();
  st->h2d_bytes = R.stats.h2d;
  st->d2h_bytes = R.stats.d2h;
  st->evictions = R.stats.evictions;
  st->tile_hits = R.stats.hits;
  st->tile_misses = R.stats.misses;
  // Ozaki contractions are counted on the device (the moduli count of a call
  // may be chosen there); reading the counters waits for the device
  st->ozaki_calls = st->ozaki_moduli = 0;
  unsigned long long oz[3];
  if (R.ready && xkb_ozaki_counts(oz, nullptr, 0) == XKB_OK) {
    st->ozaki_calls = oz[0] - R.stats.ozaki_calls;
    st->ozaki_moduli = oz[1] - R.stats.ozaki_moduli;
  }
  st->flops = R.stats.flops;
  st->batches = R.batches;
  st->batched_calls = R.batched_calls;
  return 0;
}

void xkblas_reset_stats(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  R.stats = Stats();
  // the Ozaki counters' values at the reset (get_stats reports the growth)
  unsigned long long oz[3];
  if (R.ready && xkb_ozaki_counts(oz, nullptr, 0) == XKB_OK) {
    R.stats.ozaki_calls = oz[0];
    R.stats.ozaki_moduli = oz[1];
  }
  R.batches = 0;
  R.batched_calls = 0;
}

}  // extern "C"
