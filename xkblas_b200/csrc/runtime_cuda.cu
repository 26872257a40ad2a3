// runtime_cuda.cu -- host helpers under the thin C ABI: tensor-map encoding
// through the driver entry point (no link-time libcuda dependency, so the
// library loads on machines without a GPU driver), stream resolution,
// launch accounting and the device error word readers.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "xkb_dev.cuh"

namespace xkb {

typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                    const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                    const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion,
                                    CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
  static PFN_encodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_encodeTiled>(p);
  });
  return fn;
}

bool encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes,
                    const void* base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t bx,
                    uint32_t by, CUtensorMapSwizzle swz) {
  PFN_encodeTiled enc = get_encode();
  if (!enc || !base || rows == 0 || cols == 0) return false;
  // TMA rules: 16-byte aligned base, strides multiple of 16 bytes, inner
  // box extent a multiple of 16 bytes, box dims <= 256.
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
  if (((ld * (uint64_t)elem_bytes) & 15u) != 0) return false;
  if (((uint64_t)bx * elem_bytes) % 16 != 0 || bx > 256 || by > 256) return false;
  if (ld < rows) return false;
  cuuint64_t dims[2] = {rows, cols};
  cuuint64_t strides[1] = {ld * (uint64_t)elem_bytes};
  cuuint32_t box[2] = {bx, by};
  cuuint32_t estr[2] = {1, 1};
  std::memset(map, 0, sizeof(*map));
  CUresult r = enc(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool encode_tmap_3d_u8(CUtensorMap* map, const void* base, uint64_t inner, uint64_t rows,
                       uint64_t planes, uint32_t box_inner, uint32_t box_rows,
                       uint64_t plane_rows) {
  PFN_encodeTiled enc = get_encode();
  if (!enc || !base || inner == 0 || rows == 0 || planes == 0) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (inner & 15u) != 0) return false;
  if (box_inner > 128 || box_rows > 256 || (box_inner & 15u) != 0) return false;
  cuuint64_t dims[3] = {inner, rows, planes};
  if (plane_rows == 0) plane_rows = rows;
  if (plane_rows < rows) return false;
  cuuint64_t strides[2] = {inner, inner * plane_rows};
  cuuint32_t box[3] = {box_inner, box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  std::memset(map, 0, sizeof(*map));
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static cudaStream_t g_lib_stream = nullptr;
static std::atomic<uint64_t> g_launches{0};

cudaStream_t resolve_stream(void* s) {
  return s ? static_cast<cudaStream_t>(s) : g_lib_stream;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

// Events of one host thread (created on its first use, destroyed when it
// exits): the fork / join events of the side streams and the dependency
// events of the blocked factorizations.  Per thread, so that calls made from
// several threads at once never record over each other's events; the
// streams themselves are shared.
namespace {
struct ThreadEvents {
  cudaEvent_t side[kSideStreams][2] = {};
  cudaEvent_t dep[8] = {};
  bool side_ok[kSideStreams] = {}, dep_ok = false, dep_tried = false;
  bool side_tried[kSideStreams] = {};
  ~ThreadEvents() {
    for (auto& p : side)
      for (cudaEvent_t e : p)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : dep)
      if (e) cudaEventDestroy(e);
    cudaGetLastError();  // at process exit the runtime may already be gone
  }
};
ThreadEvents& thread_events() {
  thread_local ThreadEvents te;
  return te;
}
}  // namespace

const SideStream& side_stream(int slot) {
  static cudaStream_t streams[kSideStreams] = {};
  static std::once_flag once[kSideStreams];
  slot = std::max(0, std::min(kSideStreams - 1, slot));
  std::call_once(once[slot], [slot] {
    int least = 0, greatest = 0;
    if (slot >= kHiStream && cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
      cudaGetLastError();
      greatest = 0;
    }
    if (cudaStreamCreateWithPriority(&streams[slot], cudaStreamNonBlocking,
                                     slot >= kHiStream ? greatest : 0) != cudaSuccess) {
      cudaGetLastError();
      streams[slot] = nullptr;
    }
  });
  // the calling thread's fork / join events for this stream
  thread_local SideStream ss[kSideStreams];
  ThreadEvents& te = thread_events();
  if (!te.side_tried[slot]) {
    te.side_tried[slot] = true;
    te.side_ok[slot] =
        cudaEventCreateWithFlags(&te.side[slot][0], cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&te.side[slot][1], cudaEventDisableTiming) == cudaSuccess;
    if (!te.side_ok[slot]) cudaGetLastError();
  }
  SideStream& t = ss[slot];
  t.s = te.side_ok[slot] ? streams[slot] : nullptr;
  t.fork = te.side[slot][0];
  t.join = te.side[slot][1];
  return t;
}

cudaEvent_t* dep_events() {
  ThreadEvents& te = thread_events();
  if (!te.dep_tried) {
    te.dep_tried = true;
    te.dep_ok = true;
    for (auto& e : te.dep)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) te.dep_ok = false;
    if (!te.dep_ok) cudaGetLastError();
  }
  return te.dep_ok ? te.dep : nullptr;
}

cudaStream_t side_fork(const SideStream& side, cudaStream_t st) {
  if (side.s && cudaEventRecord(side.fork, st) == cudaSuccess &&
      cudaStreamWaitEvent(side.s, side.fork, 0) == cudaSuccess)
    return side.s;
  cudaGetLastError();
  return st;
}

bool side_join(const SideStream& side, cudaStream_t forked, cudaStream_t st) {
  if (forked == st) return true;
  return cudaEventRecord(side.join, forked) == cudaSuccess &&
         cudaStreamWaitEvent(st, side.join, 0) == cudaSuccess;
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    n = v;
  }
  return n;
}

static std::vector<ErrReader>& readers() {
  static std::vector<ErrReader> r;
  return r;
}
int register_error_reader(ErrReader r) {
  readers().push_back(r);
  return 1;
}

void set_library_stream(cudaStream_t s) { g_lib_stream = s; }

// ---- trace ring ---------------------------------------------------------------
struct TraceSlot {
  xkb_trace_rec rec;
  cudaEvent_t ev[4];
  bool created = false, pending = false;
};
static std::mutex g_trace_mu;
static bool g_trace_on = false;
static TraceSlot g_trace[256];
static int g_trace_head = 0;  // next slot to write
static int g_trace_count = 0;

bool trace_on() { return g_trace_on; }

int trace_begin(const char* op, int dtype, int M, int N, int K, int nmod, cudaStream_t st) {
  if (!g_trace_on) return -1;
  std::lock_guard<std::mutex> g(g_trace_mu);
  const int i = g_trace_head;
  TraceSlot& t = g_trace[i];
  if (!t.created) {
    for (auto& e : t.ev)
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
    t.created = true;
  }
  std::memset(&t.rec, 0, sizeof(t.rec));
  std::strncpy(t.rec.op, op, sizeof(t.rec.op) - 1);
  t.rec.dtype = dtype;
  t.rec.M = M;
  t.rec.N = N;
  t.rec.K = K;
  t.rec.nmod = nmod;
  t.pending = true;
  g_trace_head = (g_trace_head + 1) % 256;
  if (g_trace_count < 256) ++g_trace_count;
  cudaEventRecord(t.ev[0], st);
  return i;
}

void trace_mark(int slot, int k, cudaStream_t st) {
  if (slot < 0 || k < 1 || k > 3) return;
  cudaEventRecord(g_trace[slot].ev[k], st);
}

}  // namespace xkb

extern "C" int xkb_trace_enable(int on) {
  std::lock_guard<std::mutex> g(xkb::g_trace_mu);
  const int prev = xkb::g_trace_on;
  xkb::g_trace_on = on != 0;
  return prev;
}

extern "C" int xkb_trace_take(xkb_trace_rec* out, int max) {
  using namespace xkb;
  std::lock_guard<std::mutex> g(g_trace_mu);
  int n = 0;
  const int first = (g_trace_head - g_trace_count + 256) % 256;
  for (int c = 0; c < g_trace_count && n < max; ++c) {
    TraceSlot& t = g_trace[(first + c) % 256];
    if (!t.pending) continue;
    if (cudaEventSynchronize(t.ev[3]) != cudaSuccess) continue;
    float a = 0, b = 0, d = 0, tot = 0;
    cudaEventElapsedTime(&tot, t.ev[0], t.ev[3]);
    cudaEventElapsedTime(&a, t.ev[0], t.ev[1]);
    cudaEventElapsedTime(&b, t.ev[1], t.ev[2]);
    cudaEventElapsedTime(&d, t.ev[2], t.ev[3]);
    t.rec.ms_total = tot;
    t.rec.ms_convert = a;
    t.rec.ms_gemm = b;
    t.rec.ms_crt = d;
    t.pending = false;
    if (out) out[n] = t.rec;
    ++n;
  }
  g_trace_count = 0;
  return n;
}

namespace xkb {

}  // namespace xkb

extern "C" int xkb_cuda_take_device_error(void) {
  int v = 0;
  for (auto r : xkb::readers()) {
    int e = r();
    if (e && !v) v = e;
  }
  return v;
}

extern "C" uint64_t xkb_cuda_kernel_count(void) { return xkb::g_launches.load(); }

// ---------------------------------------------------------------------------
// Tuning table: the choices the autotuner (xkblas_b200/autotune.py) measures
// on the device -- tile shapes, the Ozaki / plain crossover, moduli counts
// per K band, the executor's schedule -- as key -> value pairs.  Every key
// has a built-in default; xkb_tune_load reads "key value" lines ('#' starts
// a comment) written by the autotuner.
namespace xkb {
static std::mutex g_tune_mu;
static std::map<std::string, double>& tune_table() {
  static std::map<std::string, double> t;
  return t;
}
double tune(const char* key, double dflt) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto& t = tune_table();
  auto it = t.find(key);
  return it == t.end() ? dflt : it->second;
}
// smallest band "<prefix><K_i>" with K <= K_i; 0 when none covers K
int tune_band(const char* prefix, long K) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  const size_t n = std::strlen(prefix);
  long best_k = -1;
  int best = 0;
  for (auto& kv : tune_table()) {
    if (kv.first.compare(0, n, prefix) != 0) continue;
    const long ki = std::atol(kv.first.c_str() + n);
    if (ki >= K && (best_k < 0 || ki < best_k)) {
      best_k = ki;
      best = (int)kv.second;
    }
  }
  return best;
}
}  // namespace xkb

extern "C" int xkb_tune_set(const char* key, double value) {
  if (!key || !*key) return XKB_EINVAL;
  std::lock_guard<std::mutex> g(xkb::g_tune_mu);
  xkb::tune_table()[key] = value;
  return XKB_OK;
}

extern "C" double xkb_tune_get(const char* key, double dflt) {
  if (!key) return dflt;
  return xkb::tune(key, dflt);
}

extern "C" int xkb_tune_load(const char* path) {
  if (!path) return XKB_EINVAL;
  FILE* f = std::fopen(path, "r");
  if (!f) return XKB_EINVAL;
  char line[512];
  int n = 0;
  while (std::fgets(line, sizeof line, f)) {
    char* hash = std::strchr(line, '#');
    if (hash) *hash = 0;
    char key[256];
    double v;
    if (std::sscanf(line, "%255s %lf", key, &v) == 2) {
      xkb_tune_set(key, v);
      ++n;
    }
  }
  std::fclose(f);
  return n;
}

extern "C" int xkb_tune_clear(void) {
  std::lock_guard<std::mutex> g(xkb::g_tune_mu);
  xkb::tune_table().clear();
  return XKB_OK;
}
