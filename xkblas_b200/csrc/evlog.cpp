// evlog.cpp -- event recorder and CSV export (xkblas_trace_record,
// xkblas_trace_export); see evlog.hpp.
//
// Column layouts follow the reference converter's CSV tables
// (bin/ukilli.cpp:875-1115): times in seconds with 15 decimals, one row per
// event, the same headers, so scripts written for the reference's tables
// read these unchanged.  Resources: host threads are "CPU" resources 0, 1,
// ... in order of first appearance; the GPU is "CUDA" resource = its device
// ordinal.  Streams use the reference's stream table
// (kaapi/kaapi_offload_stream.h:48-52): 0 = H2D, 1 = D2H, 3 = kernels.
#include "evlog.hpp"

#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "xkblas.h"

namespace xkb {
namespace {

constexpr size_t kMaxRecords = 1 << 16;  // per table; later events are counted as dropped

struct DevRec {  // a kernel or a copy, bracketed by two events
  double push = 0;
  cudaEvent_t b = nullptr, e = nullptr;
  int device = 0, stream = 0;
  uint64_t id = 0, bytes = 0;
  int dir = 0;
  bool ended = false;
  char name[64] = {0};
  // executor launch: per-call completion stamps copied back after it
  unsigned long long* h_times = nullptr;  // pinned, n + 1 entries
  cudaEvent_t e_times = nullptr;
  int ncalls = 0;
  std::vector<std::string> call_names;
  uint64_t first_call_id = 0;
};

struct CallRec {
  int thread = 0;
  double start = 0, ret = 0, end = 0;
  bool closed = false, task_written = false;
  int level = 0, nparam = 0;
  uint64_t id = 0;
  uint64_t p[16] = {0};
  char name[8] = {0};
};

struct Log {
  std::mutex mu;
  std::atomic<bool> on{false};
  std::chrono::steady_clock::time_point t0;
  cudaEvent_t base = nullptr;
  double base_s = 0;  // host time of the base event, seconds since t0
  int base_dev = -1;
  std::vector<DevRec> kern, cpy;
  std::vector<CallRec> calls;
  std::vector<cudaEvent_t> spare;
  std::map<std::thread::id, int> threads;
  std::map<int, int> devices;  // device ordinal -> seen
  uint64_t next_id = 1, dropped = 0;
};

Log& L() {
  static Log* l = new Log();  // never destroyed: usable from atexit paths
  return *l;
}

thread_local const char* t_name = nullptr;

double now_s(const Log& l) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - l.t0).count();
}

int thread_index(Log& l) {
  auto it = l.threads.find(std::this_thread::get_id());
  if (it != l.threads.end()) return it->second;
  const int i = (int)l.threads.size();
  l.threads.emplace(std::this_thread::get_id(), i);
  return i;
}

cudaEvent_t take_event(Log& l) {
  if (!l.spare.empty()) {
    cudaEvent_t e = l.spare.back();
    l.spare.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

// The base event pins device time to host time: recorded on the legacy
// stream, waited for, and stamped with the host clock right after.
bool ensure_base(Log& l) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (l.base && l.base_dev == dev) return true;
  if (l.base) return false;  // one device per recording
  if (cudaEventCreate(&l.base) != cudaSuccess || cudaEventRecord(l.base, 0) != cudaSuccess ||
      cudaEventSynchronize(l.base) != cudaSuccess) {
    cudaGetLastError();
    if (l.base) cudaEventDestroy(l.base);
    l.base = nullptr;
    return false;
  }
  l.base_s = now_s(l);
  l.base_dev = dev;
  l.devices[dev] = 1;
  return true;
}

long long dev_begin(std::vector<DevRec>& tab, cudaStream_t st, int stream, const char* name,
                    size_t bytes, int dir) {
  Log& l = L();
  if (!l.on.load(std::memory_order_relaxed)) return -1;
  std::lock_guard<std::mutex> g(l.mu);
  if (!l.on.load()) return -1;
  if (tab.size() >= kMaxRecords || !ensure_base(l)) {
    ++l.dropped;
    return -1;
  }
  DevRec r;
  r.push = now_s(l);
  r.b = take_event(l);
  r.e = take_event(l);
  if (!r.b || !r.e) {
    if (r.b) l.spare.push_back(r.b);
    if (r.e) l.spare.push_back(r.e);
    ++l.dropped;
    return -1;
  }
  r.device = l.base_dev;
  r.stream = stream;
  r.id = l.next_id++;
  r.bytes = bytes;
  r.dir = dir;
  if (name) {
    if (t_name)
      std::snprintf(r.name, sizeof(r.name), "%s/%s", t_name, name);
    else
      std::snprintf(r.name, sizeof(r.name), "%s", name);
  }
  cudaEventRecord(r.b, st);
  tab.push_back(r);
  return (long long)r.id;
}

void dev_end(std::vector<DevRec>& tab, long long id, cudaStream_t st) {
  if (id < 0) return;
  Log& l = L();
  std::lock_guard<std::mutex> g(l.mu);
  for (size_t i = tab.size(); i-- > 0;)  // the record is nearly always the last one
    if (tab[i].id == (uint64_t)id) {
      cudaEventRecord(tab[i].e, st);
      tab[i].ended = true;
      return;
    }
}

void release_calls(DevRec& r, Log& l) {
  if (r.h_times) cudaFreeHost(r.h_times);
  if (r.e_times) l.spare.push_back(r.e_times);
  r.h_times = nullptr;
  r.e_times = nullptr;
}

// device time of `e` in seconds since t0; false if it cannot be read
bool dev_time(Log& l, cudaEvent_t e, double* t) {
  float ms = 0;
  if (cudaEventSynchronize(e) != cudaSuccess || cudaEventElapsedTime(&ms, l.base, e) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  *t = l.base_s + 1e-3 * (double)ms;
  return true;
}

FILE* open_table(const std::string& dir, const char* file, const char* header) {
  const std::string path = dir + "/" + file;
  FILE* f = std::fopen(path.c_str(), "w");
  if (f) std::fprintf(f, "%s\n", header);
  return f;
}

}  // namespace

bool evlog_on() { return L().on.load(std::memory_order_relaxed); }

long long evlog_kern_begin(cudaStream_t st, const char* kernel) {
  return dev_begin(L().kern, st, 3, kernel, 0, 0);
}
void evlog_kern_end(long long id, cudaStream_t st) { dev_end(L().kern, id, st); }

void evlog_kern_calls(long long id, cudaStream_t st, const unsigned long long* d_times, int n,
                      const char* const* names) {
  if (id < 0 || n <= 0 || !d_times) return;
  Log& l = L();
  std::lock_guard<std::mutex> g(l.mu);
  for (size_t i = l.kern.size(); i-- > 0;) {
    DevRec& r = l.kern[i];
    if (r.id != (uint64_t)id) continue;
    void* h = nullptr;
    if (cudaMallocHost(&h, ((size_t)n + 1) * sizeof(unsigned long long)) != cudaSuccess) {
      cudaGetLastError();
      ++l.dropped;
      return;
    }
    r.h_times = static_cast<unsigned long long*>(h);
    r.e_times = take_event(l);
    if (!r.e_times ||
        cudaMemcpyAsync(r.h_times, d_times, ((size_t)n + 1) * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaEventRecord(r.e_times, st) != cudaSuccess) {
      cudaGetLastError();
      release_calls(r, l);
      ++l.dropped;
      return;
    }
    r.ncalls = n;
    r.call_names.assign(names, names + n);
    r.first_call_id = l.next_id;
    l.next_id += (uint64_t)n;
    return;
  }
}

long long evlog_copy_begin(cudaStream_t st, size_t bytes, int dir) {
  return dev_begin(L().cpy, st, dir == 1 ? 0 : 1, nullptr, bytes, dir);
}
void evlog_copy_end(long long id, cudaStream_t st) { dev_end(L().cpy, id, st); }

EvCall::EvCall(const char* name, std::initializer_list<uint64_t> params) {
  prev_ = t_name;
  Log& l = L();
  if (!l.on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> g(l.mu);
  if (!l.on.load()) return;
  t_name = name;
  if (l.calls.size() >= kMaxRecords) {
    ++l.dropped;
    return;
  }
  CallRec c;
  c.thread = thread_index(l);
  c.start = now_s(l);
  c.id = l.next_id++;
  std::strncpy(c.name, name, sizeof(c.name) - 1);  // 7 characters, as the reference
  for (uint64_t v : params)
    if (c.nparam < 16) c.p[c.nparam++] = v;
  l.calls.push_back(c);
  id_ = c.id;
}

EvCall::~EvCall() {
  t_name = prev_;
  if (!id_) return;
  Log& l = L();
  std::lock_guard<std::mutex> g(l.mu);
  for (size_t i = l.calls.size(); i-- > 0;)
    if (l.calls[i].id == id_) {
      l.calls[i].ret = now_s(l);
      return;
    }
}

EvName::EvName(const char* name) : prev_(t_name) { t_name = name; }
EvName::~EvName() { t_name = prev_; }

void evlog_sync_done() {
  Log& l = L();
  if (!l.on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> g(l.mu);
  const int me = thread_index(l);
  const double t = now_s(l);
  int level = 0;
  for (CallRec& c : l.calls)
    if (!c.closed && c.thread == me) {
      c.end = t;
      c.level = level++;
      c.closed = true;
    }
}

}  // namespace xkb

extern "C" int xkblas_trace_record(int on) {
  using namespace xkb;
  Log& l = L();
  std::lock_guard<std::mutex> g(l.mu);
  const bool prev = l.on.load();
  if (on && !prev && l.kern.empty() && l.cpy.empty() && l.calls.empty()) {
    l.t0 = std::chrono::steady_clock::now();  // a fresh recording starts its clock
    if (l.base) cudaEventDestroy(l.base);
    l.base = nullptr;
    l.base_dev = -1;
  }
  l.on.store(on != 0);
  return prev ? 1 : 0;
}

extern "C" int xkblas_trace_export(const char* dir) {
  using namespace xkb;
  if (!dir || !*dir) return EINVAL;
  Log& l = L();
  std::lock_guard<std::mutex> g(l.mu);
  const std::string d(dir);
  // headers: bin/ukilli.cpp:887-889, 916-918, 934-936, 952-954, 966-971
  FILE* fk = open_table(d, "kern.csv", "Resource,Type,Stream,Push,Start,End,Duration,Name,TaskId");
  FILE* fc = open_table(d, "cpy.csv", "Resource,Type,Stream,Push,Start,End,Duration,Size,Dir");
  FILE* ft = open_table(d, "task.csv", "Resource,Type,Push,Start,End,Duration,Name,TaskId");
  FILE* fp = open_table(d, "parallel.csv", "Resource,Type,Start,End,Duration,Name");
  std::string call_hdr = "Resource,Level,Start,End,Duration,Name,NParam";
  for (int i = 0; i < 16; ++i) call_hdr += ",Param" + std::to_string(i);
  FILE* fl = open_table(d, "call.csv", call_hdr.c_str());
  int rc = (fk && fc && ft && fp && fl) ? 0 : EIO;
  if (rc == 0) {
    std::vector<DevRec> kept_k, kept_c;
    for (const DevRec& r : l.kern) {
      double s, e;
      if (!r.ended) {
        kept_k.push_back(r);
        continue;
      }
      if (!dev_time(l, r.b, &s) || !dev_time(l, r.e, &e)) {
        ++l.dropped;
        continue;
      }
      std::fprintf(fk, "%i,CUDA,%i,%.15f,%.15f,%.15f,%.15f,%s,%llu\n", r.device, r.stream, r.push,
                   s, e, e - s, r.name, (unsigned long long)r.id);
      if (r.h_times && r.e_times && cudaEventSynchronize(r.e_times) == cudaSuccess) {
        const unsigned long long t0 = r.h_times[r.ncalls];
        for (int i = 0; i < r.ncalls; ++i) {
          const unsigned long long ti = r.h_times[i];
          if (!ti || ti < t0) continue;  // a call without tasks
          const double ce = s + 1e-9 * (double)(ti - t0);
          std::fprintf(fk, "%i,CUDA,%i,%.15f,%.15f,%.15f,%.15f,batch/%s#%i,%llu\n", r.device,
                       r.stream, r.push, s, ce, ce - s, r.call_names[i].c_str(), i,
                       (unsigned long long)(r.first_call_id + (uint64_t)i));
        }
      } else if (r.h_times) {
        cudaGetLastError();
      }
    }
    for (const DevRec& r : l.cpy) {
      double s, e;
      if (!r.ended) {
        kept_c.push_back(r);
        continue;
      }
      if (!dev_time(l, r.b, &s) || !dev_time(l, r.e, &e)) {
        ++l.dropped;
        continue;
      }
      std::fprintf(fc, "%i,CUDA,%i,%.15f,%.15f,%.15f,%.15f,%llu,%i\n", r.device, r.stream, r.push,
                   s, e, e - s, (unsigned long long)r.bytes, r.dir);
    }
    std::vector<CallRec> open;
    for (CallRec& c : l.calls) {
      // the host part of the call (entry to return) as a task of its thread
      if (!c.task_written && c.ret > 0) {
        std::fprintf(ft, "%i,CPU,%.15f,%.15f,%.15f,%.15f,%s,%llu\n", c.thread, c.start, c.start,
                     c.ret, c.ret - c.start, c.name, (unsigned long long)c.id);
        c.task_written = true;
      }
      if (!c.closed) {
        open.push_back(c);
        continue;
      }
      std::fprintf(fl, "%i,%i,%.15f,%.15f,%.15f,%s,%i", c.thread, c.level, c.start, c.end,
                   c.end - c.start, c.name, c.nparam);
      for (int i = 0; i < 16; ++i)
        std::fprintf(fl, ",%llu", (unsigned long long)(i < c.nparam ? c.p[i] : 0));
      std::fprintf(fl, "\n");
    }
    const double t = now_s(l);
    for (const auto& kv : l.threads)
      std::fprintf(fp, "%i,CPU,%.15f,%.15f,%.15f,CPU-%i\n", kv.second, 0.0, t, t, kv.second);
    for (const auto& kv : l.devices)
      std::fprintf(fp, "%i,CUDA,%.15f,%.15f,%.15f,CUDA-%i\n", kv.first, 0.0, t, t, kv.first);
    // the written events leave the log; launches still open and calls not
    // yet closed by a sync stay
    for (std::vector<DevRec>* tab : {&l.kern, &l.cpy})
      for (DevRec& r : *tab)
        if (r.ended) {
          l.spare.push_back(r.b);
          l.spare.push_back(r.e);
          release_calls(r, l);
        }
    l.kern.swap(kept_k);
    l.cpy.swap(kept_c);
    l.calls.swap(open);
  }
  for (FILE* f : {fk, fc, ft, fp, fl})
    if (f && std::fclose(f) != 0) rc = EIO;
  return rc;
}

extern "C" uint64_t xkblas_trace_dropped(void) {
  xkb::Log& l = xkb::L();
  std::lock_guard<std::mutex> g(l.mu);
  return l.dropped;
}
