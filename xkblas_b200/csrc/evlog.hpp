// evlog.hpp -- event recorder behind xkblas_trace_record / xkblas_trace_export.
//
// The reference records binary KAAPI events (kaapi/kaapi_trace_lib.c:754-840,
// enabled by KAAPI_RECORD_TRACE) and converts them post mortem with
// bin/ukilli.cpp into CSV tables (csv_parallel_region_t, ukilli.cpp:875-1115).
// Here the library records the same kinds of events directly -- kernel
// launches and host<->device copies bracketed by CUDA events on their
// streams, API calls by host clocks -- and writes those tables itself.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <initializer_list>

namespace xkb {

bool evlog_on();
// A kernel launch on `st`: begin before the launch, end right after it.
// Returns -1 (and records nothing) while recording is off.
long long evlog_kern_begin(cudaStream_t st, const char* kernel);
void evlog_kern_end(long long id, cudaStream_t st);
// The executor launch `id` ran `n` calls: `d_times` holds, in globaltimer
// nanoseconds, each call's completion (0 if it had no task) followed by the
// launch's first task start; they are copied back on `st` after the launch
// and written as one row per call ("batch/<name>#<i>", start = the launch's
// start, end = start + the call's completion delay).
void evlog_kern_calls(long long id, cudaStream_t st, const unsigned long long* d_times, int n,
                      const char* const* names);
// A host<->device copy of `bytes` on `st`; dir uses the reference's
// direction table (bin/ukilli.cpp:223): 1 = H2D, 2 = D2H.
long long evlog_copy_begin(cudaStream_t st, size_t bytes, int dir);
void evlog_copy_end(long long id, cudaStream_t st);

// One API call (reference: the KAAPI_EVT_CALL begin / info events of each
// level-3 driver, e.g. blas/zgemm.c:259-276): name and up to 16 parameters.
// Kernels launched on this thread while the scope lives carry its name.
class EvCall {
 public:
  EvCall(const char* name, std::initializer_list<uint64_t> params);
  ~EvCall();
  EvCall(const EvCall&) = delete;
  EvCall& operator=(const EvCall&) = delete;

 private:
  uint64_t id_ = 0;
  const char* prev_ = nullptr;
};

// Names the kernels launched on this thread while it lives (deferred calls
// launched by a later flush keep their own name).
class EvName {
 public:
  explicit EvName(const char* name);
  ~EvName();
  EvName(const EvName&) = delete;
  EvName& operator=(const EvName&) = delete;

 private:
  const char* prev_ = nullptr;
};

// xkblas_sync completed: the calls issued before it end now (the reference
// closes its open call records at the task-sync event, ukilli.cpp:762-775).
void evlog_sync_done();

}  // namespace xkb
