// runtime_cuda.cu -- host helpers under the thin C ABI: tensor-map encoding
// through the driver entry point (no link-time libcuda dependency, so the
// library loads on machines without a GPU driver), stream resolution,
// launch accounting and the device error word readers.
#include <atomic>
#include <cstring>
#include <mutex>
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

static cudaStream_t g_lib_stream = nullptr;
static std::atomic<uint64_t> g_launches{0};

cudaStream_t resolve_stream(void* s) {
  return s ? static_cast<cudaStream_t>(s) : g_lib_stream;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

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
