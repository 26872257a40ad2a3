// dmma_common.cuh -- storage-type traits and FP64 DMMA fragment helpers
// shared by the whole-matrix GEMM (gemm_dmma.cu) and the tile-task executor
// (sched.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "xkb_cuda.h"

namespace xkb {

template <class T>
struct St;
template <>
struct St<float> {
  using S = float;
  static constexpr int W = 1;
  static constexpr bool CPLX = false;
  static constexpr CUtensorMapDataType DT = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
};
template <>
struct St<double> {
  using S = double;
  static constexpr int W = 1;
  static constexpr bool CPLX = false;
  static constexpr CUtensorMapDataType DT = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
};
template <>
struct St<float2> {
  using S = float;
  static constexpr int W = 2;
  static constexpr bool CPLX = true;
  static constexpr CUtensorMapDataType DT = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
};
template <>
struct St<double2> {
  using S = double;
  static constexpr int W = 2;
  static constexpr bool CPLX = true;
  static constexpr CUtensorMapDataType DT = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
};

__device__ __forceinline__ void dmma_k8(double (&d)[4], const double (&a)[4],
                                        const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <class T>
__device__ __forceinline__ void ld_elem(const typename St<T>::S* s, int e, double& re,
                                        double& im) {
  if constexpr (St<T>::CPLX) {
    re = static_cast<double>(s[2 * e]);
    im = static_cast<double>(s[2 * e + 1]);
  } else {
    re = static_cast<double>(s[e]);
    im = 0.0;
  }
}

__device__ __forceinline__ bool in_mask(int uplo, long diag, int row, int col) {
  if (uplo == XKB_LOWER) return (long)row + diag >= (long)col;
  if (uplo == XKB_UPPER) return (long)row + diag <= (long)col;
  return true;
}

}  // namespace xkb
