// ozaki.cu -- FP64 contraction on INT8 tensor cores (Ozaki scheme II).
// Placeholder entry points until the tcgen05 pipeline lands: they report
// ERANGE so the caller runs the plain DMMA contraction.
#include "xkb_dev.cuh"

extern "C" int xkb_ozaki_default_moduli(long K) {
  (void)K;
  return 0;
}

extern "C" int xkb_cuda_ozaki_gemm(const xkb_gemm_args* a, int nmod, void* stream) {
  (void)a;
  (void)nmod;
  (void)stream;
  return XKB_ERANGE;
}
