// potrf.cu -- Cholesky factorization on the device: A = L L^H (lower) or
// A = U^H U (upper), in place, for s/d/c/z.
//
// Replaces the reference's tile Cholesky driver (blas/zpotrf.c:46-220:
// diagonal zpotrf tasks, trsm right/lower/conj-trans of the panel, herk and
// gemm of the trailing tiles) and its diagonal-tile body (cuSOLVER potrf in
// ztask_potrf.c).  Here the factorization is recursive on the matrix index
// (split points multiple of 64): factor the leading block, solve the panel
// against it with xkb_cuda_trsm (FP64 leaves + DMMA GEMMs), update the
// trailing block with one triangle-masked GEMM (the HERK/SYRK of the
// reference: C = C - P P^H, only the stored triangle written), factor the
// trailing block.  Blocks of <= 64 are factored in FP64 by k_potrf_leaf
// (register-resident elements, one CTA).
// A non-positive (or non-finite) pivot stops nothing on the device -- later
// blocks become NaN as in LAPACK's unchecked use -- but the first failing
// column (1-based, over the whole matrix) is recorded in *d_info (0 = none).
#include <algorithm>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {

constexpr int kPotrfLeaf = 64;

// Factor the n x n (n <= 64) Hermitian block at A in place.  The block is
// read as its lower triangle L (upper: L = U^H, read transposed and
// conjugated) and factored right-looking column by column.  Element (i, k)
// of the triangle lives in a register of thread ((i + k) mod 256) -- 8 or 9
// elements per thread; per column j the pivot and the scaled column go
// through shared memory (two barriers), and every thread updates its own
// elements L(i,k) -= L(i,j) conj(L(k,j)), k > j.  Written back to the stored
// triangle only.
constexpr int kPotrfThreads = 256;
constexpr int kPotrfPer = (kPotrfLeaf * (kPotrfLeaf + 1) / 2 + kPotrfThreads - 1) / kPotrfThreads;

template <class T>
__global__ void __launch_bounds__(kPotrfThreads) k_potrf_leaf(int n, typename St<T>::S* A,
                                                              long lda, int upper, int col0,
                                                              int* info) {
  constexpr bool CP = St<T>::CPLX;
  using S = typename St<T>::S;
  __shared__ double cr[kPotrfLeaf], ci[kPotrfLeaf];  // column j after scaling
  __shared__ int s_bad;
  // this thread's elements: the e-th element of the packed lower triangle
  // (column-major, (i, k) with i >= k) for e = tid + 256 q
  int ei[kPotrfPer], ek[kPotrfPer];
  double vr[kPotrfPer], vi[kPotrfPer];
#pragma unroll
  for (int q = 0; q < kPotrfPer; ++q) {
    const int e = threadIdx.x + q * kPotrfThreads;
    // column k holds n - k elements: find k, i for packed index e
    int k = 0, base = 0;
    while (k < kPotrfLeaf && base + (kPotrfLeaf - k) <= e) {
      base += kPotrfLeaf - k;
      ++k;
    }
    const int i = k + (e - base);
    ei[q] = i;
    ek[q] = k;
    vr[q] = vi[q] = 0.0;
    if (k < kPotrfLeaf && i < n && k < n) {
      const size_t idx = upper ? (size_t)k + (size_t)i * lda : (size_t)i + (size_t)k * lda;
      if (CP) {
        vr[q] = (double)A[2 * idx];
        vi[q] = (i == k) ? 0.0 : (upper ? -(double)A[2 * idx + 1] : (double)A[2 * idx + 1]);
      } else {
        vr[q] = (double)A[idx];
      }
    } else {
      ei[q] = -1;  // padding slot
    }
  }
  if (threadIdx.x == 0) s_bad = 0;
  int j = 0;
  for (; j < n; ++j) {
    // 1. the owner of (j, j) publishes the pivot; owners of column j publish it
#pragma unroll
    for (int q = 0; q < kPotrfPer; ++q)
      if (ek[q] == j && ei[q] >= 0) {
        cr[ei[q]] = vr[q];
        if (CP) ci[ei[q]] = vi[q];
      }
    __syncthreads();
    const double d = cr[j];
    if (!(d > 0.0)) {  // non-positive or NaN pivot: uniform decision
      if (threadIdx.x == 0 && info) atomicCAS(info, 0, col0 + j + 1);
      break;
    }
    const double ljj = sqrt(d), inv = 1.0 / ljj;
    // 2. scale column j in place (owners) and in the shared copy
#pragma unroll
    for (int q = 0; q < kPotrfPer; ++q)
      if (ek[q] == j && ei[q] >= 0) {
        if (ei[q] == j) {
          vr[q] = ljj;
        } else {
          vr[q] *= inv;
          if (CP) vi[q] *= inv;
        }
      }
    __syncthreads();  // everyone read cr[j] before it is overwritten below
    if (threadIdx.x < kPotrfLeaf && threadIdx.x > j && threadIdx.x < n) {
      cr[threadIdx.x] *= inv;
      if (CP) ci[threadIdx.x] *= inv;
    }
    __syncthreads();
    // 3. trailing update of this thread's elements, column k > j
#pragma unroll
    for (int q = 0; q < kPotrfPer; ++q) {
      const int i = ei[q], k = ek[q];
      if (i >= 0 && k > j && i < n) {
        const double ar = cr[i], br = cr[k];
        if (CP) {
          const double ai = ci[i], bi = ci[k];
          vr[q] -= ar * br + ai * bi;  // L(i,j) conj(L(k,j))
          if (i != k) vi[q] -= ai * br - ar * bi;
        } else {
          vr[q] -= ar * br;
        }
      }
    }
    __syncthreads();  // column j + 1 is published next
  }
  // write back the stored triangle (columns past a failure hold partial values)
#pragma unroll
  for (int q = 0; q < kPotrfPer; ++q) {
    const int i = ei[q], k = ek[q];
    if (i < 0 || i >= n || k >= n) continue;
    const size_t idx = upper ? (size_t)k + (size_t)i * lda : (size_t)i + (size_t)k * lda;
    if (CP) {
      A[2 * idx] = static_cast<S>(vr[q]);
      A[2 * idx + 1] = static_cast<S>(upper ? -vi[q] : vi[q]);
    } else {
      A[idx] = static_cast<S>(vr[q]);
    }
  }
  (void)s_bad;
}

struct PotrfCtx {
  int dt, es, upper;
  char* A;
  long lda;
  int* info;
  cudaStream_t st;
};

template <class T>
static int launch_leaf(const PotrfCtx& c, char* Ad, long n, long i0) {
  k_potrf_leaf<T><<<1, kPotrfThreads, 0, c.st>>>(
      (int)n, reinterpret_cast<typename St<T>::S*>(Ad), c.lda, c.upper, (int)i0, c.info);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static int leaf(const PotrfCtx& c, long i0, long n) {
  char* Ad = c.A + (i0 + i0 * c.lda) * (long)c.es;
  switch (c.dt) {
    case XKB_S: return launch_leaf<float>(c, Ad, n, i0);
    case XKB_D: return launch_leaf<double>(c, Ad, n, i0);
    case XKB_C: return launch_leaf<float2>(c, Ad, n, i0);
    case XKB_Z: return launch_leaf<double2>(c, Ad, n, i0);
  }
  return XKB_EINVAL;
}

static int factor(const PotrfCtx& c, long i0, long i1) {
  const long n = i1 - i0;
  if (n <= kPotrfLeaf) return leaf(c, i0, n);
  long h = i0 + ((n / 2 + kPotrfLeaf - 1) / kPotrfLeaf) * kPotrfLeaf;
  if (h >= i1) h = i1 - kPotrfLeaf;
  const long n1 = h - i0, n2 = i1 - h;
  int e;
  if ((e = factor(c, i0, h))) return e;
  const bool cplx = c.dt == XKB_C || c.dt == XKB_Z;
  const int ctr = cplx ? XKB_OP_C : XKB_OP_T;
  const double one[2] = {1.0, 0.0};
  char* A11 = c.A + (i0 + i0 * c.lda) * (long)c.es;
  char* A22 = c.A + (h + h * c.lda) * (long)c.es;
  char* P;  // the panel: A21 (lower) or A12 (upper)
  xkb_gemm_args g{};
  g.dtype = c.dt;
  g.alpha[0] = -1.0;
  g.beta[0] = 1.0;
  g.M = g.N = (int)n2;
  g.K = (int)n1;
  g.C = A22;
  g.ldc = c.lda;
  g.herm_diag = cplx ? 1 : 0;
  if (!c.upper) {
    // A21 = A21 L11^-H; A22 -= A21 A21^H (lower triangle)
    P = c.A + (h + i0 * c.lda) * (long)c.es;
    if ((e = xkb_cuda_trsm(c.dt, 1, XKB_LOWER, ctr, 0, (int)n2, (int)n1, one, A11, c.lda, P,
                           c.lda, 0, c.st)))
      return e;
    g.opA = XKB_OP_N;
    g.opB = ctr;
    g.uplo = XKB_LOWER;
  } else {
    // A12 = U11^-H A12; A22 -= A12^H A12 (upper triangle)
    P = c.A + (i0 + h * c.lda) * (long)c.es;
    if ((e = xkb_cuda_trsm(c.dt, 0, XKB_UPPER, ctr, 0, (int)n1, (int)n2, one, A11, c.lda, P,
                           c.lda, 0, c.st)))
      return e;
    g.opA = ctr;
    g.opB = XKB_OP_N;
    g.uplo = XKB_UPPER;
  }
  g.A = P;
  g.lda = c.lda;
  g.B = P;
  g.ldb = c.lda;
  if ((e = xkb_cuda_gemm(&g, c.st))) return e;
  return factor(c, h, i1);
}

}  // namespace xkb

using namespace xkb;

extern "C" int xkb_cuda_potrf(int dtype, int uplo, int N, void* A, long lda, int* d_info,
                              void* stream) {
  if (dtype < XKB_S || dtype > XKB_Z || (uplo != XKB_LOWER && uplo != XKB_UPPER) || N < 0 ||
      lda < std::max(1, N) || (!A && N > 0))
    return XKB_EINVAL;
  if (N == 0) return XKB_OK;
  PotrfCtx c;
  c.dt = dtype;
  c.es = dtype == XKB_S ? 4 : (dtype == XKB_Z ? 16 : 8);
  c.upper = uplo == XKB_UPPER ? 1 : 0;
  c.A = static_cast<char*>(A);
  c.lda = lda;
  c.info = d_info;
  c.st = resolve_stream(stream);
  return factor(c, 0, N);
}
