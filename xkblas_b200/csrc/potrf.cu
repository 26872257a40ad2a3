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
// trailing block.  Blocks of <= 64 are factored in FP64 by k_potrf_leaf.
// A non-positive (or non-finite) pivot stops nothing on the device -- later
// blocks become NaN as in LAPACK's unchecked use -- but the first failing
// column (1-based, over the whole matrix) is recorded in *d_info (0 = none).
#include <algorithm>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {

constexpr int kPotrfLeaf = 64;

// Factor the n x n (n <= 64) Hermitian block at A in place.  The block is
// staged as its lower triangle L (upper: L = U^H, read transposed and
// conjugated), factored right-looking column by column in shared memory,
// and written back to the stored triangle only.
template <class T>
__global__ void __launch_bounds__(256) k_potrf_leaf(int n, typename St<T>::S* A, long lda,
                                                    int upper, int col0, int* info) {
  constexpr bool CP = St<T>::CPLX;
  using S = typename St<T>::S;
  extern __shared__ double sm_potrf[];  // Lr (and Li): 64 x 65 doubles each
  double (*Lr)[kPotrfLeaf + 1] = reinterpret_cast<double (*)[kPotrfLeaf + 1]>(sm_potrf);
  double (*Li)[kPotrfLeaf + 1] =
      reinterpret_cast<double (*)[kPotrfLeaf + 1]>(sm_potrf + kPotrfLeaf * (kPotrfLeaf + 1));
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;  // L(i, j), i >= j
    if (i < j) continue;
    const size_t idx = upper ? (size_t)j + (size_t)i * lda : (size_t)i + (size_t)j * lda;
    double re, im = 0.0;
    if (CP) {
      re = (double)A[2 * idx];
      im = (double)A[2 * idx + 1];
      if (upper) im = -im;  // L = U^H
    } else {
      re = (double)A[idx];
    }
    Lr[i][j] = re;
    if (CP) Li[i][j] = (i == j) ? 0.0 : im;  // Hermitian: real diagonal
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double d = Lr[j][j];
    if (!(d > 0.0)) {  // non-positive or NaN pivot
      if (threadIdx.x == 0 && info) atomicCAS(info, 0, col0 + j + 1);
      __syncthreads();
      break;
    }
    const double ljj = sqrt(d);
    const double inv = 1.0 / ljj;
    __syncthreads();  // every thread has read the pivot
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      Lr[i][j] *= inv;
      if (CP) Li[i][j] *= inv;
    }
    if (threadIdx.x == 0) Lr[j][j] = ljj;
    __syncthreads();
    // trailing update: L(i,k) -= L(i,j) conj(L(k,j)), j < k <= i < n
    const int m = n - j - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = j + 1 + e % m, k = j + 1 + e / m;
      if (k > i) continue;
      const double ar = Lr[i][j], br = Lr[k][j];
      if (CP) {
        const double ai = Li[i][j], bi = Li[k][j];
        Lr[i][k] -= ar * br + ai * bi;  // (ar + i ai)(br - i bi)
        if (i != k) Li[i][k] -= ai * br - ar * bi;
      } else {
        Lr[i][k] -= ar * br;
      }
    }
    __syncthreads();
  }
  // write back the stored triangle (columns past a failure hold partial values)
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    if (i < j) continue;
    const size_t idx = upper ? (size_t)j + (size_t)i * lda : (size_t)i + (size_t)j * lda;
    if (CP) {
      A[2 * idx] = static_cast<S>(Lr[i][j]);
      A[2 * idx + 1] = static_cast<S>(upper ? -Li[i][j] : Li[i][j]);
    } else {
      A[idx] = static_cast<S>(Lr[i][j]);
    }
  }
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
  constexpr size_t smem = (St<T>::CPLX ? 2 : 1) * sizeof(double) * kPotrfLeaf * (kPotrfLeaf + 1);
  static bool attr = false;  // one per instantiation
  if (!attr) {
    if (cudaFuncSetAttribute(k_potrf_leaf<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  k_potrf_leaf<T><<<1, 256, smem, c.st>>>((int)n, reinterpret_cast<typename St<T>::S*>(Ad),
                                           c.lda, c.upper, (int)i0, c.info);
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
