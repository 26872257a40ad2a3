// trsm.cu -- triangular solve / multiply and symmetric multiply on the device.
//
// Replaces the reference's diagonal-tile bodies cublasZtrsm
// (blas/ztask_trsm.c:172), cublasZtrmm (ztask_trmm.c:156) and cublasZsymm /
// cublasZhemm (ztask_symm.c:133, ztask_hemm.c:132), and the tile loops around
// them (blas/ztrsm.c:243-499).
//
// TRSM is solved recursively on the system index: the triangle is split in
// two (split points multiple of 64), the leading half is solved, the coupling
// block is applied to the trailing half as one GEMM (DMMA, or Ozaki when
// requested and large), and the trailing half is solved.  Leaves of <= 64
// unknowns are solved in FP64 by k_trsm_leaf (trsm_leaf.cuh): each
// right-hand side held in the registers of a few lanes, the 64x64 triangle in
// shared memory, about two CTAs per SM.
// This keeps every flop except O(n * 64 * nrhs) inside large GEMMs.
#include <algorithm>

#include "trsm_leaf.cuh"
#include "xkb_dev.cuh"

namespace xkb {

constexpr int kLeaf = 64;

template <class T>
struct TT;
template <>
struct TT<float> {
  using S = float;
  static constexpr bool C = false;
};
template <>
struct TT<double> {
  using S = double;
  static constexpr bool C = false;
};
template <>
struct TT<float2> {
  using S = float;
  static constexpr bool C = true;
};
template <>
struct TT<double2> {
  using S = double;
  static constexpr bool C = true;
};

template <class T>
__device__ __forceinline__ void ldv(const T* p, size_t i, double& re, double& im) {
  using S = typename TT<T>::S;
  const S* s = reinterpret_cast<const S*>(p);
  if constexpr (TT<T>::C) {
    re = (double)s[2 * i];
    im = (double)s[2 * i + 1];
  } else {
    re = (double)s[i];
    im = 0.0;
  }
}
template <class T>
__device__ __forceinline__ void stv(T* p, size_t i, double re, double im) {
  using S = typename TT<T>::S;
  S* s = reinterpret_cast<S*>(p);
  if constexpr (TT<T>::C) {
    s[2 * i] = (S)re;
    s[2 * i + 1] = (S)im;
  } else {
    s[i] = (S)re;
  }
}

// Leaf solve: T x = alpha b for the right-hand sides of this CTA's column
// range, T (n x n, n <= 64) the effective triangle: T(i,j) = A[swap ? j + i*lda
// : i + j*lda] (conjugated when conj), lower when LOWER.  RHS c, unknown i
// lives at B[rhs_rows ? c + i*ldb : i + c*ldb] (rhs_rows: the right-side
// form).  Body: trsm_leaf.cuh (register-resident substitution).
constexpr int kLeafThreads = 128;
constexpr int kLeafRplReal = 8;  // many right-hand sides: more lanes per column

template <class T, bool LOWER>
__global__ void __launch_bounds__(kLeafThreads)
    k_trsm_leaf(int n, int nrhs, int cols_per_cta, const typename St<T>::S* A, long lda, int swap,
                int conj, int unit, typename St<T>::S* B, long ldb, int rhs_rows, double ar,
                double ai) {
  extern __shared__ double sm_leaf[];
  leaf_stage<T, kLeafThreads, kLeafRplReal>(A, lda, n, swap != 0, conj != 0, LOWER, unit != 0,
                                            sm_leaf);
  const int c0 = blockIdx.x * cols_per_cta;
  const int c1 = min(nrhs, c0 + cols_per_cta);
  leaf_solve<T, kLeafThreads, LOWER, kLeafRplReal>(B, ldb, rhs_rows != 0, n, c0, c1, ar, ai,
                                                   sm_leaf);
}

template <class T>
__global__ void k_tri_fill(int n, const T* A, long lda, int lower, int unit, T* O, long ldo) {
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    double re = 0, im = 0;
    if (i == j && unit) re = 1.0;
    else if (lower ? i >= j : i <= j) ldv<T>(A, (size_t)i + (size_t)j * lda, re, im);
    stv<T>(O, (size_t)i + (size_t)j * ldo, re, im);
  }
}

// out = full symmetric (herm = 0) or Hermitian (herm = 1) matrix from the
// stored uplo triangle of A; Hermitian diagonal taken real.
template <class T>
__global__ void k_sym_fill(int n, const T* A, long lda, int lower, int herm, T* O, long ldo) {
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    const bool stored = lower ? i >= j : i <= j;
    double re, im;
    if (stored) ldv<T>(A, (size_t)i + (size_t)j * lda, re, im);
    else {
      ldv<T>(A, (size_t)j + (size_t)i * lda, re, im);
      if (herm) im = -im;
    }
    if (herm && i == j) im = 0.0;
    stv<T>(O, (size_t)i + (size_t)j * ldo, re, im);
  }
}

template <class T>
__global__ void k_copy2d(int m, int n, const T* S, long lds, T* D, long ldd) {
  const size_t total = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    D[(size_t)i + (size_t)j * ldd] = S[(size_t)i + (size_t)j * lds];
  }
}

static int esize(int dt) {
  switch (dt) {
    case XKB_S: return 4;
    case XKB_D: return 8;
    case XKB_C: return 8;
    case XKB_Z: return 16;
  }
  return 0;
}

static unsigned grid_for(size_t total, int per_block = 256) {
  size_t b = (total + per_block - 1) / per_block;
  const size_t cap = (size_t)sm_count() * 16;
  return (unsigned)std::max<size_t>(1, std::min(b, cap));
}

template <class T>
static int launch_diag(int n, int nrhs, const void* A, long lda, int swap, int conj, int lower,
                       int unit, void* B, long ldb, int rhs_rows, const double* al,
                       cudaStream_t st) {
  using S = typename St<T>::S;
  constexpr int cpp = kLeafThreads / LeafShape<T, kLeafRplReal>::G;  // right-hand sides per pass
  // about two CTAs per SM; each stages the block once for all its passes
  const long want = 2L * sm_count();
  long per = ((long)nrhs + want - 1) / want;
  per = std::max<long>(cpp, (per + cpp - 1) / cpp * cpp);
  const unsigned grid = (unsigned)std::max<long>(1, ((long)nrhs + per - 1) / per);
  const size_t smem = LeafShape<T, kLeafRplReal>::SMEM;
  auto kl = lower ? k_trsm_leaf<T, true> : k_trsm_leaf<T, false>;
  static bool attr[2] = {false, false};
  if (!attr[lower ? 1 : 0]) {
    if (cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return XKB_ECUDA;
    attr[lower ? 1 : 0] = true;
  }
  kl<<<grid, kLeafThreads, smem, st>>>(n, nrhs, (int)per, static_cast<const S*>(A), lda, swap,
                                       conj, unit, static_cast<S*>(B), ldb, rhs_rows, al[0],
                                       al[1]);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static int diag_dispatch(int dt, int n, int nrhs, const void* A, long lda, int swap, int conj,
                         int lower, int unit, void* B, long ldb, int rhs_rows, const double* al,
                         cudaStream_t st) {
  switch (dt) {
    case XKB_S: return launch_diag<float>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_D: return launch_diag<double>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_C: return launch_diag<float2>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_Z: return launch_diag<double2>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
  }
  return XKB_EINVAL;
}

struct TrsmCtx {
  int dt, es, left, trans, unit, fwd, ozaki;
  const char* A;
  long lda;
  char* B;
  long ldb;
  int nrhs;
  cudaStream_t st;
  int swap, conj, lower_eff;
};

static const char* aptr(const TrsmCtx& c, long r, long col) {
  return c.A + (r + col * c.lda) * (long)c.es;
}

// GEMM with op(A)[P, Q] as one operand.  op(A)[P,Q] = A[P,Q] (trans N) or
// op(A[Q,P]).
static int update(const TrsmCtx& c, long p0, long p1, long q0, long q1, const double* alpha) {
  xkb_gemm_args g{};
  g.dtype = c.dt;
  const double m1[2] = {-1.0, 0.0};
  g.alpha[0] = m1[0];
  g.alpha[1] = m1[1];
  g.beta[0] = alpha[0];
  g.beta[1] = alpha[1];
  g.uplo = XKB_FULL;
  const long P = p1 - p0, Q = q1 - q0;
  const bool tn = c.trans == XKB_OP_N;
  if (c.left) {
    // B[P,:] = alpha B[P,:] - op(A)[P,Q] X[Q,:]
    g.M = (int)P;
    g.N = c.nrhs;
    g.K = (int)Q;
    g.opA = tn ? XKB_OP_N : c.trans;
    g.A = tn ? aptr(c, p0, q0) : aptr(c, q0, p0);
    g.lda = c.lda;
    g.opB = XKB_OP_N;
    g.B = c.B + q0 * (long)c.es;
    g.ldb = c.ldb;
    g.C = c.B + p0 * (long)c.es;
    g.ldc = c.ldb;
  } else {
    // B[:,P] = alpha B[:,P] - X[:,Q] op(A)[Q,P]
    g.M = c.nrhs;
    g.N = (int)P;
    g.K = (int)Q;
    g.opA = XKB_OP_N;
    g.A = c.B + q0 * c.ldb * (long)c.es;
    g.lda = c.ldb;
    g.opB = tn ? XKB_OP_N : c.trans;
    g.B = tn ? aptr(c, q0, p0) : aptr(c, p0, q0);
    g.ldb = c.lda;
    g.C = c.B + p0 * c.ldb * (long)c.es;
    g.ldc = c.ldb;
  }
  if (c.ozaki > 0 && std::min<long>(std::min<long>(g.M, g.N), g.K) >= c.ozaki) {
    int e = xkb_cuda_ozaki_gemm(&g, 0, c.st);
    if (e != XKB_ERANGE) return e;
  }
  return xkb_cuda_gemm(&g, c.st);
}

static int solve(const TrsmCtx& c, long i0, long i1, const double* alpha) {
  const long n = i1 - i0;
  if (n <= kLeaf) {
    // leaf: diagonal block of the effective triangle
    const char* Ad = aptr(c, i0, i0);
    char* Bd = c.left ? c.B + i0 * (long)c.es : c.B + i0 * c.ldb * (long)c.es;
    return diag_dispatch(c.dt, (int)n, c.nrhs, Ad, c.lda, c.swap, c.conj, c.lower_eff, c.unit, Bd,
                         c.ldb, c.left ? 0 : 1, alpha, c.st);
  }
  long h = i0 + ((n / 2 + kLeaf - 1) / kLeaf) * kLeaf;
  if (h >= i1) h = i1 - kLeaf;
  const double one[2] = {1.0, 0.0};
  int e;
  if (c.fwd) {
    if ((e = solve(c, i0, h, alpha))) return e;
    if ((e = update(c, h, i1, i0, h, alpha))) return e;
    return solve(c, h, i1, one);
  }
  if ((e = solve(c, h, i1, alpha))) return e;
  if ((e = update(c, i0, h, h, i1, alpha))) return e;
  return solve(c, i0, h, one);
}

}  // namespace xkb

using namespace xkb;

extern "C" int xkb_cuda_trsm(int dtype, int side, int uplo, int trans, int diag, int M, int N,
                             const double* alpha, const void* A, long lda, void* B, long ldb,
                             int ozaki, void* stream) {
  if (dtype < XKB_S || dtype > XKB_Z || M < 0 || N < 0 || !alpha) return XKB_EINVAL;
  if (trans < XKB_OP_N || trans > XKB_OP_C) return XKB_EINVAL;
  if (M == 0 || N == 0) return XKB_OK;
  const bool cplx = dtype == XKB_C || dtype == XKB_Z;
  TrsmCtx c;
  c.dt = dtype;
  c.es = esize(dtype);
  c.left = side == 0;
  c.trans = (!cplx && trans == XKB_OP_C) ? XKB_OP_T : trans;
  c.unit = diag != 0;
  c.ozaki = (dtype == XKB_D || dtype == XKB_Z) ? ozaki : 0;
  c.A = static_cast<const char*>(A);
  c.lda = lda;
  c.B = static_cast<char*>(B);
  c.ldb = ldb;
  c.nrhs = c.left ? N : M;
  c.st = resolve_stream(stream);
  const bool lower = uplo == XKB_LOWER;
  const bool op_lower = lower ^ (c.trans != XKB_OP_N);  // op(A) lower?
  // effective triangle element access, as in k_trsm_leaf
  if (c.left) {
    c.swap = c.trans != XKB_OP_N;
    c.conj = c.trans == XKB_OP_C;
    c.lower_eff = op_lower;
  } else {
    c.swap = c.trans == XKB_OP_N;
    c.conj = c.trans == XKB_OP_C;
    c.lower_eff = !op_lower;
  }
  c.fwd = c.lower_eff;
  const long n = c.left ? M : N;
  return solve(c, 0, n, alpha);
}

extern "C" int xkb_cuda_trmm(int dtype, int side, int uplo, int trans, int diag, int M, int N,
                             const double* alpha, const void* A, long lda, void* B, long ldb,
                             void* stream) {
  if (dtype < XKB_S || dtype > XKB_Z || M < 0 || N < 0 || !alpha) return XKB_EINVAL;
  if (M == 0 || N == 0) return XKB_OK;
  cudaStream_t st = resolve_stream(stream);
  const int es = esize(dtype);
  const long na = side == 0 ? M : N;
  const long ldt = (na + 31) / 32 * 32, ldc = ((long)M + 31) / 32 * 32;
  void *T = nullptr, *Bc = nullptr;
  if (cudaMallocAsync(&T, (size_t)ldt * na * es, st) != cudaSuccess) return XKB_ENOMEM;
  if (cudaMallocAsync(&Bc, (size_t)ldc * N * es, st) != cudaSuccess) {
    cudaFreeAsync(T, st);
    return XKB_ENOMEM;
  }
  const unsigned g1 = grid_for((size_t)na * na), g2 = grid_for((size_t)M * N);
  const int lower = uplo == XKB_LOWER, unit = diag != 0;
  switch (dtype) {
    case XKB_S:
      k_tri_fill<float><<<g1, 256, 0, st>>>((int)na, (const float*)A, lda, lower, unit, (float*)T, ldt);
      k_copy2d<float><<<g2, 256, 0, st>>>(M, N, (const float*)B, ldb, (float*)Bc, ldc);
      break;
    case XKB_D:
      k_tri_fill<double><<<g1, 256, 0, st>>>((int)na, (const double*)A, lda, lower, unit, (double*)T, ldt);
      k_copy2d<double><<<g2, 256, 0, st>>>(M, N, (const double*)B, ldb, (double*)Bc, ldc);
      break;
    case XKB_C:
      k_tri_fill<float2><<<g1, 256, 0, st>>>((int)na, (const float2*)A, lda, lower, unit, (float2*)T, ldt);
      k_copy2d<float2><<<g2, 256, 0, st>>>(M, N, (const float2*)B, ldb, (float2*)Bc, ldc);
      break;
    case XKB_Z:
      k_tri_fill<double2><<<g1, 256, 0, st>>>((int)na, (const double2*)A, lda, lower, unit, (double2*)T, ldt);
      k_copy2d<double2><<<g2, 256, 0, st>>>(M, N, (const double2*)B, ldb, (double2*)Bc, ldc);
      break;
  }
  count_launch(2);
  xkb_gemm_args g{};
  g.dtype = dtype;
  g.M = M;
  g.N = N;
  g.K = (int)na;
  g.alpha[0] = alpha[0];
  g.alpha[1] = alpha[1];
  g.beta[0] = g.beta[1] = 0.0;
  g.uplo = XKB_FULL;
  if (side == 0) {  // B = alpha op(T) Bc
    g.opA = trans;
    g.A = T;
    g.lda = ldt;
    g.opB = XKB_OP_N;
    g.B = Bc;
    g.ldb = ldc;
  } else {          // B = alpha Bc op(T)
    g.opA = XKB_OP_N;
    g.A = Bc;
    g.lda = ldc;
    g.opB = trans;
    g.B = T;
    g.ldb = ldt;
  }
  g.C = B;
  g.ldc = ldb;
  int e = xkb_cuda_gemm(&g, st);
  cudaFreeAsync(T, st);
  cudaFreeAsync(Bc, st);
  return e;
}

extern "C" int xkb_cuda_symm(int dtype, int herm, int side, int uplo, int M, int N,
                             const double* alpha, const void* A, long lda, const void* B,
                             long ldb, const double* beta, void* C, long ldc, void* stream) {
  if (dtype < XKB_S || dtype > XKB_Z || M < 0 || N < 0 || !alpha || !beta) return XKB_EINVAL;
  if (M == 0 || N == 0) return XKB_OK;
  cudaStream_t st = resolve_stream(stream);
  const int es = esize(dtype);
  const long na = side == 0 ? M : N;
  const long ldt = (na + 31) / 32 * 32;
  void* S = nullptr;
  if (cudaMallocAsync(&S, (size_t)ldt * na * es, st) != cudaSuccess) return XKB_ENOMEM;
  const unsigned g1 = grid_for((size_t)na * na);
  const int lower = uplo == XKB_LOWER;
  const int hm = herm && (dtype == XKB_C || dtype == XKB_Z);
  switch (dtype) {
    case XKB_S: k_sym_fill<float><<<g1, 256, 0, st>>>((int)na, (const float*)A, lda, lower, 0, (float*)S, ldt); break;
    case XKB_D: k_sym_fill<double><<<g1, 256, 0, st>>>((int)na, (const double*)A, lda, lower, 0, (double*)S, ldt); break;
    case XKB_C: k_sym_fill<float2><<<g1, 256, 0, st>>>((int)na, (const float2*)A, lda, lower, hm, (float2*)S, ldt); break;
    case XKB_Z: k_sym_fill<double2><<<g1, 256, 0, st>>>((int)na, (const double2*)A, lda, lower, hm, (double2*)S, ldt); break;
  }
  count_launch();
  xkb_gemm_args g{};
  g.dtype = dtype;
  g.M = M;
  g.N = N;
  g.K = (int)na;
  g.alpha[0] = alpha[0];
  g.alpha[1] = alpha[1];
  g.beta[0] = beta[0];
  g.beta[1] = beta[1];
  g.uplo = XKB_FULL;
  g.opA = XKB_OP_N;
  g.opB = XKB_OP_N;
  if (side == 0) {
    g.A = S;
    g.lda = ldt;
    g.B = B;
    g.ldb = ldb;
  } else {
    g.A = B;
    g.lda = ldb;
    g.B = S;
    g.ldb = ldt;
  }
  g.C = C;
  g.ldc = ldc;
  int e = xkb_cuda_gemm(&g, st);
  cudaFreeAsync(S, st);
  return e;
}
