// potrf.cu -- Cholesky factorization on the device: A = L L^H (lower) or
// A = U^H U (upper), in place, for s/d/c/z.
//
// Replaces the reference's tile Cholesky driver (blas/zpotrf.c:46-220:
// diagonal zpotrf tasks, trsm right/lower/conj-trans of the panel, herk and
// gemm of the trailing tiles) and its diagonal-tile body (cuSOLVER potrf in
// ztask_potrf.c).  Here the factorization is recursive on the matrix index
// (split points multiple of 64): factor the leading block, solve the panel
// against it with xkb_cuda_trsm (block solves + DMMA GEMMs), update the
// trailing block with one triangle-masked GEMM (the HERK/SYRK of the
// reference: C = C - P P^H, only the stored triangle written), factor the
// trailing block.  Blocks of <= 128 columns (64 complex) are factored in
// FP64 by one CTA of k_potrf_block (the block in shared memory, 8-column
// steps with DMMA panel solves and updates).
// A non-positive (or non-finite) pivot stops nothing on the device -- later
// blocks become NaN as in LAPACK's unchecked use -- but the first failing
// column (1-based, over the whole matrix) is recorded in *d_info (0 = none).
#include <algorithm>
#include <type_traits>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {

// Diagonal blocks of up to NMAX (128 real, 64 complex) columns are factored
// by one CTA with the block in shared memory (FP64), 8 columns per step:
//   1. warp 0 factors the 8 x 8 diagonal block in registers: lane
//      (r, k) = (lane >> 3, lane & 7) holds entries (r, k) and (r + 4, k);
//      per column j the pivot and the column come by shuffles, then the
//      reciprocal square root, the scaling and the rank-1 update of the
//      entries right of j;
//   2. the panel below, L(i, s) = A(i, s) L_ss^-H, by substitution, one
//      thread per row (8 dependent steps, products with the reciprocal
//      pivots);
//   3. the rank-8 update of the trailing lower triangle,
//      A(i, j) -= L(i, s) L(j, s)^H, with DMMA 16 x 8 tiles that meet the
//      triangle, two tiles per warp in flight; warp 0 updates the tile
//      holding the next diagonal block and factors that block while warps
//      1..7 update the rest (look-ahead).
// Same operations as the blocked right-looking Cholesky.  The loops over
// columns are not unrolled: the kernel runs once per launch on an SM whose
// instruction cache is cold, and a fully unrolled 8 x 8 factor paid about
// 19k cycles of instruction fetch on its first pass (clock64 stamps: 22.5k
// cycles cold, 3.75k warm).
constexpr int kPoThreads = 256;

template <class T>
struct PoShape {
  static constexpr bool CP = St<T>::CPLX;
  static constexpr int NMAX = CP ? 64 : 128;
  static constexpr int ROWS = NMAX + 16;  // rows incl. the last partial 16-row tile
  static constexpr int COLS = NMAX + 8;   // columns incl. the last partial 8-column tile
  static constexpr int LD = ROWS + 2;     // column stride, = 2 mod 16
  static constexpr int PL = CP ? 2 : 1;
  static constexpr size_t SMEM = sizeof(double) * ((size_t)PL * COLS * LD + PL * 64 * 2);
};

template <class T>
__global__ void __launch_bounds__(kPoThreads, 1)
    k_potrf_block(int n, typename St<T>::S* A, long lda, int upper, int col0, int* info) {
  using Sh = PoShape<T>;
  using S = typename St<T>::S;
  constexpr bool CP = Sh::CP;
  constexpr int LD = Sh::LD;
  constexpr int W = CP ? 2 : 1;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ double sm_po[];
  double* Xr = sm_po;  // L(i, k) at X[k * LD + i], lower part only
  double* Xi = Xr + (CP ? Sh::COLS * LD : 0);
  double* Lsr = sm_po + (size_t)Sh::PL * Sh::COLS * LD;  // 8 x 8 factor, [i][k]
  double* Lsi = Lsr + 64;
  double* Rv = Lsr + Sh::PL * 64;  // reciprocals of its diagonal
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;

  // ---- load the effective lower triangle (upper: L = U^H) ----
  // Real lower blocks with 16-byte aligned columns: every 16-byte piece of
  // the lower triangle's columns is copied by cp.async at once (one memory
  // latency for the whole block); the rows and columns past n are zeroed.
  // Pieces that straddle the diagonal also bring the element above it,
  // which nothing reads (every tile update stores only its lower part).
  // Other blocks: loads in groups of 8 per thread before their stores.
  bool fast = false;
  if constexpr (!CP && std::is_same<S, double>::value) {
    fast = !upper && (n % 2) == 0 && (lda % 2) == 0 &&
           (reinterpret_cast<uintptr_t>(A) % 16) == 0;
  }
  if constexpr (!CP && std::is_same<S, double>::value) if (fast) {
    for (int k = warp; k < n; k += kPoThreads / 32)
      for (int i = (k & ~1) + 2 * lane; i < n; i += 64)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(Xr + k * LD + i)),
                     "l"(A + (size_t)i + (size_t)k * lda)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int k = warp; k < Sh::COLS; k += kPoThreads / 32)
      for (int i = (k < n ? n : 0) + lane; i < LD; i += 32) Xr[k * LD + i] = 0.0;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
  }
  constexpr int GRP = 8;
  for (int e0 = 0; !fast && e0 < Sh::COLS * LD; e0 += kPoThreads * GRP) {
    double vr[GRP], vi[GRP];
#pragma unroll
    for (int q = 0; q < GRP; ++q) {
      const int e = e0 + q * kPoThreads + tid;
      const int k = e / LD, i = e % LD;
      vr[q] = vi[q] = 0.0;
      if (i < n && k < n && i >= k) {
        const size_t idx = upper ? (size_t)k + (size_t)i * lda : (size_t)i + (size_t)k * lda;
        vr[q] = (double)A[W * idx];
        if (CP) vi[q] = (i == k) ? 0.0 : (upper ? -(double)A[2 * idx + 1] : (double)A[2 * idx + 1]);
      }
    }
#pragma unroll
    for (int q = 0; q < GRP; ++q) {
      const int e = e0 + q * kPoThreads + tid;
      if (e < Sh::COLS * LD) {
        Xr[e] = vr[q];
        if (CP) Xi[e] = vi[q];
      }
    }
  }

  // warp 0: factor the 8 x 8 diagonal block at b (final values in X, the
  // strictly lower part of the factor in Ls, the reciprocals of its diagonal
  // in Rv).  Every lane holds the whole triangle and computes the same
  // factor, so the chain per column is the reciprocal square root, one
  // product and one update (no shuffles); lane 0 stores.  Rows past the block
  // (w < 8) are identity rows.
  auto diag_factor = [&](int b) {
    const int w = min(8, n - b);
    double ar[8][8], ai[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int k = 0; k <= i; ++k) {
        ar[i][k] = i < w ? Xr[(b + k) * LD + b + i] : (k == i ? 1.0 : 0.0);
        ai[i][k] = (CP && i < w && k < i) ? Xi[(b + k) * LD + b + i] : 0.0;
      }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double d = ar[j][j];
      if (!(d > 0.0) && lane == 0 && j < w && info) atomicCAS(info, 0, col0 + b + j + 1);
      const double rj = rsqrt(d);
      ar[j][j] = d * rj;
      if (lane == 0) Rv[j] = rj;
#pragma unroll
      for (int i = j + 1; i < 8; ++i) {
        ar[i][j] *= rj;
        if (CP) ai[i][j] *= rj;
      }
#pragma unroll
      for (int k = j + 1; k < 8; ++k)
#pragma unroll
        for (int i = k; i < 8; ++i) {  // A(i, k) -= L(i, j) conj(L(k, j))
          ar[i][k] -= ar[i][j] * ar[k][j] + (CP ? ai[i][j] * ai[k][j] : 0.0);
          if (CP) ai[i][k] -= ai[i][j] * ar[k][j] - ar[i][j] * ai[k][j];
        }
    }
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int k = 0; k <= i; ++k) {
          if (k < i) {
            Lsr[i * 8 + k] = ar[i][k];
            if (CP) Lsi[i * 8 + k] = ai[i][k];
          }
          if (i < w) {
            Xr[(b + k) * LD + b + i] = ar[i][k];
            if (CP) Xi[(b + k) * LD + b + i] = k < i ? ai[i][k] : 0.0;
          }
        }
    }
  };

  __syncthreads();
  // step -1 factors block 0; step s >= 0 solves panel s, updates the trailing
  // triangle and factors block s + 1 (one call site of the unrolled factor:
  // its code is fetched once)
  const int nsteps = (n + 7) / 8;
  for (int s = -1; s < nsteps; ++s) {
    const int b = 8 * s;
    const int r0 = b + 8, R = n - r0;
    if (R <= 0) break;
    if (s >= 0) {
    // 1. panel: L(i, s) = A(i, s) L_ss^-H, in place, one thread per row:
    //    x_j = (a_j - sum_{m<j} x_m conj(L(j, m))) / L(j, j)
    for (int i = r0 + tid; i < n; i += kPoThreads) {
      double xr[8], xi[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        xr[j] = Xr[(b + j) * LD + i];
        xi[j] = CP ? Xi[(b + j) * LD + i] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double rj = Rv[j];
        xr[j] *= rj;
        if (CP) xi[j] *= rj;
#pragma unroll
        for (int q = j + 1; q < 8; ++q) {
          const double lr = Lsr[q * 8 + j], li = CP ? Lsi[q * 8 + j] : 0.0;
          xr[q] -= xr[j] * lr + xi[j] * li;
          if (CP) xi[q] -= xi[j] * lr - xr[j] * li;
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        Xr[(b + j) * LD + i] = xr[j];
        if (CP) Xi[(b + j) * LD + i] = xi[j];
      }
    }
    __syncthreads();
    }
    // 2. trailing update of the lower triangle: A(i, j) -= L(i, s) L(j, s)^H
    //    over the 16 x 8 tiles (ti, tj) that meet it (tj < min(nt, 2 ti + 2)),
    //    numbered row by row.  Tile 0 holds the next diagonal block: warp 0
    //    updates it and factors that block while warps 1..7 take tiles
    //    warp, warp + 7, ... (look-ahead).
    const int mt = (R + 15) / 16, nt = (R + 7) / 8;
    const int k0 = 2 * t, k1 = k0 + 1;
    auto advance = [&](int& ti, int& tj, int step) {
      tj += step;
      while (ti < mt) {
        const int cnt = min(nt, 2 * ti + 2);
        if (tj < cnt) break;
        tj -= cnt;
        ++ti;
      }
    };
    struct Frag {
      double ar[4], ai[4], br[2], bi[2], cr[4], ci[4];
      int m0, n0;
    };
    auto frag_load = [&](Frag& f, int ti, int tj) {
      f.m0 = r0 + 16 * ti;
      f.n0 = r0 + 8 * tj;
      const int m0 = f.m0, n0 = f.n0;
      f.ar[0] = -Xr[(b + k0) * LD + m0 + g];
      f.ar[1] = -Xr[(b + k0) * LD + m0 + g + 8];
      f.ar[2] = -Xr[(b + k1) * LD + m0 + g];
      f.ar[3] = -Xr[(b + k1) * LD + m0 + g + 8];
      // B (k, c) = conj(L(n0 + c, b + k))
      f.br[0] = Xr[(b + k0) * LD + n0 + g];
      f.br[1] = Xr[(b + k1) * LD + n0 + g];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = m0 + g + ((v >> 1) << 3), col = n0 + 2 * t + (v & 1);
        f.cr[v] = Xr[col * LD + row];
        f.ci[v] = CP ? Xi[col * LD + row] : 0.0;
      }
      if constexpr (CP) {
        f.ai[0] = -Xi[(b + k0) * LD + m0 + g];
        f.ai[1] = -Xi[(b + k0) * LD + m0 + g + 8];
        f.ai[2] = -Xi[(b + k1) * LD + m0 + g];
        f.ai[3] = -Xi[(b + k1) * LD + m0 + g + 8];
        f.bi[0] = -Xi[(b + k0) * LD + n0 + g];
        f.bi[1] = -Xi[(b + k1) * LD + n0 + g];
      }
    };
    auto frag_mma = [&](Frag& f) {
      if constexpr (CP) {
        // C += (-L_i)(conj L_j)
        const double a_ni[4] = {-f.ai[0], -f.ai[1], -f.ai[2], -f.ai[3]};
        dmma_k8(f.cr, f.ar, f.br);
        dmma_k8(f.cr, a_ni, f.bi);
        dmma_k8(f.ci, f.ar, f.bi);
        dmma_k8(f.ci, f.ai, f.br);
      } else {
        dmma_k8(f.cr, f.ar, f.br);
      }
    };
    auto frag_store = [&](const Frag& f) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = f.m0 + g + ((v >> 1) << 3), col = f.n0 + 2 * t + (v & 1);
        if (row >= col) {  // lower part only (the diagonal's imaginary part is dropped at the end)
          Xr[col * LD + row] = f.cr[v];
          if (CP) Xi[col * LD + row] = f.ci[v];
        }
      }
    };
    if (warp == 0) {
      if (s >= 0) {
        Frag f;
        frag_load(f, 0, 0);
        frag_mma(f);
        frag_store(f);
        __syncwarp();
      }
      diag_factor(r0);  // block s + 1 (final after tile 0)
    } else if (s >= 0) {
      int ti = 0, tj = 0;
      advance(ti, tj, warp);
      while (ti < mt) {
        int ti2 = ti, tj2 = tj;
        advance(ti2, tj2, kPoThreads / 32 - 1);
        const bool two = ti2 < mt;  // warp-uniform
        Frag f0, f1;
        frag_load(f0, ti, tj);
        if (two) frag_load(f1, ti2, tj2);
        frag_mma(f0);
        if (two) frag_mma(f1);
        frag_store(f0);
        if (two) frag_store(f1);
        ti = ti2;
        tj = tj2;
        if (two) advance(ti, tj, kPoThreads / 32 - 1);
      }
    }
    __syncthreads();
  }

  // ---- store the factor (the stored triangle only), column by column ----
  for (int k = warp; k < n; k += kPoThreads / 32)
    for (int i = k + lane; i < n; i += 32) {
      const size_t idx = upper ? (size_t)k + (size_t)i * lda : (size_t)i + (size_t)k * lda;
      A[W * idx] = static_cast<S>(Xr[k * LD + i]);
      if (CP) A[2 * idx + 1] = static_cast<S>(i == k ? 0.0 : (upper ? -Xi[k * LD + i] : Xi[k * LD + i]));
    }
}

struct PotrfCtx {
  int dt, es, upper;
  int ozaki;  // > 0: updates whose dimensions are all >= ozaki use the Ozaki form
  char* A;
  long lda;
  int* info;
  cudaStream_t st;
  // hybrid form: the recursion hands sub-problems of at most blk_leaf rows to
  // the blocked look-ahead form (widest block blk_nb); 0: recursion only
  long blk_leaf = 0, blk_nb = 0;
};

static int factor_blocked(const PotrfCtx& c, long i0, long i1, long nb);

template <class T>
static int launch_leaf(const PotrfCtx& c, char* Ad, long n, long i0) {
  using Sh = PoShape<T>;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_potrf_block<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Sh::SMEM) != cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  const long long tv = evlog_kern_begin(c.st, "k_potrf_block");
  k_potrf_block<T><<<1, kPoThreads, Sh::SMEM, c.st>>>(
      (int)n, reinterpret_cast<typename St<T>::S*>(Ad), c.lda, c.upper, (int)i0, c.info);
  evlog_kern_end(tv, c.st);
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

// Trailing update C -= op(P) op(P)^H on `st`: Ozaki in tensor-op mode above
// the crossover, else the DMMA kernel.
static int update(const PotrfCtx& c, xkb_gemm_args g, cudaStream_t st) {
  if (c.ozaki > 0 && std::min<long>(g.K, std::min(g.M, g.N)) >= c.ozaki) {
    const int e = xkb_cuda_ozaki_gemm(&g, 0, st);
    if (e != XKB_ERANGE) return e;
  }
  return xkb_cuda_gemm(&g, st);
}

static long split_point(long i0, long i1) {
  constexpr long kSplit = 64;
  const long n = i1 - i0;
  long h = i0 + ((n / 2 + kSplit - 1) / kSplit) * kSplit;
  if (h >= i1) h = i1 - kSplit;
  return h;
}

// Recursive Cholesky of rows / columns [i0, i1).  Look-ahead (la): the
// trailing update is split at the next level's split point; the part the
// next level factors first (its leading column block, lower; row block,
// upper) is updated on the caller's stream, the rest of the trailing
// triangle on a side stream, so that the next level's leading factorization
// and panel solve overlap that larger update.  pend: the caller forked such
// an update over this call's trailing triangle; it is joined before this
// call's own update.  Left subtrees run without look-ahead, so that they do
// not queue behind the side stream's update.
static int factor(const PotrfCtx& c, long i0, long i1, bool la, bool pend) {
  const long n = i1 - i0;
  const bool cplx = c.dt == XKB_C || c.dt == XKB_Z;
  const long nmax = cplx ? PoShape<double2>::NMAX : PoShape<double>::NMAX;
  if (n <= nmax) return leaf(c, i0, n);  // never pending: callers fork only above nmax
  if (c.blk_leaf > 0 && n <= c.blk_leaf && n > 2 * nmax) {
    // hybrid: this sub-problem in the blocked form, after the caller's
    // pending update of it
    const SideStream& ss0 = side_stream(0);
    if (pend && !side_join(ss0, ss0.s, c.st)) return XKB_ECUDA;
    PotrfCtx cb = c;
    cb.blk_leaf = 0;
    return factor_blocked(cb, i0, i1, c.blk_nb);
  }
  const long h = split_point(i0, i1);
  const long n1 = h - i0, n2 = i1 - h;
  int e;
  if ((e = factor(c, i0, h, false, false))) return e;
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
                           c.lda, c.ozaki, c.st)))
      return e;
    g.opA = XKB_OP_N;
    g.opB = ctr;
    g.uplo = XKB_LOWER;
  } else {
    // A12 = U11^-H A12; A22 -= A12^H A12 (upper triangle)
    P = c.A + (i0 + h * c.lda) * (long)c.es;
    if ((e = xkb_cuda_trsm(c.dt, 0, XKB_UPPER, ctr, 0, (int)n1, (int)n2, one, A11, c.lda, P,
                           c.lda, c.ozaki, c.st)))
      return e;
    g.opA = ctr;
    g.opB = XKB_OP_N;
    g.uplo = XKB_UPPER;
  }
  g.A = P;
  g.lda = c.lda;
  g.B = P;
  g.ldb = c.lda;
  const SideStream& ss = side_stream(0);
  if (pend && !side_join(ss, ss.s, c.st)) return XKB_ECUDA;
  if (!la || n2 <= nmax || !ss.s) {
    if ((e = update(c, g, c.st))) return e;
    return factor(c, h, i1, la, false);
  }
  // part 1: the next level's leading block of columns (rows) [0, m1) of A22
  const long m1 = split_point(h, i1) - h;
  xkb_gemm_args g1 = g, g2 = g;
  if (!c.upper) {
    g1.N = (int)m1;  // rows [0, n2) x cols [0, m1), lower mask
  } else {
    g1.M = (int)m1;  // rows [0, m1) x cols [0, n2), upper mask
  }
  // part 2: the trailing triangle [m1, n2)^2
  const long off = m1 * (c.upper ? c.lda : 1) * (long)c.es;  // panel rows (lower) / cols (upper)
  g2.M = g2.N = (int)(n2 - m1);
  g2.A = static_cast<const char*>(g.A) + off;
  g2.B = static_cast<const char*>(g.B) + off;
  g2.C = A22 + (m1 + m1 * c.lda) * (long)c.es;
  if ((e = update(c, g1, c.st))) return e;
  cudaStream_t s2 = side_fork(ss, c.st);
  if ((e = update(c, g2, s2))) return e;
  return factor(c, h, i1, la, s2 != c.st);
}

// Blocked right-looking Cholesky of rows / columns [i0, i1) with look-ahead,
// in blocks of nb columns (a multiple of 64); lower storage described (upper
// is its conjugate transpose).  Step k, with diagonal block D_k factored and
// the panel below it split into P1 (the next block's nb rows) and P2 (the
// rest):
//   critical path (high-priority stream hp):  P1 = P1 D_k^-H, then
//     D_{k+1} -= P1 P1^H, then factor D_{k+1}, then the next step's P1;
//   beside it (high-priority stream hp2):     P2 = P2 D_k^-H, then the rest
//     of block column k+1, B -= P2 P1^H (the next step's panel);
//   trailing triangle (caller's stream):      T -= P2 P2^H, one
//     triangle-masked GEMM.
// The tile-level critical path of the reference's tile loop
// (blas/zpotrf.c:46-220, potrf -> trsm -> syrk -> potrf per tile column),
// with nb-wide tiles; the large updates run while the next diagonal block
// is factored.  Dependencies between the streams are events: D_{k+1}'s
// update and block column k+1's update wait for the previous trailing
// update (it wrote both); the next P1 solve waits for block column k+1.
// The block width shrinks as the factorization proceeds: while the trailing
// triangle is large its update bounds each step and wider blocks make that
// GEMM more efficient (larger K); near the end the critical path bounds each
// step and narrower blocks shorten it.  Width for `m` remaining rows: nb,
// halved (rounded down to a multiple of 64, at least nmin) while
// m <= shrink * width (tuning keys potrf_shrink, default 8, and in tensor-op
// mode potrf_shrink_oz, default 12; DPOTRF 8192 plain, shrink 8 / 12 / 16 /
// 24: 9.88 / 10.05 / 10.88 / 11.69 ms).
static long block_width(long m, long nb, long nmin, bool oz) {
  const double shrink = oz ? tune("potrf_shrink_oz", 12.0) : tune("potrf_shrink", 8.0);
  long w = nb;
  while (w > nmin && (double)m <= shrink * (double)w) w = std::max(nmin, (w / 2) / 64 * 64);
  return w;
}

static int factor_blocked(const PotrfCtx& c, long i0, long i1, long nb) {
  const SideStream& hp = side_stream(kHiStream);
  const SideStream& hp2 = side_stream(kHiStream2);
  cudaEvent_t* ev = dep_events();
  if (!hp.s || !hp2.s || !ev) return factor(c, i0, i1, true, false);
  cudaEvent_t e_diag = ev[0], e_p1 = ev[1], e_p2 = ev[2], e_col = ev[3], e_trail = ev[4];
  const bool cplx = c.dt == XKB_C || c.dt == XKB_Z;
  const int ctr = cplx ? XKB_OP_C : XKB_OP_T;
  const double one[2] = {1.0, 0.0};
  const long es = c.es, lda = c.lda;
  auto at = [&](long i, long j) { return c.A + (i + j * lda) * es; };
  // (rows r, cols q) of the lower-storage picture, mapped to the storage
  auto blk = [&](long r, long q) { return c.upper ? at(q, r) : at(r, q); };
  // solve rows [r, r + m) of the panel under block [b, b + nk)
  auto solve = [&](long b, long nk, long r, long m, cudaStream_t st) {
    return c.upper ? trsm_entry(c.dt, 0, XKB_UPPER, ctr, 0, (int)nk, (int)m, one, at(b, b), lda,
                                blk(r, b), lda, 0, st, false)
                   : trsm_entry(c.dt, 1, XKB_LOWER, ctr, 0, (int)m, (int)nk, one, at(b, b), lda,
                                blk(r, b), lda, 0, st, false);
  };
  // C(rows [r, r + m), cols [q, q + w)) -= P(rows r..) P(rows q..)^H over the
  // panel of block [b, b + nk); masked to the stored triangle when r == q
  auto rank_update = [&](long b, long nk, long r, long m, long q, long w, cudaStream_t st,
                         const PotrfCtx& cx) {
    xkb_gemm_args g{};
    g.dtype = c.dt;
    g.alpha[0] = -1.0;
    g.beta[0] = 1.0;
    g.K = (int)nk;
    g.herm_diag = (cplx && r == q) ? 1 : 0;  // a diagonal block: its diagonal is real
    g.lda = g.ldb = g.ldc = lda;
    if (!c.upper) {  // C = A(r.., q..) -= P_r P_q^H, P_x = A(x.., b..)
      g.opA = XKB_OP_N;
      g.opB = ctr;
      g.M = (int)m;
      g.N = (int)w;
      g.A = at(r, b);
      g.B = at(q, b);
      g.C = at(r, q);
      g.uplo = r == q ? XKB_LOWER : XKB_FULL;
    } else {  // C = A(q.., r..) -= P_q^H P_r, P_x = A(b.., x..)
      g.opA = ctr;
      g.opB = XKB_OP_N;
      g.M = (int)w;
      g.N = (int)m;
      g.A = at(b, q);
      g.B = at(b, r);
      g.C = at(q, r);
      g.uplo = r == q ? XKB_UPPER : XKB_FULL;
    }
    return update(cx, g, st);
  };
  PotrfCtx ch = c;
  ch.st = side_fork(hp, c.st);
  int e = XKB_OK;
  auto rec = [&](cudaEvent_t x, cudaStream_t st) {
    if (!e && cudaEventRecord(x, st) != cudaSuccess) e = XKB_ECUDA;
  };
  auto wait = [&](cudaStream_t st, cudaEvent_t x) {
    if (!e && cudaStreamWaitEvent(st, x, 0) != cudaSuccess) e = XKB_ECUDA;
  };
  rec(e_trail, c.st);  // "previous trailing update": the caller's work so far
  const long nmin = cplx ? PoShape<double2>::NMAX : PoShape<double>::NMAX;
  long b = i0, nk = std::min(block_width(i1 - i0, nb, nmin, c.ozaki > 0), i1 - i0);
  e = factor(ch, b, b + nk, false, false);
  rec(e_diag, ch.st);
  while (!e && b + nk < i1) {
    const long r0 = b + nk, m2 = i1 - r0;
    const long n1 = std::min(block_width(m2, nb, nmin, c.ozaki > 0), m2), m3 = m2 - n1;  // next block; below it
    if (m3 > 0) {  // hp2: P2 solve (needs D_k)
      wait(hp2.s, e_diag);
      if (!e) e = solve(b, nk, r0 + n1, m3, hp2.s);
      rec(e_p2, hp2.s);
    }
    if (!e) e = solve(b, nk, r0, n1, ch.st);  // hp: P1 solve
    rec(e_p1, ch.st);
    if (m3 > 0) {  // hp2: block column k+1 below D_{k+1} (needs P1, previous trailing update)
      wait(hp2.s, e_p1);
      wait(hp2.s, e_trail);
      if (!e) e = rank_update(b, nk, r0 + n1, m3, r0, n1, hp2.s, ch);
      rec(e_col, hp2.s);
    }
    wait(ch.st, e_trail);  // hp: D_{k+1} update (previous trailing update wrote it)
    if (!e) e = rank_update(b, nk, r0, n1, r0, n1, ch.st, ch);
    if (m3 > 0) {  // caller's stream: trailing triangle (needs P2)
      wait(c.st, e_p2);
      if (!e) e = rank_update(b, nk, r0 + n1, m3, r0 + n1, m3, c.st, c);
      rec(e_trail, c.st);
    }
    if (!e) e = factor(ch, r0, r0 + n1, false, false);  // hp: D_{k+1}
    rec(e_diag, ch.st);
    if (m3 > 0) wait(ch.st, e_col);  // the next P1 lies in block column k+1
    b = r0;
    nk = n1;
  }
  if (!side_join(hp2, hp2.s, c.st) && !e) e = XKB_ECUDA;
  if (!side_join(hp, ch.st, c.st) && !e) e = XKB_ECUDA;
  return e;
}

}  // namespace xkb

using namespace xkb;

extern "C" int xkb_cuda_potrf(int dtype, int uplo, int N, void* A, long lda, int* d_info,
                              int ozaki, void* stream) {
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
  c.ozaki = (dtype == XKB_D || dtype == XKB_Z) ? std::max(ozaki, 0) : 0;
  c.st = resolve_stream(stream);
  // Blocked look-ahead form (tuning key potrf_blocked: 0 off, 1 in plain
  // mode, 2 in both modes; 3, the default: in plain mode, and in tensor-op
  // mode the hybrid -- the recursion with Ozaki updates down to
  // potrf_oz_leaf rows (4096), the blocked form below; widest block
  // potrf_nb, in tensor-op mode potrf_nb_oz) or the recursive form.
  // Measured on a B200, tensor-op DPOTRF 8192: hybrid 9.37 ms, blocked
  // 10.14, recursive 12.64; 16384: 35.8, 58.2, 42.2 ms.  In tensor-op mode the blocked
  // form's updates (inner dimension = block width, 512) stay below the Ozaki
  // threshold; measured on a B200 it still beat the recursive form with
  // Ozaki updates at 8192 (10.2 vs 13.3 ms), whose panel solves and leaf
  // chain are exposed.
  const long nmax = (dtype == XKB_C || dtype == XKB_Z) ? PoShape<double2>::NMAX
                                                       : PoShape<double>::NMAX;
  const int mode = (int)tune("potrf_blocked", 3.0);
  const long nb = std::max(nmax, ((long)tune(c.ozaki ? "potrf_nb_oz" : "potrf_nb", 512.0) + 63) /
                                     64 * 64);
  if (N > 2 * nmax && (mode == 2 || ((mode == 1 || mode == 3) && c.ozaki == 0)))
    return factor_blocked(c, 0, N, nb);
  if (mode == 3 && c.ozaki > 0) {
    c.blk_leaf = std::max(2 * nmax + 1, (long)tune("potrf_oz_leaf", 4096.0));
    c.blk_nb = nb;
  }
  return factor(c, 0, N, true, false);
}
