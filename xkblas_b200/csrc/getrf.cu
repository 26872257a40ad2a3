// getrf.cu -- LU factorization without pivoting on the device, A = L U in
// place (L unit lower, U upper), square matrices, s/d/c/z.
//
// Replaces the reference's tile LU without pivoting (blas/zgetrf_nopiv.c:
// 48-101, Chameleon pzgetrf_nopiv: diagonal getrf_nopiv tasks, trsm
// right/upper/notrans/non-unit of the column panel, trsm left/lower/notrans/
// unit of the row panel, gemm of the trailing tiles).  Here the
// factorization is recursive on the matrix index (split points multiple of
// 64): factor the leading block, solve the row panel U12 = L11^-1 A12 and
// the column panel L21 = A21 U11^-1 with xkb_cuda_trsm, update the trailing
// block with one GEMM (A22 -= L21 U12; Ozaki in tensor-op mode when all
// dimensions reach the threshold), factor the trailing block.  Blocks of
// <= 128 columns (64 complex) are factored by one CTA of k_getrf_block.
// A zero pivot stops nothing on the device (later values become Inf/NaN, as
// with LAPACK's unchecked use); the first one (1-based, over the whole
// matrix) is recorded in *d_info (0 = none).
#include <algorithm>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {

// One CTA, the block in shared memory (FP64), 8 columns per step:
//   1. warp 0 factors the 8 x 8 diagonal block in registers (lane l holds
//      row l; per column: pivot by shuffle, reciprocal, multipliers, rank-1
//      update) and inverts both factors (lane c solves for column c);
//   2. all warps solve the column panel L(i, s) = A(i, s) U_ss^-1 and the
//      row panel U(s, j) = L_ss^-1 A(s, j) with FP64 DMMA (K = 8);
//   3. all warps apply the rank-8 update A(i, j) -= L(i, s) U(s, j) to the
//      trailing block; warp 0 first updates the tile holding the next
//      diagonal block and factors it while warps 1..7 update the rest.
// Same operations as the blocked right-looking LU; the 8 x 8 panel solves
// go through the explicit inverses of the 8 x 8 factors.
constexpr int kLuThreads = 256;

template <class T>
struct LuShape {
  static constexpr bool CP = St<T>::CPLX;
  static constexpr int NMAX = CP ? 64 : 128;
  static constexpr int ROWS = NMAX + 16;  // rows incl. the last partial 16-row tile
  static constexpr int COLS = NMAX + 8;   // columns incl. the last partial 8-column tile
  static constexpr int LD = ROWS + 2;     // column stride, = 2 mod 16
  static constexpr int PL = CP ? 2 : 1;
  // X, then the 8 x 8 factors, inv(L_ss), inv(U_ss) (each [i][k], PL planes)
  static constexpr size_t SMEM = sizeof(double) * ((size_t)PL * COLS * LD + 3 * PL * 64);
};

template <class T>
__global__ void __launch_bounds__(kLuThreads, 1)
    k_getrf_block(int n, typename St<T>::S* A, long lda, int col0, int* info) {
  using Sh = LuShape<T>;
  using S = typename St<T>::S;
  constexpr bool CP = Sh::CP;
  constexpr int LD = Sh::LD;
  constexpr int W = CP ? 2 : 1;
  extern __shared__ double sm_lu[];
  double* Xr = sm_lu;  // A(i, k) at X[k * LD + i]
  double* Xi = Xr + (CP ? Sh::COLS * LD : 0);
  double* Fr = sm_lu + (size_t)Sh::PL * Sh::COLS * LD;  // 8 x 8 factors (L below, U on/above)
  double* Fi = Fr + 64;
  double* VLr = Fr + Sh::PL * 64;  // inv(L_ss)
  double* VLi = VLr + 64;
  double* VUr = VLr + Sh::PL * 64;  // inv(U_ss)
  double* VUi = VUr + 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;

  // ---- load the block (zero past n); loads in groups of 8 per thread ----
  constexpr int GRP = 8;
  for (int e0 = 0; e0 < Sh::COLS * LD; e0 += kLuThreads * GRP) {
    double vr[GRP], vi[GRP];
#pragma unroll
    for (int q = 0; q < GRP; ++q) {
      const int e = e0 + q * kLuThreads + tid;
      const int k = e / LD, i = e % LD;
      vr[q] = vi[q] = 0.0;
      if (i < n && k < n) {
        const size_t idx = (size_t)i + (size_t)k * lda;
        vr[q] = (double)A[W * idx];
        if (CP) vi[q] = (double)A[2 * idx + 1];
      }
    }
#pragma unroll
    for (int q = 0; q < GRP; ++q) {
      const int e = e0 + q * kLuThreads + tid;
      if (e < Sh::COLS * LD) {
        Xr[e] = vr[q];
        if (CP) Xi[e] = vi[q];
      }
    }
  }

  // warp 0: factor the 8 x 8 diagonal block at b (final values in X) and
  // invert both factors
  auto diag_factor = [&](int b) {
    const int w = min(8, n - b);
    const int l = lane & 7;  // lanes 8..31 mirror lanes 0..7 (shuffles span the warp)
    double ar[8], ai[8], rr[8], ri[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const bool in = l < w && k < w;
      ar[k] = in ? Xr[(b + k) * LD + b + l] : (k == l ? 1.0 : 0.0);
      ai[k] = (in && CP) ? Xi[(b + k) * LD + b + l] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double dr = __shfl_sync(0xffffffffu, ar[j], j);
      const double di = CP ? __shfl_sync(0xffffffffu, ai[j], j) : 0.0;
      if (dr == 0.0 && di == 0.0 && lane == 0 && j < w && info) atomicCAS(info, 0, col0 + b + j + 1);
      double pr, pi = 0.0;  // 1 / pivot
      if (CP) {
        const double den = dr * dr + di * di;
        pr = dr / den;
        pi = -di / den;
      } else {
        pr = 1.0 / dr;
      }
      rr[j] = pr;
      ri[j] = pi;
      if (l > j) {  // multiplier L(l, j) = A(l, j) / U(j, j)
        const double xr = ar[j] * pr - ai[j] * pi;
        ai[j] = ar[j] * pi + ai[j] * pr;
        ar[j] = xr;
      }
#pragma unroll
      for (int k = j + 1; k < 8; ++k) {
        const double ur = __shfl_sync(0xffffffffu, ar[k], j);  // U(j, k)
        const double ui = CP ? __shfl_sync(0xffffffffu, ai[k], j) : 0.0;
        if (l > j) {  // A(l, k) -= L(l, j) U(j, k)
          ar[k] -= ar[j] * ur - ai[j] * ui;
          if (CP) ai[k] -= ar[j] * ui + ai[j] * ur;
        }
      }
    }
    if (lane < 8) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        Fr[l * 8 + k] = ar[k];
        if (CP) Fi[l * 8 + k] = ai[k];
        if (l < w && k < w) {
          Xr[(b + k) * LD + b + l] = ar[k];
          if (CP) Xi[(b + k) * LD + b + l] = ai[k];
        }
      }
    }
    __syncwarp();
    if (lane < 8) {
      const int c = lane;
      // column c of inv(L_ss) (unit lower), forward
      double zr[8], zi[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        zr[i] = i == c ? 1.0 : 0.0;
        zi[i] = 0.0;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j >= c) {
#pragma unroll
          for (int i = j + 1; i < 8; ++i) {
            const double lr = Fr[i * 8 + j], li = CP ? Fi[i * 8 + j] : 0.0;
            zr[i] -= lr * zr[j] - li * zi[j];
            if (CP) zi[i] -= lr * zi[j] + li * zr[j];
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        VLr[i * 8 + c] = zr[i];
        if (CP) VLi[i * 8 + c] = zi[i];
      }
      // column c of inv(U_ss) (upper), backward
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        zr[i] = i == c ? 1.0 : 0.0;
        zi[i] = 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = 7 - q;
        if (j <= c) {
          const double vr = zr[j] * rr[j] - zi[j] * ri[j];
          const double vi = zr[j] * ri[j] + zi[j] * rr[j];
          zr[j] = vr;
          zi[j] = vi;
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            if (i < j) {
              const double ur = Fr[i * 8 + j], ui = CP ? Fi[i * 8 + j] : 0.0;
              zr[i] -= ur * vr - ui * vi;
              if (CP) zi[i] -= ur * vi + ui * vr;
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        VUr[i * 8 + c] = zr[i];
        if (CP) VUi[i * 8 + c] = zi[i];
      }
    }
  };

  __syncthreads();
  if (warp == 0) diag_factor(0);
  __syncthreads();
  const int nsteps = (n + 7) / 8;
  const int k0 = 2 * t, k1 = k0 + 1;
  for (int s = 0; s < nsteps; ++s) {
    const int b = 8 * s;
    const int r0 = b + 8, R = n - r0;
    if (R <= 0) break;
    const int mt = (R + 15) / 16, nt = (R + 7) / 8;
    // 1. panels: tiles 0..mt-1 of the column panel L(i, s) = A(i, s) inv(U_ss),
    //    then tiles 0..nt-1 of the row panel U(s, j) = inv(L_ss) A(s, j)
    for (int tile = warp; tile < mt + nt; tile += kLuThreads / 32) {
      double dr[4] = {0.0, 0.0, 0.0, 0.0}, di[4] = {0.0, 0.0, 0.0, 0.0};
      if (tile < mt) {
        const int m0 = r0 + tile * 16;
        const double a_r[4] = {Xr[(b + k0) * LD + m0 + g], Xr[(b + k0) * LD + m0 + g + 8],
                               Xr[(b + k1) * LD + m0 + g], Xr[(b + k1) * LD + m0 + g + 8]};
        const double b_r[2] = {VUr[k0 * 8 + g], VUr[k1 * 8 + g]};
        if constexpr (CP) {
          const double a_i[4] = {Xi[(b + k0) * LD + m0 + g], Xi[(b + k0) * LD + m0 + g + 8],
                                 Xi[(b + k1) * LD + m0 + g], Xi[(b + k1) * LD + m0 + g + 8]};
          const double a_ni[4] = {-a_i[0], -a_i[1], -a_i[2], -a_i[3]};
          const double b_i[2] = {VUi[k0 * 8 + g], VUi[k1 * 8 + g]};
          dmma_k8(dr, a_r, b_r);
          dmma_k8(dr, a_ni, b_i);
          dmma_k8(di, a_r, b_i);
          dmma_k8(di, a_i, b_r);
        } else {
          dmma_k8(dr, a_r, b_r);
        }
        __syncwarp();  // all lanes read the tile before any lane writes it
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int row = m0 + g + ((v >> 1) << 3), col = b + 2 * t + (v & 1);
          Xr[col * LD + row] = dr[v];
          if (CP) Xi[col * LD + row] = di[v];
        }
      } else {
        const int n0 = r0 + (tile - mt) * 8;
        // A operand inv(L_ss), rows 8..15 zero; B operand A(b + k, n0 + c)
        const double a_r[4] = {VLr[g * 8 + k0], 0.0, VLr[g * 8 + k1], 0.0};
        const double b_r[2] = {Xr[(n0 + g) * LD + b + k0], Xr[(n0 + g) * LD + b + k1]};
        if constexpr (CP) {
          const double a_i[4] = {VLi[g * 8 + k0], 0.0, VLi[g * 8 + k1], 0.0};
          const double a_ni[4] = {-a_i[0], 0.0, -a_i[2], 0.0};
          const double b_i[2] = {Xi[(n0 + g) * LD + b + k0], Xi[(n0 + g) * LD + b + k1]};
          dmma_k8(dr, a_r, b_r);
          dmma_k8(dr, a_ni, b_i);
          dmma_k8(di, a_r, b_i);
          dmma_k8(di, a_i, b_r);
        } else {
          dmma_k8(dr, a_r, b_r);
        }
        __syncwarp();
#pragma unroll
        for (int v = 0; v < 2; ++v) {  // rows 0..7 of the result: (g, n0 + 2t + v)
          const int col = n0 + 2 * t + v;
          Xr[col * LD + b + g] = dr[v];
          if (CP) Xi[col * LD + b + g] = di[v];
        }
      }
    }
    __syncthreads();
    // 2. trailing update A(i, j) -= L(i, s) U(s, j) over 16 x 8 tiles; tile 0
    //    holds the next diagonal block (look-ahead on warp 0)
    auto upd_tile = [&](int tile) {
      const int ti = tile / nt, tj = tile % nt;
      const int m0 = r0 + 16 * ti, n0 = r0 + 8 * tj;
      const double a_r[4] = {-Xr[(b + k0) * LD + m0 + g], -Xr[(b + k0) * LD + m0 + g + 8],
                             -Xr[(b + k1) * LD + m0 + g], -Xr[(b + k1) * LD + m0 + g + 8]};
      const double b_r[2] = {Xr[(n0 + g) * LD + b + k0], Xr[(n0 + g) * LD + b + k1]};
      double cr[4], ci[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = m0 + g + ((v >> 1) << 3), col = n0 + 2 * t + (v & 1);
        cr[v] = Xr[col * LD + row];
        ci[v] = CP ? Xi[col * LD + row] : 0.0;
      }
      if constexpr (CP) {
        const double a_i[4] = {-Xi[(b + k0) * LD + m0 + g], -Xi[(b + k0) * LD + m0 + g + 8],
                               -Xi[(b + k1) * LD + m0 + g], -Xi[(b + k1) * LD + m0 + g + 8]};
        const double a_ni[4] = {-a_i[0], -a_i[1], -a_i[2], -a_i[3]};
        const double b_i[2] = {Xi[(n0 + g) * LD + b + k0], Xi[(n0 + g) * LD + b + k1]};
        dmma_k8(cr, a_r, b_r);
        dmma_k8(cr, a_ni, b_i);
        dmma_k8(ci, a_r, b_i);
        dmma_k8(ci, a_i, b_r);
      } else {
        dmma_k8(cr, a_r, b_r);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = m0 + g + ((v >> 1) << 3), col = n0 + 2 * t + (v & 1);
        Xr[col * LD + row] = cr[v];
        if (CP) Xi[col * LD + row] = ci[v];
      }
    };
    if (warp == 0) {
      upd_tile(0);
      __syncwarp();
      diag_factor(r0);  // step s + 1 (its block is final after tile 0)
    } else {
      for (int tile = warp; tile < mt * nt; tile += kLuThreads / 32 - 1) upd_tile(tile);
    }
    __syncthreads();
  }

  // ---- store ----
  for (int e = tid; e < n * n; e += kLuThreads) {
    const int i = e % n, k = e / n;
    const size_t idx = (size_t)i + (size_t)k * lda;
    A[W * idx] = static_cast<S>(Xr[k * LD + i]);
    if (CP) A[2 * idx + 1] = static_cast<S>(Xi[k * LD + i]);
  }
}

struct LuCtx {
  int dt, es, ozaki;
  char* A;
  long lda;
  int* info;
  cudaStream_t st;
  // hybrid form: the recursion hands sub-problems of at most blk_leaf rows to
  // the blocked look-ahead form (widest block blk_nb); 0: recursion only
  long blk_leaf = 0, blk_nb = 0;
};

static int factor_blocked(const LuCtx& c, long i0, long i1, long nb);

template <class T>
static int launch_block(const LuCtx& c, char* Ad, long n, long i0) {
  using Sh = LuShape<T>;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_getrf_block<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Sh::SMEM) != cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  const long long tv = evlog_kern_begin(c.st, "k_getrf_block");
  k_getrf_block<T><<<1, kLuThreads, Sh::SMEM, c.st>>>(
      (int)n, reinterpret_cast<typename St<T>::S*>(Ad), c.lda, (int)i0, c.info);
  evlog_kern_end(tv, c.st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static int block(const LuCtx& c, long i0, long n) {
  char* Ad = c.A + (i0 + i0 * c.lda) * (long)c.es;
  switch (c.dt) {
    case XKB_S: return launch_block<float>(c, Ad, n, i0);
    case XKB_D: return launch_block<double>(c, Ad, n, i0);
    case XKB_C: return launch_block<float2>(c, Ad, n, i0);
    case XKB_Z: return launch_block<double2>(c, Ad, n, i0);
  }
  return XKB_EINVAL;
}

static int factor(const LuCtx& c, long i0, long i1) {
  const long n = i1 - i0;
  const bool cplx = c.dt == XKB_C || c.dt == XKB_Z;
  const long nmax = cplx ? LuShape<double2>::NMAX : LuShape<double>::NMAX;
  if (n <= nmax) return block(c, i0, n);
  if (c.blk_leaf > 0 && n <= c.blk_leaf && n > 2 * nmax) {  // hybrid: blocked below
    LuCtx cb = c;
    cb.blk_leaf = 0;
    return factor_blocked(cb, i0, i1, c.blk_nb);
  }
  constexpr long kSplit = 64;
  long h = i0 + ((n / 2 + kSplit - 1) / kSplit) * kSplit;
  if (h >= i1) h = i1 - kSplit;
  const long n1 = h - i0, n2 = i1 - h;
  int e;
  if ((e = factor(c, i0, h))) return e;
  const double one[2] = {1.0, 0.0};
  char* A11 = c.A + (i0 + i0 * c.lda) * (long)c.es;
  char* A12 = c.A + (i0 + h * c.lda) * (long)c.es;
  char* A21 = c.A + (h + i0 * c.lda) * (long)c.es;
  char* A22 = c.A + (h + h * c.lda) * (long)c.es;
  // U12 = L11^-1 A12 (left, lower, unit) on the caller's stream and
  // L21 = A21 U11^-1 (right, upper, non-unit) on a side stream: both read
  // only the factored A11 (the small, latency-bound solves of the deep
  // levels then run two at a time); the update below waits for both
  const SideStream& ss = side_stream(0);
  cudaStream_t s2 = side_fork(ss, c.st);
  if ((e = trsm_entry(c.dt, 0, XKB_LOWER, XKB_OP_N, 1, (int)n1, (int)n2, one, A11, c.lda, A12,
                      c.lda, c.ozaki, c.st, false)))
    return e;
  if ((e = trsm_entry(c.dt, 1, XKB_UPPER, XKB_OP_N, 0, (int)n2, (int)n1, one, A11, c.lda, A21,
                      c.lda, c.ozaki, s2, false)))
    return e;
  if (!side_join(ss, s2, c.st)) return XKB_ECUDA;
  // A22 -= L21 U12
  xkb_gemm_args g{};
  g.dtype = c.dt;
  g.opA = XKB_OP_N;
  g.opB = XKB_OP_N;
  g.M = g.N = (int)n2;
  g.K = (int)n1;
  g.alpha[0] = -1.0;
  g.beta[0] = 1.0;
  g.A = A21;
  g.lda = c.lda;
  g.B = A12;
  g.ldb = c.lda;
  g.C = A22;
  g.ldc = c.lda;
  g.uplo = XKB_FULL;
  bool done = false;
  if (c.ozaki > 0 && std::min(n1, n2) >= c.ozaki) {
    e = xkb_cuda_ozaki_gemm(&g, 0, c.st);
    if (e != XKB_ERANGE) {
      if (e) return e;
      done = true;
    }
  }
  if (!done && (e = xkb_cuda_gemm(&g, c.st))) return e;
  return factor(c, h, i1);
}

// Block width for `m` remaining rows in the blocked form: nb, halved
// (rounded down to a multiple of 64, at least nmin) while m <= shrink *
// width (tuning key getrf_shrink, default 12): wide blocks while the
// trailing update bounds each step, narrow ones once the critical path does.
static long block_width(long m, long nb, long nmin) {
  const double shrink = tune("getrf_shrink", 12.0);
  long w = nb;
  while (w > nmin && (double)m <= shrink * (double)w) w = std::max(nmin, (w / 2) / 64 * 64);
  return w;
}

// Blocked right-looking LU of rows / columns [i0, i1) with look-ahead.  Step
// k, with diagonal block D_k = L_k U_k factored; its column panel (below) and
// row panel (to the right) are each split into part 1 (the next block's
// rows / columns) and part 2 (the rest):
//   critical path (high-priority stream hp):  column part 1 = . U_k^-1 and
//     row part 1 = L_k^-1 ., then D_{k+1} -= L1 U1, then factor D_{k+1};
//   beside it (high-priority stream hp2):     both parts 2, then the rest of
//     block column k+1 (-= L2 U1) and block row k+1 (-= L1 U2);
//   trailing block (caller's stream):         -= L2 U2, one GEMM.
// The tile-level critical path of the reference's tile loop
// (blas/zgetrf_nopiv.c:48-101: getrf -> trsm -> gemm -> getrf per tile
// column) with nb-wide tiles.  Dependencies between the streams are events,
// as in the blocked Cholesky: the next diagonal block's update and block
// column / row k+1's updates wait for the previous trailing update; the next
// part-1 solves wait for block column / row k+1.
static int factor_blocked(const LuCtx& c, long i0, long i1, long nb) {
  const SideStream& hp = side_stream(kHiStream);
  const SideStream& hp2 = side_stream(kHiStream2);
  cudaEvent_t* ev = dep_events();
  if (!hp.s || !hp2.s || !ev) return factor(c, i0, i1);
  cudaEvent_t e_diag = ev[0], e_p1 = ev[1], e_p2 = ev[2], e_col = ev[3], e_trail = ev[4];
  const bool cplx = c.dt == XKB_C || c.dt == XKB_Z;
  const double one[2] = {1.0, 0.0};
  const long es = c.es, lda = c.lda;
  auto at = [&](long i, long j) { return c.A + (i + j * lda) * es; };
  // rows [r, r + m) of the column panel under block [b, b + nk): L = A U^-1
  auto solve_col = [&](long b, long nk, long r, long m, cudaStream_t st) {
    return trsm_entry(c.dt, 1, XKB_UPPER, XKB_OP_N, 0, (int)m, (int)nk, one, at(b, b), lda,
                      at(r, b), lda, 0, st, false);
  };
  // columns [q, q + w) of the row panel right of block [b, b + nk): U = L^-1 A
  auto solve_row = [&](long b, long nk, long q, long w, cudaStream_t st) {
    return trsm_entry(c.dt, 0, XKB_LOWER, XKB_OP_N, 1, (int)nk, (int)w, one, at(b, b), lda,
                      at(b, q), lda, 0, st, false);
  };
  // A(r.., q..) (m x w) -= L(r.., b..) U(b.., q..), inner nk
  auto rank_update = [&](long b, long nk, long r, long m, long q, long w, cudaStream_t st) {
    xkb_gemm_args g{};
    g.dtype = c.dt;
    g.opA = g.opB = XKB_OP_N;
    g.M = (int)m;
    g.N = (int)w;
    g.K = (int)nk;
    g.alpha[0] = -1.0;
    g.beta[0] = 1.0;
    g.A = at(r, b);
    g.B = at(b, q);
    g.C = at(r, q);
    g.lda = g.ldb = g.ldc = lda;
    g.uplo = XKB_FULL;
    if (c.ozaki > 0 && std::min(nk, std::min(m, w)) >= c.ozaki) {
      const int e = xkb_cuda_ozaki_gemm(&g, 0, st);
      if (e != XKB_ERANGE) return e;
    }
    return xkb_cuda_gemm(&g, st);
  };
  LuCtx ch = c;
  ch.st = side_fork(hp, c.st);
  int e = XKB_OK;
  auto rec = [&](cudaEvent_t x, cudaStream_t st) {
    if (!e && cudaEventRecord(x, st) != cudaSuccess) e = XKB_ECUDA;
  };
  auto wait = [&](cudaStream_t st, cudaEvent_t x) {
    if (!e && cudaStreamWaitEvent(st, x, 0) != cudaSuccess) e = XKB_ECUDA;
  };
  rec(e_trail, c.st);  // "previous trailing update": the caller's work so far
  const long nmin = cplx ? LuShape<double2>::NMAX : LuShape<double>::NMAX;
  long b = i0, nk = std::min(block_width(i1 - i0, nb, nmin), i1 - i0);
  e = factor(ch, b, b + nk);
  rec(e_diag, ch.st);
  while (!e && b + nk < i1) {
    const long r0 = b + nk, m2 = i1 - r0;
    const long n1 = std::min(block_width(m2, nb, nmin), m2), m3 = m2 - n1;
    if (m3 > 0) {  // hp2: both parts 2 (need D_k)
      wait(hp2.s, e_diag);
      if (!e) e = solve_col(b, nk, r0 + n1, m3, hp2.s);
      if (!e) e = solve_row(b, nk, r0 + n1, m3, hp2.s);
      rec(e_p2, hp2.s);
    }
    if (!e) e = solve_col(b, nk, r0, n1, ch.st);  // hp: both parts 1
    if (!e) e = solve_row(b, nk, r0, n1, ch.st);
    rec(e_p1, ch.st);
    if (m3 > 0) {  // hp2: block column and block row k+1 (need parts 1, previous trailing)
      wait(hp2.s, e_p1);
      wait(hp2.s, e_trail);
      if (!e) e = rank_update(b, nk, r0 + n1, m3, r0, n1, hp2.s);
      if (!e) e = rank_update(b, nk, r0, n1, r0 + n1, m3, hp2.s);
      rec(e_col, hp2.s);
    }
    wait(ch.st, e_trail);  // hp: D_{k+1} update (the previous trailing update wrote it)
    if (!e) e = rank_update(b, nk, r0, n1, r0, n1, ch.st);
    if (m3 > 0) {  // caller's stream: trailing block (needs parts 2)
      wait(c.st, e_p2);
      if (!e) e = rank_update(b, nk, r0 + n1, m3, r0 + n1, m3, c.st);
      rec(e_trail, c.st);
    }
    if (!e) e = factor(ch, r0, r0 + n1);  // hp: D_{k+1}
    rec(e_diag, ch.st);
    if (m3 > 0) wait(ch.st, e_col);  // the next parts 1 lie in block column / row k+1
    b = r0;
    nk = n1;
  }
  if (!side_join(hp2, hp2.s, c.st) && !e) e = XKB_ECUDA;
  if (!side_join(hp, ch.st, c.st) && !e) e = XKB_ECUDA;
  return e;
}

}  // namespace xkb

using namespace xkb;

extern "C" int xkb_cuda_getrf_nopiv(int dtype, int N, void* A, long lda, int* d_info, int ozaki,
                                    void* stream) {
  if (dtype < XKB_S || dtype > XKB_Z || N < 0 || lda < std::max(1, N) || (!A && N > 0))
    return XKB_EINVAL;
  if (N == 0) return XKB_OK;
  LuCtx c;
  c.dt = dtype;
  c.es = dtype == XKB_S ? 4 : (dtype == XKB_Z ? 16 : 8);
  c.ozaki = (dtype == XKB_D || dtype == XKB_Z) ? std::max(ozaki, 0) : 0;
  c.A = static_cast<char*>(A);
  c.lda = lda;
  c.info = d_info;
  c.st = resolve_stream(stream);
  // Blocked look-ahead form (tuning key getrf_blocked: 0 off, 1 in plain
  // mode, 2 in both modes; 3, the default: the hybrid in both modes -- the
  // recursion (its couplings in the Ozaki form in tensor-op mode) down to
  // getrf_oz_leaf rows (4096), the blocked form below; widest block
  // getrf_nb, in tensor-op mode getrf_nb_oz) or the recursive form.
  // Measured on a B200, tensor-op DGETRF 8192: hybrid 14.4 ms, recursive
  // 15.7, blocked 18.8.
  const long nmax = (dtype == XKB_C || dtype == XKB_Z) ? LuShape<double2>::NMAX
                                                       : LuShape<double>::NMAX;
  const int mode = (int)tune("getrf_blocked", 3.0);
  const long nb = std::max(nmax, ((long)tune(c.ozaki ? "getrf_nb_oz" : "getrf_nb",
                                             c.ozaki ? 2048.0 : 512.0) + 63) / 64 * 64);
  if (N > 2 * nmax && (mode == 2 || (mode == 1 && c.ozaki == 0)))
    return factor_blocked(c, 0, N, nb);
  if (mode == 3) {  // in plain mode too: DMMA couplings (8192: 18.3 against 18.9 ms)
    c.blk_leaf = std::max(2 * nmax + 1, (long)tune("getrf_oz_leaf", 4096.0));
    c.blk_nb = std::max(nmax, ((long)tune("getrf_nb", 512.0) + 63) / 64 * 64);
  }
  return factor(c, 0, N);
}
