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
// requested and large), and the trailing half is solved.  Diagonal blocks of
// <= 256 unknowns are solved in one launch of k_trsm_block (8-unknown
// substitution steps in registers + rank-8 DMMA updates, right-hand sides in
// shared memory).  This keeps every flop except O(n * 256 * nrhs) inside
// large GEMMs.
#include <algorithm>
#include <vector>

#include "trsm_leaf.cuh"
#include "xkb_dev.cuh"

namespace xkb {

constexpr int kSplit = 64;  // recursion split points are multiples of this

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

// Solve of one diagonal block of <= kBlk unknowns for all right-hand sides
// in one launch.  Each CTA takes CW right-hand sides and keeps them in shared
// memory (FP64, alpha applied on load).  The block is walked in steps of 8
// unknowns (forward for a lower effective triangle, backward for an upper
// one).  At the start the inverses of the block's 8 x 8 diagonal sub-blocks
// are formed in parallel, one thread per column (substitution against a unit
// vector); each step then takes Y = inv(T_ss) X_s with one DMMA per 8
// right-hand sides and applies the rank-8 update of the unknowns still to
// solve with DMMA (m16n8k8; complex: four real products).  The coupling strip
// T(rows still to solve, 8 columns) of each step is copied with cp.async two
// steps ahead into a ring of three buffers.
constexpr int kBlk = 256;
constexpr int kBlkThreads = 256;

template <class T>
struct BlkShape {
  using S = typename St<T>::S;
  static constexpr bool CP = St<T>::CPLX;
  static constexpr int CW = CP ? 8 : 16;      // right-hand sides per CTA
  static constexpr int NT = CW / 8;           // 8-column MMA tiles
  static constexpr int XROWS = kBlk + 16;     // rows incl. the last partial 16-row tile
  static constexpr int XS = XROWS + 2;        // column stride, = 2 mod 16
  static constexpr int YW = CW + 2;           // solved rows [8][YW]
  static constexpr int SRL = kBlk + 16 + 2;   // strip column stride (elements of S)
  static constexpr int PL = CP ? 2 : 1;       // real planes
  static constexpr int NBUF = 3;
  static constexpr size_t X_D = (size_t)PL * CW * XS;         // doubles
  static constexpr size_t Y_D = (size_t)PL * 8 * YW;          // doubles
  static constexpr size_t V_D = (size_t)PL * (kBlk / 8) * 64;  // doubles: inverses, [blk][i][j]
  static constexpr size_t S_B = sizeof(S) * PL * 8 * SRL;    // bytes per strip buffer
  static constexpr size_t SMEM = sizeof(double) * (X_D + Y_D + V_D) + NBUF * S_B;
  static constexpr int PE = kBlk * 8 / kBlkThreads;  // strip elements per thread
  static_assert(sizeof(S) * PL * kBlk * 8 <= S_B, "diagonal blocks are staged in one buffer");
};

template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* smem, const void* gmem, bool valid) {
  static_assert(BYTES == 4 || BYTES == 8, "element copy");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(smem)), "l"(gmem),
               "n"(BYTES), "r"(valid ? BYTES : 0)
               : "memory");
}

// leaves != nullptr: the inverses of several diagonal blocks at once, block
// y of the grid inverting the block of leaves[3y + 1] unknowns at
// (leaves[3y], leaves[3y]) into B + leaves[3y + 2] elements (ld ldb): the
// right-hand sides are the identity's columns (B is only written).
template <class T, bool LOWER>
__global__ void __launch_bounds__(kBlkThreads, 2)
    k_trsm_block(int nb_, int nrhs_, const typename St<T>::S* A_, long lda, int swap, int conj,
                 int unit, typename St<T>::S* B_, long ldb, int rhs_rows, double ar, double ai,
                 const int* leaves) {
  using Sh = BlkShape<T>;
  using S = typename St<T>::S;
  constexpr bool CP = Sh::CP;
  constexpr int CW = Sh::CW, XS = Sh::XS, YW = Sh::YW, SRL = Sh::SRL, PE = Sh::PE;
  constexpr int W = CP ? 2 : 1;
  int nb = nb_, nrhs = nrhs_;
  const S* A = A_;
  S* B = B_;
  const bool ident = leaves != nullptr;
  if (ident) {
    const int i0 = leaves[3 * blockIdx.y];
    nb = nrhs = leaves[3 * blockIdx.y + 1];
    A = A_ + (size_t)W * ((size_t)i0 + (size_t)i0 * (size_t)lda);
    B = B_ + (size_t)W * (size_t)(unsigned)leaves[3 * blockIdx.y + 2];
    if ((int)blockIdx.x * CW >= nb) return;  // the whole CTA is past this block's columns
  }
  extern __shared__ double sm_blk[];
  double* Xr = sm_blk;  // X[c * XS + row]
  double* Xi = Xr + (CP ? CW * XS : 0);
  double* Yr = sm_blk + Sh::X_D;  // Y[k * YW + c]: the 8 rows just solved
  double* Yi = Yr + (CP ? 8 * YW : 0);
  double* Vr = Yr + Sh::Y_D;  // inverse of diagonal sub-block m: V[m * 64 + i * 8 + j]
  double* Vi = Vr + (CP ? (kBlk / 8) * 64 : 0);
  S* strips = reinterpret_cast<S*>(Vr + Sh::V_D);
  auto strip_buf = [&](int q) { return strips + (size_t)q * (Sh::S_B / sizeof(S)); };
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int c0 = blockIdx.x * CW;
  const int cols = min(CW, nrhs - c0);
  const int nsub = (nb + 7) / 8;
  auto sub_of = [&](int s) { return LOWER ? s : nsub - 1 - s; };

  // ---- coupling strips: step s covers unknowns b = 8 sub(s) .. b+7; strip
  // row j is matrix row r0 + j (lower r0 = b, rows b..nb-1; upper r0 = 0,
  // rows 0..b+7), column k is matrix column b + k; stored [plane][k][row]
  // as raw elements of A.  This thread's elements, q = 0..PE-1: no swap
  // (columns of A contiguous) row tid, column q; swap (rows contiguous) row
  // 32 q + tid / 8, column tid % 8: consecutive threads, consecutive addresses.
  const int jt = swap ? tid >> 3 : tid, kt = swap ? tid & 7 : 0;
  const int jq = swap ? 32 : 0, kq = swap ? 0 : 1;
  auto strip_issue = [&](int s) {
    if (s < nsub) {
      const int b = 8 * sub_of(s), r0 = LOWER ? b : 0;
      const int rows = LOWER ? nb - b : min(nb, b + 8);
      S* dst = strip_buf(s % Sh::NBUF);
#pragma unroll
      for (int q = 0; q < PE; ++q) {
        const int j = jt + q * jq, k = kt + q * kq;
        const bool ok = j < rows && b + k < nb;
        const size_t idx = swap ? (size_t)(b + k) + (size_t)(r0 + j) * lda
                                : (size_t)(r0 + j) + (size_t)(b + k) * lda;
        const S* src = ok ? A + W * idx : A;
        cp_async_zfill<sizeof(S)>(dst + k * SRL + j, src, ok);
        if (CP) cp_async_zfill<sizeof(S)>(dst + 8 * SRL + k * SRL + j, ok ? src + 1 : A, ok);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");  // possibly empty: uniform counting
  };
  strip_issue(0);
  strip_issue(1);

  // ---- right-hand sides into shared memory (zero past nb rows / cols) ----
  for (int e = tid; e < CW * (Sh::XROWS - nb); e += kBlkThreads) {
    const int c = e / (Sh::XROWS - nb), r = nb + e % (Sh::XROWS - nb);
    Xr[c * XS + r] = 0.0;
    if (CP) Xi[c * XS + r] = 0.0;
  }
  {
    constexpr int GRP = kBlk * CW / kBlkThreads;  // one round of loads
    for (int e0 = 0; e0 < nb * CW; e0 += kBlkThreads * GRP) {
      double br[GRP], bi[GRP];
#pragma unroll
      for (int q = 0; q < GRP; ++q) {
        const int e = e0 + q * kBlkThreads + tid;
        const int i = rhs_rows ? e / CW : e % nb, c = rhs_rows ? e % CW : e / nb;
        br[q] = bi[q] = 0.0;
        if (e < nb * CW && c < cols) {
          if (ident) {
            br[q] = (i == c0 + c) ? 1.0 : 0.0;
          } else {
            const size_t idx = leaf_at(i, c0 + c, ldb, rhs_rows != 0);
            br[q] = (double)__ldcg(B + W * idx);
            if (CP) bi[q] = (double)__ldcg(B + 2 * idx + 1);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < GRP; ++q) {
        const int e = e0 + q * kBlkThreads + tid;
        const int i = rhs_rows ? e / CW : e % nb, c = rhs_rows ? e % CW : e / nb;
        if (e < nb * CW) {
          Xr[c * XS + i] = ar * br[q] - ai * bi[q];
          if (CP) Xi[c * XS + i] = ar * bi[q] + ai * br[q];
        }
      }
    }
  }

  // ---- inverses of the diagonal 8 x 8 sub-blocks ----
  {
    // stage the sub-blocks (raw, [m][plane][i][j]) in the third strip buffer
    S* D = strip_buf(2);
    constexpr int DE = kBlk * 8 / kBlkThreads;
#pragma unroll
    for (int q = 0; q < DE; ++q) {
      const int e = q * kBlkThreads + tid;
      const int m = e >> 6, i = (e >> 3) & 7, j = e & 7;
      const int rr = 8 * m + i, qq = 8 * m + j;
      S vr = S(0), vi = S(0);
      if (m < nsub && rr < nb && qq < nb && (LOWER ? rr >= qq : rr <= qq)) {
        const size_t idx = swap ? (size_t)qq + (size_t)rr * lda : (size_t)rr + (size_t)qq * lda;
        vr = __ldcg(A + W * idx);
        if (CP) vi = __ldcg(A + 2 * idx + 1);
      }
      D[m * 64 * Sh::PL + i * 8 + j] = vr;
      if (CP) D[m * 128 + 64 + i * 8 + j] = vi;
    }
    __syncthreads();
    // thread (m, kk): column kk of inv(T_m), T_m z = e_kk by substitution;
    // rows / columns past nb (zero when staged) act as the identity.  Every
    // thread takes part (the shuffles below span whole warps); sub-blocks
    // past the last one invert the identity.
    const int m = tid >> 3, kk = tid & 7;
    {
      const S* Dm = D + m * 64 * Sh::PL;
      auto tv = [&](int i, int j, double& re, double& im) {
        re = (double)Dm[i * 8 + j];
        im = CP ? (conj ? -(double)Dm[64 + i * 8 + j] : (double)Dm[64 + i * 8 + j]) : 0.0;
      };
      // reciprocal diagonal: thread kk forms entry kk, the 8 threads of the
      // sub-block (consecutive lanes) share them
      double rk = 1.0, ik = 0.0;
      {
        double dr, di;
        tv(kk, kk, dr, di);
        if (!(unit || 8 * m + kk >= nb)) {
          if (CP) {
            const double den = dr * dr + di * di;
            rk = dr / den;
            ik = -di / den;
          } else {
            rk = 1.0 / dr;
          }
        }
      }
      double rr_[8], ri_[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        rr_[i] = __shfl_sync(0xffffffffu, rk, (lane & ~7) | i);
        ri_[i] = CP ? __shfl_sync(0xffffffffu, ik, (lane & ~7) | i) : 0.0;
      }
      // column form: each step one multiply, then independent updates.  All
      // register arrays are indexed by unrolled loop counters (kk only enters
      // predicates), so they stay in registers.
      double zr[8], zi[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        zr[i] = i == kk ? 1.0 : 0.0;
        zi[i] = 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int jj = LOWER ? q : 7 - q;
        if (LOWER ? jj >= kk : jj <= kk) {
          const double vr = zr[jj] * rr_[jj] - zi[jj] * ri_[jj];
          const double vi = zr[jj] * ri_[jj] + zi[jj] * rr_[jj];
          zr[jj] = vr;
          zi[jj] = vi;
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            if (LOWER ? i > jj : i < jj) {
              double tr, ti;
              tv(i, jj, tr, ti);
              zr[i] -= tr * vr - ti * vi;
              zi[i] -= tr * vi + ti * vr;
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        Vr[m * 64 + i * 8 + kk] = zr[i];
        if (CP) Vi[m * 64 + i * 8 + kk] = zi[i];
      }
    }
  }

  // Each step: every warp forms Y^T = X_s^T inv(T_ss)^T itself -- one DMMA
  // with M = the CTA's right-hand sides (16; complex 8, rows 8..15 zero),
  // N = K = the 8 unknowns.  Its accumulator fragment is exactly the B
  // fragment the rank-8 update needs: lane (g, t) holds Y(2t, c) and
  // Y(2t+1, c) for c = g (registers 0, 1) and c = g + 8 (registers 2, 3).  So
  // no warp waits for another between the solve and the update (one barrier
  // per step).  Warp 0 writes the solved rows back into X after the next
  // barrier, when no warp reads X_s any more.
  double pyr[4] = {0.0, 0.0, 0.0, 0.0}, pyi[4] = {0.0, 0.0, 0.0, 0.0};
  int pb = -1;  // unknowns of the step whose rows warp 0 still holds
  auto store_y = [&]() {
    const int k0 = 2 * t;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int c = g + ((v >> 1) << 3), row = pb + k0 + (v & 1);
      if (c < CW) {
        Xr[c * XS + row] = pyr[v];
        if (CP) Xi[c * XS + row] = pyi[v];
      }
    }
  };
  for (int s = 0; s < nsub; ++s) {
    const int b = 8 * sub_of(s), r0 = LOWER ? b : 0;
    // strip s landed (strip s+1 may still be in flight); the barrier also
    // ends the previous step (its update, its reads of X_s) and the inverses
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    if (warp == 0 && pb >= 0) store_y();
    strip_issue(s + 2);  // into the buffer step s-1 read
    // 1. Y^T = X_s^T inv(T_ss)^T in every warp (k indices 2t, 2t+1 for both
    //    operands: the same permutation on A and B leaves the sum unchanged)
    double yr[4] = {0.0, 0.0, 0.0, 0.0}, yi[4] = {0.0, 0.0, 0.0, 0.0};
    {
      const int m = b / 8, k0 = 2 * t, k1 = k0 + 1;
      const double* vr = Vr + m * 64;
      const double* vi = Vi + m * 64;
      const bool hi = CW > 8;  // right-hand sides g + 8 exist
      const double a_r[4] = {Xr[g * XS + b + k0], hi ? Xr[(g + 8) * XS + b + k0] : 0.0,
                             Xr[g * XS + b + k1], hi ? Xr[(g + 8) * XS + b + k1] : 0.0};
      const double b_r[2] = {vr[g * 8 + k0], vr[g * 8 + k1]};
      if constexpr (CP) {
        const double a_i[4] = {Xi[g * XS + b + k0], hi ? Xi[(g + 8) * XS + b + k0] : 0.0,
                               Xi[g * XS + b + k1], hi ? Xi[(g + 8) * XS + b + k1] : 0.0};
        const double a_ni[4] = {-a_i[0], -a_i[1], -a_i[2], -a_i[3]};
        const double b_i[2] = {vi[g * 8 + k0], vi[g * 8 + k1]};
        dmma_k8(yr, a_r, b_r);
        dmma_k8(yr, a_ni, b_i);
        dmma_k8(yi, a_r, b_i);
        dmma_k8(yi, a_i, b_r);
      } else {
        dmma_k8(yr, a_r, b_r);
      }
    }
    if (warp == 0) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        pyr[v] = yr[v];
        pyi[v] = yi[v];
      }
      pb = b;
    }
    // 2. rows still to solve -= T(rows, b..b+7) Y: 16 x 8 DMMA tiles
    const S* str = strip_buf(s % Sh::NBUF);
    const S* sti = str + 8 * SRL;
    const int u0 = LOWER ? b + 8 : 0, u1 = LOWER ? nb : b;
    const int mt = (u1 - u0 + 15) / 16;
    for (int tile = warp; tile < mt * Sh::NT; tile += kBlkThreads / 32) {
      const int m0 = u0 + (tile / Sh::NT) * 16, n0 = (tile % Sh::NT) * 8;
      const int ra = m0 + g - r0, rb = ra + 8;  // strip rows of this lane
      const int k0 = 2 * t, k1 = k0 + 1;
      const double a_r[4] = {-(double)str[k0 * SRL + ra], -(double)str[k0 * SRL + rb],
                             -(double)str[k1 * SRL + ra], -(double)str[k1 * SRL + rb]};
      const double b_r[2] = {n0 ? yr[2] : yr[0], n0 ? yr[3] : yr[1]};
      double cr[4], ci[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = m0 + g + ((v >> 1) << 3), col = n0 + 2 * t + (v & 1);
        cr[v] = Xr[col * XS + row];
        ci[v] = CP ? Xi[col * XS + row] : 0.0;
      }
      if constexpr (CP) {
        // T = A or conj(A); C -= T Y: re += (-Tr) Yr + Ti Yi, im += (-Tr) Yi + (-Ti) Yr
        const double sg = conj ? 1.0 : -1.0;  // -Ti
        const double a_i[4] = {sg * (double)sti[k0 * SRL + ra], sg * (double)sti[k0 * SRL + rb],
                               sg * (double)sti[k1 * SRL + ra], sg * (double)sti[k1 * SRL + rb]};
        const double a_ni[4] = {-a_i[0], -a_i[1], -a_i[2], -a_i[3]};
        const double b_i[2] = {n0 ? yi[2] : yi[0], n0 ? yi[3] : yi[1]};
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
        if (row < u1) {
          Xr[col * XS + row] = cr[v];
          if (CP) Xi[col * XS + row] = ci[v];
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  if (warp == 0 && pb >= 0) store_y();
  __syncthreads();

  // ---- store ----
#pragma unroll 4
  for (int e = tid; e < nb * CW; e += kBlkThreads) {
    const int i = rhs_rows ? e / CW : e % nb, c = rhs_rows ? e % CW : e / nb;
    if (c >= cols) continue;
    const size_t idx = leaf_at(i, c0 + c, ldb, rhs_rows != 0);
    B[W * idx] = static_cast<S>(Xr[c * XS + i]);
    if (CP) B[2 * idx + 1] = static_cast<S>(Xi[c * XS + i]);
  }
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
static int launch_block(int n, int nrhs, const void* A, long lda, int swap, int conj, int lower,
                        int unit, void* B, long ldb, int rhs_rows, const double* al,
                        cudaStream_t st, const int* leaves = nullptr, int nleaves = 0) {
  using S = typename St<T>::S;
  using Sh = BlkShape<T>;
  const dim3 grid(leaves ? (unsigned)((kBlk + Sh::CW - 1) / Sh::CW)
                         : (unsigned)((nrhs + Sh::CW - 1) / Sh::CW),
                  leaves ? (unsigned)nleaves : 1u);
  auto kb = lower ? k_trsm_block<T, true> : k_trsm_block<T, false>;
  static bool attr[2] = {false, false};
  if (!attr[lower ? 1 : 0]) {
    if (cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM) !=
        cudaSuccess)
      return XKB_ECUDA;
    attr[lower ? 1 : 0] = true;
  }
  const long long tv = evlog_kern_begin(st, "k_trsm_block");
  kb<<<grid, kBlkThreads, Sh::SMEM, st>>>(n, nrhs, static_cast<const S*>(A), lda, swap, conj,
                                          unit, static_cast<S*>(B), ldb, rhs_rows, al[0], al[1],
                                          leaves);
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static int block_dispatch(int dt, int n, int nrhs, const void* A, long lda, int swap, int conj,
                          int lower, int unit, void* B, long ldb, int rhs_rows, const double* al,
                          cudaStream_t st) {
  switch (dt) {
    case XKB_S: return launch_block<float>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_D: return launch_block<double>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_C: return launch_block<float2>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
    case XKB_Z: return launch_block<double2>(n, nrhs, A, lda, swap, conj, lower, unit, B, ldb, rhs_rows, al, st);
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
  // inverse leaves (null: every leaf is a block solve): inv(E_l) of the
  // effective triangle of the leaf (or pair of leaves) starting at unknown
  // inv_at[2q] at Winv + inv_at[2q + 1] elements (ld ldw); tmp holds one
  // leaf's product (ldw rows); pair p's inverse is complete once pair_ev[p]
  // has fired
  const char* Winv = nullptr;
  long ldw = kBlk;
  const std::vector<long>* inv_at = nullptr;
  const cudaEvent_t* pair_ev = nullptr;
  char* tmp = nullptr;
};

// A leaf applied through its inverse: X = alpha inv(E) B (left) or
// X = alpha B inv(E)^T (right side: E is op(A)^T there), one GEMM into tmp
// and a copy back into B.  A pair split at mid (> 0; left side only) may
// skip the zero upper-right block of its inverse (tuning key
// trsm_pair_split, default 0): X_0 = alpha inv(E_00) B_0 and X_1 = alpha
// [Z inv(E_11)] [B_0; B_1], two GEMMs into tmp.  Measured on a B200 (DTRSM
// 4096, alternating): 2.83 -> 2.86 ms plain, 2.30 -> 2.32 tensor-op -- the
// second launch on the chain costs more than the quarter of the product's
// flops it saves.
static int leaf_gemm(const TrsmCtx& c, long i0, long n, const double* alpha, long mid = 0) {
  const auto& L = *c.inv_at;
  size_t q = 0;
  while (2 * q < L.size() && L[2 * q] != i0) ++q;
  if (2 * q >= L.size()) return XKB_EINVAL;
  xkb_gemm_args g{};
  g.dtype = c.dt;
  g.alpha[0] = alpha[0];
  g.alpha[1] = alpha[1];
  g.uplo = XKB_FULL;
  const char* Wl = c.Winv + (size_t)L[2 * q + 1] * c.es;
  char* Bk = c.left ? c.B + i0 * (long)c.es : c.B + i0 * c.ldb * (long)c.es;
  size_t dpitch, spitch, width, height;
  if (c.left) {
    g.M = (int)n;
    g.N = c.nrhs;
    g.K = (int)n;
    g.opA = XKB_OP_N;
    g.A = Wl;
    g.lda = c.ldw;
    g.opB = XKB_OP_N;
    g.B = Bk;
    g.ldb = c.ldb;
    g.C = c.tmp;
    g.ldc = c.ldw;
    spitch = (size_t)c.ldw * c.es;
    width = n * (size_t)c.es;
    height = (size_t)c.nrhs;
  } else {
    g.M = c.nrhs;
    g.N = (int)n;
    g.K = (int)n;
    g.opA = XKB_OP_N;
    g.A = Bk;
    g.lda = c.ldb;
    g.opB = XKB_OP_T;
    g.B = Wl;
    g.ldb = c.ldw;
    g.C = c.tmp;
    g.ldc = c.nrhs;
    spitch = (size_t)c.nrhs * c.es;
    width = (size_t)c.nrhs * c.es;
    height = (size_t)n;
  }
  dpitch = (size_t)c.ldb * c.es;
  if (c.left && mid > 0 && tune("trsm_pair_split", 0.0) != 0.0) {
    const long n0 = mid - i0;
    xkb_gemm_args g0 = g;  // X_0: rows [0, n0) of the product
    g0.M = (int)n0;
    g0.K = (int)n0;
    if (int e = xkb_cuda_gemm(&g0, c.st)) return e;
    g.M = (int)(n - n0);  // X_1: rows [n0, n), all n columns of the inverse
    g.A = Wl + (size_t)n0 * c.es;
    g.C = c.tmp + (size_t)n0 * c.es;
  }
  if (int e = xkb_cuda_gemm(&g, c.st)) return e;
  return cudaMemcpy2DAsync(Bk, dpitch, c.tmp, spitch, width, height, cudaMemcpyDeviceToDevice,
                           c.st) == cudaSuccess
             ? XKB_OK
             : XKB_ECUDA;
}

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

// The recursion below as a flat list of operations in issue order: a leaf
// (diagonal block [i0, i0 + n)) or a coupling update (rows [p0, p1) from
// the solved rows [q0, q1)); `scaled` marks the operations that apply the
// caller's alpha (the others use 1).
// With pairs on (forward solves), a node of two leaves other than the first
// is one operation: a leaf over both (q0 = the split point, pair = its
// index), applied through the inverse of the pair's triangle.
struct SolveOp {
  bool leaf, scaled;
  long p0, p1, q0, q1;  // leaf: [p0, p1) only
  int pair;             // >= 0: a pair of leaves split at q0
};

static void plan_solve(const TrsmCtx& c, long i0, long i1, bool scaled,
                       std::vector<SolveOp>& ops, bool pairs, int& npairs) {
  const long n = i1 - i0;
  if (n <= kBlk) {
    ops.push_back({true, scaled, i0, i1, 0, 0, -1});
    return;
  }
  long h = i0 + ((n / 2 + kSplit - 1) / kSplit) * kSplit;
  if (h >= i1) h = i1 - kSplit;
  if (pairs && c.fwd && i0 > 0 && h - i0 <= kBlk && i1 - h <= kBlk) {
    ops.push_back({true, scaled, i0, i1, h, 0, npairs++});
    return;
  }
  if (c.fwd) {
    plan_solve(c, i0, h, scaled, ops, pairs, npairs);
    ops.push_back({false, scaled, h, i1, i0, h, -1});
    plan_solve(c, h, i1, false, ops, pairs, npairs);
    return;
  }
  plan_solve(c, h, i1, scaled, ops, pairs, npairs);
  ops.push_back({false, scaled, i0, h, h, i1, -1});
  plan_solve(c, i0, h, false, ops, pairs, npairs);
}

static int issue(const TrsmCtx& c, const SolveOp& op, const double* alpha) {
  const double one[2] = {1.0, 0.0};
  const double* al = op.scaled ? alpha : one;
  if (!op.leaf) return update(c, op.p0, op.p1, op.q0, op.q1, al);
  const long i0 = op.p0, n = op.p1 - op.p0;
  if (op.pair >= 0 && c.pair_ev && cudaStreamWaitEvent(c.st, c.pair_ev[op.pair], 0) != cudaSuccess)
    return XKB_ECUDA;
  if (c.Winv) return leaf_gemm(c, i0, n, al, op.pair >= 0 ? op.q0 : 0);
  // diagonal block of the effective triangle: one launch
  const char* Ad = aptr(c, i0, i0);
  char* Bd = c.left ? c.B + i0 * (long)c.es : c.B + i0 * c.ldb * (long)c.es;
  return block_dispatch(c.dt, (int)n, c.nrhs, Ad, c.lda, c.swap, c.conj, c.lower_eff, c.unit,
                        Bd, c.ldb, c.left ? 0 : 1, al, c.st);
}

}  // namespace xkb

using namespace xkb;

namespace xkb {
int trsm_entry(int dtype, int side, int uplo, int trans, int diag, int M, int N,
               const double* alpha, const void* A, long lda, void* B, long ldb, int ozaki,
               cudaStream_t st, bool split_rhs) {
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
  c.st = st;
  const bool lower = uplo == XKB_LOWER;
  const bool op_lower = lower ^ (c.trans != XKB_OP_N);  // op(A) lower?
  // effective triangle element access, as in k_trsm_block
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
  // Inverse leaves (tuning key trsm_inv_leaves, default 1; FP64 storage,
  // more than one leaf, >= 64 right-hand sides): the inverses of all the
  // recursion's diagonal blocks are formed first by ONE launch of the block
  // kernel (a grid row per block, identity right-hand sides), and each leaf
  // becomes a GEMM with its inverse -- the latency-bound substitution chains
  // leave the recursion's critical path.  The products with inv(E_l) carry
  // the condition number of the <= 256-unknown diagonal blocks, as blocked
  // solvers with inverted diagonal blocks do.
  // Pairs of leaves (tuning key trsm_pair_leaves, default 1; left side,
  // forward, op(A) = A, >= 2048 unknowns): every node of two leaves but the
  // first becomes ONE product with the inverse of its <= 512-unknown
  // triangle, [inv(E_00) 0; Z inv(E_11)] with Z = -inv(E_11) E_10 inv(E_00)
  // (two GEMMs per pair, formed on a side stream while the solve runs; a
  // pair's product waits for its event), instead of leaf, coupling update,
  // leaf -- three dependent small GEMMs on the critical path.  The products
  // then carry the condition number of the pairs' triangles.
  const bool inv = (dtype == XKB_D || dtype == XKB_Z) && n > kBlk && c.nrhs >= 64 &&
                   tune("trsm_inv_leaves", 1.0) != 0.0;
  const bool pairs = inv && c.left && c.trans == XKB_OP_N && c.fwd && n >= 2048 &&
                     tune("trsm_pair_leaves", 1.0) != 0.0;
  int npairs = 0;
  std::vector<SolveOp> ops;
  plan_solve(c, 0, n, true, ops, pairs, npairs);
  std::vector<long> inv_at;  // (first unknown, element offset) per leaf or pair
  void* Wbuf = nullptr;
  int* dtab = nullptr;
  void* Wtmp = nullptr;
  std::vector<cudaEvent_t> pev;
  cudaStream_t pst = st;  // the stream that forms the pairs' inverses
  auto release_inv = [&]() {
    if (pst != st) side_join(side_stream(kTrsmInvStream), pst, st);
    for (cudaEvent_t ev : pev)
      if (ev) cudaEventDestroy(ev);
    if (Wtmp) cudaFreeAsync(Wtmp, st);
    if (Wbuf) cudaFreeAsync(Wbuf, st);
    if (dtab) cudaFreeAsync(dtab, st);
  };
  if (inv) {
    const long ldw = npairs > 0 ? 2 * kBlk : kBlk;
    std::vector<int> table;  // inverse launch: (first unknown, size, offset) per block
    long slot = 0;
    for (const SolveOp& op : ops) {
      if (!op.leaf) continue;
      const long off = slot++ * ldw * ldw;
      inv_at.push_back(op.p0);
      inv_at.push_back(off);
      if (op.pair >= 0) {
        const long h = op.q0 - op.p0;
        table.insert(table.end(), {(int)op.p0, (int)h, (int)off});
        table.insert(table.end(), {(int)op.q0, (int)(op.p1 - op.q0), (int)(off + h + h * ldw)});
      } else {
        table.insert(table.end(), {(int)op.p0, (int)(op.p1 - op.p0), (int)off});
      }
    }
    const int nl = (int)table.size() / 3;
    const size_t wbytes = (size_t)slot * ldw * ldw * c.es;
    if (cudaMallocAsync(&Wbuf, wbytes, st) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&dtab), table.size() * sizeof(int), st) !=
            cudaSuccess ||
        (npairs > 0 && cudaMallocAsync(&Wtmp, (size_t)kBlk * kBlk * c.es, st) != cudaSuccess)) {
      cudaGetLastError();
      release_inv();
      return XKB_ENOMEM;
    }
    // a pair's upper-right block is zero; pageable source: staged before the
    // call returns
    if ((npairs > 0 && cudaMemsetAsync(Wbuf, 0, wbytes, st) != cudaSuccess) ||
        cudaMemcpyAsync(dtab, table.data(), table.size() * sizeof(int), cudaMemcpyHostToDevice,
                        st) != cudaSuccess) {
      release_inv();
      return XKB_ECUDA;
    }
    const double one[2] = {1.0, 0.0};
    int e = dtype == XKB_D
                ? launch_block<double>(kBlk, kBlk, A, lda, c.swap, c.conj, c.lower_eff, c.unit,
                                       Wbuf, ldw, 0, one, st, dtab, nl)
                : launch_block<double2>(kBlk, kBlk, A, lda, c.swap, c.conj, c.lower_eff, c.unit,
                                        Wbuf, ldw, 0, one, st, dtab, nl);
    if (e) {
      release_inv();
      return e;
    }
    c.Winv = static_cast<const char*>(Wbuf);
    c.ldw = ldw;
    c.inv_at = &inv_at;
    if (npairs > 0) {
      pev.assign((size_t)npairs, nullptr);
      for (cudaEvent_t& ev : pev)
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
          cudaGetLastError();
          ev = nullptr;
          release_inv();
          return XKB_ECUDA;
        }
      pst = side_fork(side_stream(kTrsmInvStream), st);
      size_t q = 0;
      for (const SolveOp& op : ops) {
        if (!op.leaf) continue;
        const long off = inv_at[2 * q + 1];
        ++q;
        if (op.pair < 0) continue;
        const long n0 = op.q0 - op.p0, n1 = op.p1 - op.q0;
        char* P = static_cast<char*>(Wbuf) + (size_t)off * c.es;
        xkb_gemm_args g{};
        g.dtype = dtype;
        g.uplo = XKB_FULL;
        g.opA = g.opB = XKB_OP_N;
        // W = E_10 inv(E_00), n1 x n0
        g.M = (int)n1;
        g.N = (int)n0;
        g.K = (int)n0;
        g.alpha[0] = 1.0;
        g.A = aptr(c, op.q0, op.p0);
        g.lda = lda;
        g.B = P;
        g.ldb = ldw;
        g.C = Wtmp;
        g.ldc = kBlk;
        if ((e = xkb_cuda_gemm(&g, pst))) break;
        // Z = -inv(E_11) W into the pair's lower-left block
        g.K = (int)n1;
        g.alpha[0] = -1.0;
        g.A = P + (size_t)(n0 + n0 * ldw) * c.es;
        g.lda = ldw;
        g.B = Wtmp;
        g.ldb = kBlk;
        g.C = P + (size_t)n0 * c.es;
        g.ldc = ldw;
        if ((e = xkb_cuda_gemm(&g, pst))) break;
        if (cudaEventRecord(pev[(size_t)op.pair], pst) != cudaSuccess) {
          e = XKB_ECUDA;
          break;
        }
      }
      if (e) {
        release_inv();
        return e;
      }
      c.pair_ev = pev.data();
    }
  }
  std::vector<void*> tmps;
  auto give_tmp = [&](TrsmCtx& part) {
    if (!inv) return XKB_OK;
    void* t = nullptr;
    if (cudaMallocAsync(&t, (size_t)c.ldw * part.nrhs * c.es, st) != cudaSuccess) {
      cudaGetLastError();
      return XKB_ENOMEM;
    }
    tmps.push_back(t);
    part.tmp = static_cast<char*>(t);
    return XKB_OK;
  };
  auto release = [&](int e) {
    release_inv();
    for (void* t : tmps) cudaFreeAsync(t, st);
    return e;
  };
  // Many right-hand sides: G independent groups (tuning key
  // trsm_rhs_groups, default 2; groups of >= 1024 right-hand sides, multiples
  // of 64), the first on the caller's stream and the others on side
  // streams, so that one group's latency-bound diagonal-block solves overlap
  // the other groups' coupling GEMMs.  In the Ozaki form each group converts
  // the coupling blocks of A again, which pays only with more right-hand
  // sides than unknowns.
  constexpr long kSplitRhs = 2048;
  const long groups = std::min<long>(std::max(1.0, tune("trsm_rhs_groups", 2.0)),
                                     std::min<long>(4, c.nrhs / (kSplitRhs / 2)));
  if (split_rhs && c.nrhs >= kSplitRhs && groups >= 2 && (c.ozaki == 0 || c.nrhs > n)) {
    const long per = (c.nrhs / groups + 63) / 64 * 64;
    TrsmCtx parts[4];
    cudaStream_t forked[4];
    long start = 0;
    int np = 0;
    for (long g = 0; g < groups && start < c.nrhs; ++g, ++np) {
      parts[g] = c;
      parts[g].nrhs = g == groups - 1 ? c.nrhs - start : std::min(per, c.nrhs - start);
      parts[g].B = c.B + (c.left ? start * ldb : start) * (long)c.es;
      if (int e = give_tmp(parts[g])) return release(e);
      start += parts[g].nrhs;
    }
    for (int g = 0; g < np; ++g) {
      forked[g] = g == 0 ? c.st : side_fork(side_stream(g), c.st);
      parts[g].st = forked[g];
    }
    // the groups' operations are issued interleaved, one operation of every
    // group in turn, so that all groups start together and run side by side
    // to the end (issued group after group, the last group started one
    // group's host issue time late and finished alone)
    int e = XKB_OK;
    for (const SolveOp& op : ops)
      for (int g = 0; g < np && !e; ++g) e = issue(parts[g], op, alpha);
    for (int g = 1; g < np; ++g)
      if (!side_join(side_stream(g), forked[g], c.st) && !e) e = XKB_ECUDA;
    return release(e);
  }
  if (int e = give_tmp(c)) return release(e);
  for (const SolveOp& op : ops)
    if (int e = issue(c, op, alpha)) return release(e);
  return release(XKB_OK);
}
}  // namespace xkb

extern "C" int xkb_cuda_trsm(int dtype, int side, int uplo, int trans, int diag, int M, int N,
                             const double* alpha, const void* A, long lda, void* B, long ldb,
                             int ozaki, void* stream) {
  return trsm_entry(dtype, side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb, ozaki,
                    resolve_stream(stream), true);
}

// The product on the materialised operand: Ozaki INT8 form when ozaki > 0,
// the dtype is XKB_D / XKB_Z and all three dimensions reach ozaki (falling
// back to DMMA when the contraction is beyond the exact-INT32 limit).
static int product(xkb_gemm_args& g, int ozaki, cudaStream_t st) {
  if (ozaki > 0 && (g.dtype == XKB_D || g.dtype == XKB_Z) &&
      std::min(std::min(g.M, g.N), g.K) >= ozaki) {
    const int e = xkb_cuda_ozaki_gemm(&g, 0, st);
    if (e != XKB_ERANGE) return e;
  }
  return xkb_cuda_gemm(&g, st);
}

extern "C" int xkb_cuda_trmm(int dtype, int side, int uplo, int trans, int diag, int M, int N,
                             const double* alpha, const void* A, long lda, void* B, long ldb,
                             int ozaki, void* stream) {
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
  const long long tv = evlog_kern_begin(st, "k_tri_fill+k_copy2d");
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
  evlog_kern_end(tv, st);
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
  int e = product(g, ozaki, st);
  cudaFreeAsync(T, st);
  cudaFreeAsync(Bc, st);
  return e;
}

extern "C" int xkb_cuda_symm(int dtype, int herm, int side, int uplo, int M, int N,
                             const double* alpha, const void* A, long lda, const void* B,
                             long ldb, const double* beta, void* C, long ldc, int ozaki,
                             void* stream) {
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
  const long long tv = evlog_kern_begin(st, "k_sym_fill");
  switch (dtype) {
    case XKB_S: k_sym_fill<float><<<g1, 256, 0, st>>>((int)na, (const float*)A, lda, lower, 0, (float*)S, ldt); break;
    case XKB_D: k_sym_fill<double><<<g1, 256, 0, st>>>((int)na, (const double*)A, lda, lower, 0, (double*)S, ldt); break;
    case XKB_C: k_sym_fill<float2><<<g1, 256, 0, st>>>((int)na, (const float2*)A, lda, lower, hm, (float2*)S, ldt); break;
    case XKB_Z: k_sym_fill<double2><<<g1, 256, 0, st>>>((int)na, (const double2*)A, lda, lower, hm, (double2*)S, ldt); break;
  }
  evlog_kern_end(tv, st);
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
  int e = product(g, ozaki, st);
  cudaFreeAsync(S, st);
  return e;
}
