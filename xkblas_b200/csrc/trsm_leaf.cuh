// trsm_leaf.cuh -- FP64 solve of one diagonal block of a triangular system
// (n <= 64 unknowns) against a range of right-hand sides, used by the
// tile-task executor's solve tasks (sched.cu); leaf_at is shared with the
// whole-matrix solver (trsm.cu).  It is the body the reference hands to
// cublasZtrsm for a diagonal tile (blas/ztask_trsm.c:162-180).
//
// X = alpha op(T)^-1 B by substitution.  A right-hand side is held by G lanes
// of one warp, lane g keeping rows RPL*g .. RPL*g + RPL-1 in registers (real
// RPL 16, G 4; complex RPL 8, G 8).  At step i the owner of row i scales it
// by the reciprocal of T(i,i) (the packed-reciprocal form CPU BLAS kernels
// use), the G lanes share it by shuffle, and each lane updates its rows below
// (lower) or above (upper) i.  op(T) is staged column by column in shared
// memory, row groups GS = RPL + 2 doubles apart so that the G lanes' 16-byte
// loads fall in distinct banks.  Storage types float / double / float2 /
// double2; arithmetic in FP64.
#pragma once
#include "dmma_common.cuh"

namespace xkb {

constexpr int kLeafRows = 64;

// RPL_REAL: rows per lane for real types (complex: half of it).  Fewer rows
// per lane mean more lanes per right-hand side: more warps to hide the
// per-step shuffle latency when right-hand sides are many, more shuffles per
// step when they are few.
template <class T, int RPL_REAL = 16>
struct LeafShape {
  static constexpr bool CPLX = St<T>::CPLX;
  static constexpr int RPL = CPLX ? RPL_REAL / 2 : RPL_REAL;  // rows per lane
  static constexpr int G = kLeafRows / RPL;     // lanes per right-hand side
  static constexpr int GS = RPL + 2;            // staged row-group stride
  static constexpr int COL = G * GS;            // staged column stride
  // shared bytes: op(T) (real [+ imaginary]) and the reciprocal diagonal
  static constexpr size_t SMEM = (CPLX ? 2 : 1) * sizeof(double) * (kLeafRows * COL) +
                                 2 * sizeof(double) * kLeafRows;
};

// element (row i, right-hand side c) of B: rhs_rows ? B[c + i ldb] : B[i + c ldb]
__device__ __forceinline__ size_t leaf_at(int i, int c, long ldb, bool rhs_rows) {
  return rhs_rows ? (size_t)c + (size_t)i * (size_t)ldb : (size_t)i + (size_t)c * (size_t)ldb;
}

// Stage op(T) for the n x n block at A: T(i,j) = A[swap ? j + i lda : i + j lda]
// (conjugated when conj), zero outside the (lower / upper) triangle, on the
// diagonal and beyond n; reciprocal diagonal (1 for unit and beyond n).
// Ends with __syncthreads.
template <class T, int NT, int RPL_REAL = 16>
__device__ __forceinline__ void leaf_stage(const typename St<T>::S* A, long lda, int n, bool swap,
                                           bool conj, bool lower, bool unit, double* sm) {
  using Sh = LeafShape<T, RPL_REAL>;
  constexpr bool CP = Sh::CPLX;
  double* Tr = sm;
  double* Ti = Tr + kLeafRows * Sh::COL;
  double* Dr = Ti + (CP ? kLeafRows * Sh::COL : 0);
  double* Di = Dr + kLeafRows;
  // element e -> (a0, a1) = (e % 64, e / 64) at A[a0 + a1 lda]: consecutive
  // threads read consecutive addresses for op(T) = A's triangle or its
  // transpose; loads are issued in groups of 8 before their stores
  constexpr int PER = kLeafRows * kLeafRows / NT;
  constexpr int GRP = PER < 8 ? PER : 8;
  static_assert(PER % GRP == 0, "staging split");
#pragma unroll
  for (int k0 = 0; k0 < PER; k0 += GRP) {
    double vr[GRP], vi[GRP];
#pragma unroll
    for (int k = 0; k < GRP; ++k) {
      const int e = threadIdx.x + (k0 + k) * NT;
      const int a0 = e & (kLeafRows - 1), a1 = e / kLeafRows;
      const int i = swap ? a1 : a0, j = swap ? a0 : a1;
      vr[k] = vi[k] = 0.0;
      if (i < n && j < n && (lower ? (j < i) : (j > i))) {
        const size_t idx = (size_t)a0 + (size_t)a1 * (size_t)lda;
        if (CP) {
          vr[k] = (double)__ldcg(A + 2 * idx);
          vi[k] = (double)__ldcg(A + 2 * idx + 1);
        } else {
          vr[k] = (double)__ldcg(A + idx);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < GRP; ++k) {
      const int e = threadIdx.x + (k0 + k) * NT;
      const int a0 = e & (kLeafRows - 1), a1 = e / kLeafRows;
      const int i = swap ? a1 : a0, j = swap ? a0 : a1;
      const int o = j * Sh::COL + (i / Sh::RPL) * Sh::GS + (i % Sh::RPL);
      Tr[o] = vr[k];
      if (CP) Ti[o] = conj ? -vi[k] : vi[k];
    }
  }
  for (int i = threadIdx.x; i < kLeafRows; i += NT) {
    double dr = 1.0, di = 0.0;
    if (i < n && !unit) {
      const size_t idx = (size_t)i + (size_t)i * (size_t)lda;
      if (CP) {
        dr = (double)__ldcg(A + 2 * idx);
        di = (double)__ldcg(A + 2 * idx + 1);
        if (conj) di = -di;
      } else {
        dr = (double)__ldcg(A + idx);
      }
    }
    if (CP) {
      const double den = dr * dr + di * di;
      Dr[i] = dr / den;
      Di[i] = -di / den;
    } else {
      Dr[i] = 1.0 / dr;
    }
  }
  __syncthreads();
}

// Substitution core: right-hand sides c0 .. c1-1, unknown `row` of rhs `c`
// read by ld(row, c, re, im) (rows < n of live columns only; zero elsewhere)
// and written back by sto(row, c, re, im).  All NT threads take part (every
// warp runs the same number of passes).
template <class T, int NT, bool LOWER, int RPL_REAL, class Ld, class Sto>
__device__ __forceinline__ void leaf_solve_core(int n, int c0, int c1, const double* sm, Ld ld,
                                                Sto sto) {
  using Sh = LeafShape<T, RPL_REAL>;
  constexpr int RPL = Sh::RPL, G = Sh::G, GS = Sh::GS, COL = Sh::COL;
  constexpr int CPP = NT / G;  // right-hand sides per pass
  constexpr bool CP = Sh::CPLX;
  const double* Tr = sm;
  const double* Ti = Tr + kLeafRows * COL;
  const double* Dr = Ti + (CP ? kLeafRows * COL : 0);
  const double* Di = Dr + kLeafRows;
  const int tid = threadIdx.x, lane = tid & 31;
  const int q = tid % G, gbase = lane & ~(G - 1);
  const int passes = (c1 - c0 + CPP - 1) / CPP;
  for (int p = 0; p < passes; ++p) {
    const int c = c0 + p * CPP + tid / G;
    const bool live = c < c1;
    double xr[RPL], xi[RPL];
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = q * RPL + r;
      xr[r] = xi[r] = 0.0;
      if (row < n && live) ld(row, c, xr[r], xi[r]);
    }
    // steps in G rounds of RPL: the register index is a compile-time constant
    // within a round, the owning lane a run-time one
#pragma unroll 1
    for (int og = 0; og < G; ++og) {
#pragma unroll
      for (int ss = 0; ss < RPL; ++ss) {
        const int oq = LOWER ? og : G - 1 - og, oi = LOWER ? ss : RPL - 1 - ss;
        const int i = oq * RPL + oi;
        double vr = __shfl_sync(0xffffffffu, xr[oi], gbase | oq);
        double vi = CP ? __shfl_sync(0xffffffffu, xi[oi], gbase | oq) : 0.0;
        if (CP) {
          const double dr = Dr[i], di = Di[i];
          const double wr = vr * dr - vi * di;
          vi = vr * di + vi * dr;
          vr = wr;
        } else {
          vr *= Dr[i];
        }
        if (q == oq) {
          xr[oi] = vr;
          if (CP) xi[oi] = vi;
        }
        // update row > i (lower) / row < i (upper): the staged column holds
        // zeros outside the triangle, but the predicate keeps final rows
        // untouched even when v is not finite
        const double2* colr = reinterpret_cast<const double2*>(Tr + i * COL + q * GS);
        const double2* coli = reinterpret_cast<const double2*>(Ti + i * COL + q * GS);
#pragma unroll
        for (int h = 0; h < RPL / 2; ++h) {
          const double2 tr = colr[h];
          double2 ti = make_double2(0.0, 0.0);
          if (CP) ti = coli[h];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int r = 2 * h + u;
            const int row = q * RPL + r;
            const double a = u ? tr.y : tr.x;
            if (LOWER ? row > i : row < i) {
              if (CP) {
                const double b = u ? ti.y : ti.x;
                xr[r] -= a * vr - b * vi;
                xi[r] -= a * vi + b * vr;
              } else {
                xr[r] -= a * vr;
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = q * RPL + r;
      if (row < n && live) sto(row, c, xr[r], xi[r]);
    }
  }
}

// Solve right-hand sides c0 .. c1-1 of B in place (alpha applied on load).
template <class T, int NT, bool LOWER, int RPL_REAL = 16>
__device__ __forceinline__ void leaf_solve(typename St<T>::S* B, long ldb, bool rhs_rows, int n,
                                           int c0, int c1, double ar, double ai,
                                           const double* sm) {
  constexpr bool CP = St<T>::CPLX;
  using S = typename St<T>::S;
  leaf_solve_core<T, NT, LOWER, RPL_REAL>(
      n, c0, c1, sm,
      [&](int row, int c, double& xr, double& xi) {
        const size_t idx = leaf_at(row, c, ldb, rhs_rows);
        const double br = CP ? (double)__ldcg(B + 2 * idx) : (double)__ldcg(B + idx);
        const double bi = CP ? (double)__ldcg(B + 2 * idx + 1) : 0.0;
        xr = ar * br - ai * bi;
        if (CP) xi = ar * bi + ai * br;
      },
      [&](int row, int c, double xr, double xi) {
        const size_t idx = leaf_at(row, c, ldb, rhs_rows);
        if (CP) {
          B[2 * idx] = static_cast<S>(xr);
          B[2 * idx + 1] = static_cast<S>(xi);
        } else {
          B[idx] = static_cast<S>(xr);
        }
      });
}

}  // namespace xkb
