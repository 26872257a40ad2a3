// gemm_dmma.cu -- the plain FP64 tile GEMM for sm_100a.
//
// Replaces the reference's per-tile cuBLAS bodies (blas/ztask_gemm.c:176-216,
// cublasZgemm at :206; the triangle-masked variants used for gemmt / syrk /
// herk / syr2k / her2k diagonal tiles, ztask_gemmt.c:213, ztask_syrk.c:130,
// ztask_herk.c:130).  One launch covers the whole matrix instead of one
// NB x NB tile per task.
//
// Design (B200):
//   * TMA 2-D tile loads (cp.async.bulk.tensor) fill a 4-stage shared-memory
//     ring guarded by mbarriers (full: transaction bytes, empty: one arrive
//     per warp); eight warps run FP64 DMMA tensor-core MMAs (mma.sync
//     m16n8k8 f64), thread 0 also refilling each stage once it is released;
//   * operands of any storage type (s/d/c/z) are loaded as raw tiles and
//     widened to double when fragments are read, so every precision computes
//     in FP64 and rounds once on store; complex products are four real MMAs;
//   * the k index inside each 8-wide MMA step is permuted (logical t+4v <->
//     physical 2t+v) identically for A and B, so each lane's two k values
//     are adjacent in shared memory;
//   * alpha/beta, the triangle mask and the Hermitian real-diagonal rule are
//     applied in the register epilogue; tiles wholly outside the triangle
//     exit before touching memory;
//   * every barrier wait is bounded (xkb_dev.cuh) and records an error word.
#include <cstdio>
#include <cstdlib>

#include <algorithm>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {

struct GemmParams {
  int M, N, K;
  void* C;
  long ldc;
  double ar, ai, br, bi;
  int uplo, herm_diag;
  long diag;
  int conjA, conjB;
  int tiles_m, tiles_n, ktiles;
  const int* run_if;  // not null: the launch does nothing unless *run_if != 0
  // split-K: the k-tiles of every C tile are shared by ksplit CTAs, slice s
  // taking [s kt_slice, (s+1) kt_slice); each writes its raw accumulators to
  // ws and k_gemm_splitk sums the slices in order and runs the epilogue
  int ksplit, kt_slice;
  double* ws;
  // stream-K (k_gemm_dmma_sk): the ntiles x ktiles k-tiles, tile-major, are
  // dealt out evenly to sk_ctas CTAs; a tile's pieces land in ws slots
  // [tile][0 .. sk_slots) in CTA order
  int sk_ctas, sk_slots;
};

// The stream-K CTA whose share of the k-tile sequence holds k-tile g (of
// total T over G CTAs; CTA c holds [c T / G, (c+1) T / G)).
__host__ __device__ __forceinline__ int sk_cta(long g, long T, int G) {
  int c = (int)(g * G / T);
  while (c + 1 < G && (long)(c + 1) * T / G <= g) ++c;
  while (c > 0 && (long)c * T / G > g) --c;
  return c;
}

// Tile of CTA `bid` (< tiles_m tiles_n) in the grouped rasterisation: 8 tile
// rows share a band of B columns in L2.  False if it lies wholly outside the
// triangle mask (nothing to do).
template <int BM, int BN>
__device__ __forceinline__ bool dmma_tile(const GemmParams& p, int bid, int& m0, int& n0) {
  const int GROUP = 8;
  const int span = GROUP * p.tiles_n;
  const int first_m = (bid / span) * GROUP;
  const int gsz = min(p.tiles_m - first_m, GROUP);
  const int tm = first_m + (bid % span) % gsz;
  const int tn = (bid % span) / gsz;
  m0 = tm * BM;
  n0 = tn * BN;
  if (p.uplo == XKB_LOWER && (long)(m0 + BM - 1) + p.diag < (long)n0) return false;
  if (p.uplo == XKB_UPPER && (long)m0 + p.diag > (long)(n0 + BN - 1)) return false;
  return true;
}

// Register layout of a consumer warp's accumulators (2 x 4 warps).
template <class T, int BM, int BN>
struct AccShape {
  static constexpr int WTM = BM / 2, WTN = BN / 4;
  static constexpr int MF = WTM / 16, NF = WTN / 8;
  static constexpr int NACC = St<T>::CPLX ? 8 : 4;
  static constexpr int NREG = MF * NF * NACC;
};

// Element i (0..3) of fragment (mf, nf) of this thread: its row and column
// of C; false if outside C or the triangle mask.
template <class T, int BM, int BN>
__device__ __forceinline__ bool dmma_elem(const GemmParams& p, int m0, int n0, int mf, int nf,
                                          int i, int& row, int& col) {
  using A = AccShape<T, BM, BN>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, t = lane & 3;
  row = m0 + wm * A::WTM + mf * 16 + g + ((i >> 1) << 3);
  col = n0 + wn * A::WTN + nf * 8 + 2 * t + (i & 1);
  return row < p.M && col < p.N && in_mask(p.uplo, p.diag, row, col);
}

// The C values of fragment (mf, nf) that beta multiplies (cv[i], imaginary
// parts at cv[4 + i]; 0 where nothing is stored).  The epilogue loads a
// whole row of fragments before it stores any: C is read and written
// through one pointer, so a load placed after a store could not be issued
// before that store completes.
template <class T, int BM, int BN>
__device__ __forceinline__ void dmma_load_frag(const GemmParams& p, int m0, int n0, int mf,
                                               int nf, double* cv) {
  using S = typename St<T>::S;
  constexpr bool CPLX = St<T>::CPLX;
  const S* C = reinterpret_cast<const S*>(p.C);
  const bool use_beta = (p.br != 0.0) || (p.bi != 0.0);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int row, col;
    cv[i] = 0.0;
    if (CPLX) cv[4 + i] = 0.0;
    if (!use_beta || !dmma_elem<T, BM, BN>(p, m0, n0, mf, nf, i, row, col)) continue;
    const size_t idx = (size_t)row + (size_t)col * (size_t)p.ldc;
    if constexpr (CPLX) {
      cv[i] = (double)C[2 * idx];
      cv[4 + i] = (double)C[2 * idx + 1];
    } else {
      cv[i] = (double)C[idx];
    }
  }
}

// alpha/beta, mask, Hermitian diagonal, store of the fragment (mf, nf) of
// one thread's accumulators (a: its NACC registers; cv: from dmma_load_frag).
template <class T, int BM, int BN>
__device__ __forceinline__ void dmma_store_frag(const GemmParams& p, int m0, int n0, int mf,
                                                int nf, const double* a, const double* cv) {
  using S = typename St<T>::S;
  constexpr bool CPLX = St<T>::CPLX;
  S* C = reinterpret_cast<S*>(p.C);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int row, col;
    if (!dmma_elem<T, BM, BN>(p, m0, n0, mf, nf, i, row, col)) continue;
    const size_t idx = (size_t)row + (size_t)col * (size_t)p.ldc;
    if constexpr (CPLX) {
      const double xr = a[i], xi = a[4 + i];
      double vr = p.ar * xr - p.ai * xi;
      double vi = p.ar * xi + p.ai * xr;
      vr += p.br * cv[i] - p.bi * cv[4 + i];
      vi += p.br * cv[4 + i] + p.bi * cv[i];
      if (p.herm_diag && (long)row + p.diag == (long)col) vi = 0.0;
      C[2 * idx] = static_cast<S>(vr);
      C[2 * idx + 1] = static_cast<S>(vi);
    } else {
      C[idx] = static_cast<S>(fma(p.br, cv[i], p.ar * a[i]));
    }
  }
}

// alpha/beta, mask, Hermitian diagonal, store of one thread's accumulators,
// one row of fragments at a time: all of the row's loads, then its stores.
template <class T, int BM, int BN>
__device__ __forceinline__ void dmma_epilogue(const GemmParams& p, int m0, int n0,
                                              const double* acc) {
  using A = AccShape<T, BM, BN>;
#pragma unroll
  for (int mf = 0; mf < A::MF; ++mf) {
    double cv[A::NF][A::NACC];
#pragma unroll
    for (int nf = 0; nf < A::NF; ++nf) dmma_load_frag<T, BM, BN>(p, m0, n0, mf, nf, cv[nf]);
#pragma unroll
    for (int nf = 0; nf < A::NF; ++nf)
      dmma_store_frag<T, BM, BN>(p, m0, n0, mf, nf, acc + (mf * A::NF + nf) * A::NACC, cv[nf]);
  }
}

constexpr int kBK = 16;      // k extent of one pipeline stage
constexpr int kStages = 4;
constexpr int kConsumerWarps = 8;
constexpr int kThreads = kConsumerWarps * 32;

// One 16-deep k stage of a consumer warp: DMMAs of its fragments of A (in
// shared memory at `st`) and B (after A's BM x kBK tile) into acc.
template <class T, int BM, int BN, bool A_KC, bool B_KC>
__device__ __forceinline__ void dmma_stage(const uint8_t* st,
                                           double (&acc)[BM / 32][BN / 32][St<T>::CPLX ? 8 : 4],
                                           int wm, int wn, int g, int t, double sgnA,
                                           double sgnB) {
  using S = typename St<T>::S;
  constexpr bool CPLX = St<T>::CPLX;
  constexpr int WTM = BM / 2, WTN = BN / 4;
  constexpr int MF = WTM / 16, NF = WTN / 8;
  const S* sa = reinterpret_cast<const S*>(st);
  const S* sb = reinterpret_cast<const S*>(st + BM * kBK * sizeof(T));
#pragma unroll
  for (int kc = 0; kc < kBK / 8; ++kc) {
    const int k0 = kc * 8 + 2 * t, k1 = k0 + 1;
    double br[NF][2], bi[NF][2];
#pragma unroll
    for (int nf = 0; nf < NF; ++nf) {
      const int n = wn * WTN + nf * 8 + g;
      const int o0 = B_KC ? n * kBK + k0 : k0 * BN + n;
      const int o1 = B_KC ? n * kBK + k1 : k1 * BN + n;
      ld_elem<T>(sb, o0, br[nf][0], bi[nf][0]);
      ld_elem<T>(sb, o1, br[nf][1], bi[nf][1]);
      if (CPLX) {
        bi[nf][0] *= sgnB;
        bi[nf][1] *= sgnB;
      }
    }
#pragma unroll
    for (int mf = 0; mf < MF; ++mf) {
      const int r0 = wm * WTM + mf * 16 + g, r1 = r0 + 8;
      double ar[4], ai[4];
      ld_elem<T>(sa, A_KC ? r0 * kBK + k0 : k0 * BM + r0, ar[0], ai[0]);
      ld_elem<T>(sa, A_KC ? r1 * kBK + k0 : k0 * BM + r1, ar[1], ai[1]);
      ld_elem<T>(sa, A_KC ? r0 * kBK + k1 : k1 * BM + r0, ar[2], ai[2]);
      ld_elem<T>(sa, A_KC ? r1 * kBK + k1 : k1 * BM + r1, ar[3], ai[3]);
      if constexpr (CPLX) {
        double nai[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          ai[v] *= sgnA;
          nai[v] = -ai[v];
        }
#pragma unroll
        for (int nf = 0; nf < NF; ++nf) {
          double* a = acc[mf][nf];
          double (&re)[4] = *reinterpret_cast<double(*)[4]>(a);
          double (&im)[4] = *reinterpret_cast<double(*)[4]>(a + 4);
          dmma_k8(re, ar, br[nf]);
          dmma_k8(re, nai, bi[nf]);
          dmma_k8(im, ar, bi[nf]);
          dmma_k8(im, ai, br[nf]);
        }
      } else {
#pragma unroll
        for (int nf = 0; nf < NF; ++nf) {
          double (&d)[4] = *reinterpret_cast<double(*)[4]>(acc[mf][nf]);
          dmma_k8(d, ar, br[nf]);
        }
      }
    }
  }
}

// A_KC: op(A) != N, A tile stored [BM][BK] (k contiguous), else [BK][BM].
// B_KC: op(B) == N, B tile stored [BN][BK], else [BK][BN].
template <class T, int BM, int BN, bool A_KC, bool B_KC>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_dmma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const GemmParams p) {
  // a launch predicated on a device word (the Ozaki data rule's plain
  // fallback): every thread reads the same word, so the whole CTA leaves
  // before touching shared memory, barriers or C
  if (p.run_if && *p.run_if == 0) return;
  using S = typename St<T>::S;
  constexpr int W = St<T>::W;
  constexpr bool CPLX = St<T>::CPLX;
  constexpr int WTM = BM / 2, WTN = BN / 4;   // 2 x 4 consumer warps
  constexpr int MF = WTM / 16, NF = WTN / 8;
  constexpr uint32_t A_BYTES = BM * kBK * sizeof(T);
  constexpr uint32_t B_BYTES = BN * kBK * sizeof(T);
  constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr int NACC = CPLX ? 8 : 4;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* base =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * STAGE_BYTES);
  uint64_t* empty = full + kStages;

  const int ntiles = p.tiles_m * p.tiles_n;
  const int slice = (int)blockIdx.x / ntiles;  // 0 unless split-K
  const int bid = (int)blockIdx.x - slice * ntiles;
  int m0, n0;
  if (!dmma_tile<BM, BN>(p, bid, m0, n0)) return;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // this CTA's k-tiles: [kt0, kt0 + KT)
  const int kt0 = slice * p.kt_slice;
  const int KT = p.ksplit > 1 ? max(0, min(p.ktiles - kt0, p.kt_slice)) : p.ktiles;
  // Thread 0 also drives the TMA ring: it fills every stage up front and
  // refills stage s once all eight warps have released it.
  auto issue = [&](int it) {
    const int s = it % kStages;
    uint8_t* sa = base + s * STAGE_BYTES;
    uint8_t* sb = sa + A_BYTES;
    mbar_expect_tx(&full[s], STAGE_BYTES);
    const int k0 = (kt0 + it) * kBK;
    if (A_KC) tma_load_2d(sa, &tmA, k0 * W, m0, &full[s]);
    else tma_load_2d(sa, &tmA, m0 * W, k0, &full[s]);
    if (B_KC) tma_load_2d(sb, &tmB, k0 * W, n0, &full[s]);
    else tma_load_2d(sb, &tmB, n0 * W, k0, &full[s]);
  };
  if (threadIdx.x == 0) {
    tma_prefetch(&tmA);
    tma_prefetch(&tmB);
    for (int it = 0; it < kStages && it < KT; ++it) issue(it);
  }

  // ---------------- consumers: DMMA over the stage ring --------------------
  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, t = lane & 3;
  double acc[MF][NF][NACC];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int v = 0; v < NACC; ++v) acc[i][j][v] = 0.0;

  const double sgnA = p.conjA ? -1.0 : 1.0;
  const double sgnB = p.conjB ? -1.0 : 1.0;
  bool ok = true;
  for (int it = 0; it < KT; ++it) {
    const int s = it % kStages;
    const uint32_t ph = (it / kStages) & 1;
    // every lane observes the phase itself (acquire of the TMA bytes); the
    // vote reconverges the warp before the .aligned MMAs
    const bool got = mbar_wait(&full[s], ph, kErrFullWait);
    if (!__all_sync(0xffffffffu, got)) {
      ok = false;
      break;
    }
    const S* sa = reinterpret_cast<const S*>(base + s * STAGE_BYTES);
    const S* sb = reinterpret_cast<const S*>(base + s * STAGE_BYTES + A_BYTES);
#pragma unroll
    for (int kc = 0; kc < kBK / 8; ++kc) {
      const int k0 = kc * 8 + 2 * t, k1 = k0 + 1;
      double br[NF][2], bi[NF][2];
#pragma unroll
      for (int nf = 0; nf < NF; ++nf) {
        const int n = wn * WTN + nf * 8 + g;
        const int o0 = B_KC ? n * kBK + k0 : k0 * BN + n;
        const int o1 = B_KC ? n * kBK + k1 : k1 * BN + n;
        ld_elem<T>(sb, o0, br[nf][0], bi[nf][0]);
        ld_elem<T>(sb, o1, br[nf][1], bi[nf][1]);
        if (CPLX) {
          bi[nf][0] *= sgnB;
          bi[nf][1] *= sgnB;
        }
      }
#pragma unroll
      for (int mf = 0; mf < MF; ++mf) {
        const int r0 = wm * WTM + mf * 16 + g, r1 = r0 + 8;
        double ar[4], ai[4];
        ld_elem<T>(sa, A_KC ? r0 * kBK + k0 : k0 * BM + r0, ar[0], ai[0]);
        ld_elem<T>(sa, A_KC ? r1 * kBK + k0 : k0 * BM + r1, ar[1], ai[1]);
        ld_elem<T>(sa, A_KC ? r0 * kBK + k1 : k1 * BM + r0, ar[2], ai[2]);
        ld_elem<T>(sa, A_KC ? r1 * kBK + k1 : k1 * BM + r1, ar[3], ai[3]);
        if constexpr (CPLX) {
          double nai[4];
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            ai[v] *= sgnA;
            nai[v] = -ai[v];
          }
#pragma unroll
          for (int nf = 0; nf < NF; ++nf) {
            double* a = acc[mf][nf];
            double (&re)[4] = *reinterpret_cast<double(*)[4]>(a);
            double (&im)[4] = *reinterpret_cast<double(*)[4]>(a + 4);
            dmma_k8(re, ar, br[nf]);
            dmma_k8(re, nai, bi[nf]);
            dmma_k8(im, ar, bi[nf]);
            dmma_k8(im, ai, br[nf]);
          }
        } else {
#pragma unroll
          for (int nf = 0; nf < NF; ++nf) {
            double (&d)[4] = *reinterpret_cast<double(*)[4]>(acc[mf][nf]);
            dmma_k8(d, ar, br[nf]);
          }
        }
      }
    }
    // the stage was read through the generic proxy and will be rewritten by
    // TMA (async proxy): order the reads before the release of the stage
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (warp == 0) {
      // lane 0 refills the stage; the vote keeps warp 0 converged for the
      // next iteration's .aligned MMAs
      bool refill_ok = true;
      if (lane == 0 && it + kStages < KT) {
        refill_ok = mbar_wait(&empty[s], ph, kErrEmptyWait);
        if (refill_ok) issue(it + kStages);
      }
      if (!__all_sync(0xffffffffu, refill_ok)) {
        ok = false;
        break;
      }
    }
  }
  if (!ok) return;
  const double* accp = &acc[0][0][0];
  if (p.ksplit > 1) {
    // raw partial sums of this slice, register-major: for each register the
    // block's threads write consecutive doubles (coalesced)
    constexpr int NREG = AccShape<T, BM, BN>::NREG;
    double* w = p.ws + ((size_t)slice * ntiles + bid) * (size_t)(NREG * kThreads) + threadIdx.x;
#pragma unroll
    for (int r = 0; r < NREG; ++r) w[(size_t)r * kThreads] = accp[r];
    return;
  }
  dmma_epilogue<T, BM, BN>(p, m0, n0, accp);
}

// Stream-K form of k_gemm_dmma (real or complex, C full, 128x128 tiles):
// for shapes whose tiles leave SMs idle, every CTA takes an equal share of
// the tile-major sequence of (tile, k-tile) steps -- pieces of at most a few
// tiles -- with the TMA ring running on from one piece into the next; each
// piece's raw accumulators go to a workspace slot, and k_gemm_sk_reduce sums
// every tile's pieces in CTA order (deterministic) and runs the epilogue.
template <class T, int BM, int BN, bool A_KC, bool B_KC>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_dmma_sk(const __grid_constant__ CUtensorMap tmA,
                   const __grid_constant__ CUtensorMap tmB, const GemmParams p) {
  if (p.run_if && *p.run_if == 0) return;
  constexpr int W = St<T>::W;
  constexpr bool CPLX = St<T>::CPLX;
  constexpr int MF = BM / 32, NF = BN / 32;
  constexpr uint32_t A_BYTES = BM * kBK * sizeof(T);
  constexpr uint32_t B_BYTES = BN * kBK * sizeof(T);
  constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr int NACC = CPLX ? 8 : 4;
  constexpr int NREG = AccShape<T, BM, BN>::NREG;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* base =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * STAGE_BYTES);
  uint64_t* empty = full + kStages;

  const int kts = p.ktiles;
  const long tot = (long)p.tiles_m * p.tiles_n * kts;
  const int G = p.sk_ctas;
  const long g0 = (long)blockIdx.x * tot / G, g1 = (long)(blockIdx.x + 1) * tot / G;
  if (g0 >= g1) return;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // producer (thread 0): the next step gp of [g0, g1) into ring slot gi
  long gp = g0;
  uint32_t gi = 0;
  auto issue_next = [&]() {
    const int s = gi % kStages;
    uint8_t* sa = base + s * STAGE_BYTES;
    uint8_t* sb = sa + A_BYTES;
    int m0, n0;
    dmma_tile<BM, BN>(p, (int)(gp / kts), m0, n0);
    const int k0 = (int)(gp % kts) * kBK;
    mbar_expect_tx(&full[s], STAGE_BYTES);
    if (A_KC) tma_load_2d(sa, &tmA, k0 * W, m0, &full[s]);
    else tma_load_2d(sa, &tmA, m0 * W, k0, &full[s]);
    if (B_KC) tma_load_2d(sb, &tmB, k0 * W, n0, &full[s]);
    else tma_load_2d(sb, &tmB, n0 * W, k0, &full[s]);
    ++gi;
    ++gp;
  };
  if (threadIdx.x == 0) {
    tma_prefetch(&tmA);
    tma_prefetch(&tmB);
    for (int i = 0; i < kStages && gp < g1; ++i) issue_next();
  }

  const int wm = warp >> 2, wn = warp & 3;
  const int g = lane >> 2, t = lane & 3;
  const double sgnA = p.conjA ? -1.0 : 1.0;
  const double sgnB = p.conjB ? -1.0 : 1.0;
  uint32_t gc = 0;
  for (long gs = g0; gs < g1;) {
    const int tile = (int)(gs / kts);
    const long gend = (long)(tile + 1) * kts < g1 ? (long)(tile + 1) * kts : g1;
    const int KT = (int)(gend - gs);
    double acc[MF][NF][NACC];
#pragma unroll
    for (int i = 0; i < MF; ++i)
#pragma unroll
      for (int j = 0; j < NF; ++j)
#pragma unroll
        for (int v = 0; v < NACC; ++v) acc[i][j][v] = 0.0;
    bool ok = true;
    for (int it = 0; it < KT; ++it, ++gc) {
      const int s = gc % kStages;
      const uint32_t ph = (gc / kStages) & 1;
      const bool got = mbar_wait(&full[s], ph, kErrFullWait);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      dmma_stage<T, BM, BN, A_KC, B_KC>(base + s * STAGE_BYTES, acc, wm, wn, g, t, sgnA, sgnB);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (warp == 0) {
        bool refill_ok = true;
        if (lane == 0 && gp < g1) {
          refill_ok = mbar_wait(&empty[s], ph, kErrEmptyWait);
          if (refill_ok) issue_next();
        }
        if (!__all_sync(0xffffffffu, refill_ok)) {
          ok = false;
          break;
        }
      }
    }
    if (!ok) return;  // a bounded wait gave up (error word recorded)
    // this piece's slot: its CTA's position among the tile's CTAs
    const int slot = (int)blockIdx.x - sk_cta((long)tile * kts, tot, G);
    const double* accp = &acc[0][0][0];
    double* w = p.ws + ((size_t)tile * p.sk_slots + slot) * (size_t)(NREG * kThreads) + threadIdx.x;
#pragma unroll
    for (int r = 0; r < NREG; ++r) w[(size_t)r * kThreads] = accp[r];
    gs += KT;
  }
}

// Sum of n partial-sum slots (slot q at w0 + q * stride, NACC values
// kThreads apart) in slot order, loaded four slots at a time so that one
// memory latency covers four slots (the order of the additions, and so the
// result, is that of a slot-by-slot loop).
template <int NACC>
__device__ __forceinline__ void sum_slots(const double* w0, size_t stride, int n,
                                          double (&acc)[NACC]) {
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.0;
  for (int s0 = 0; s0 < n; s0 += 4) {
    double wv[4][NACC];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int v = 0; v < NACC; ++v)
        wv[q][v] = s0 + q < n ? w0[(size_t)(s0 + q) * stride + (size_t)v * kThreads] : 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (s0 + q < n) {
#pragma unroll
        for (int v = 0; v < NACC; ++v) acc[v] += wv[q][v];
      }
  }
}

// Stream-K reduction: block (tile, fragment f) sums fragment f of the
// tile's pieces in CTA order, then stores it as the unsplit epilogue does.
template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads) k_gemm_sk_reduce(const GemmParams p) {
  if (p.run_if && *p.run_if == 0) return;
  using A = AccShape<T, BM, BN>;
  constexpr int NREG = A::NREG;
  const int kts = p.ktiles;
  const long tot = (long)p.tiles_m * p.tiles_n * kts;
  const int bid = blockIdx.x, f = blockIdx.y;
  int m0, n0;
  if (!dmma_tile<BM, BN>(p, bid, m0, n0)) return;
  const int c0 = sk_cta((long)bid * kts, tot, p.sk_ctas);
  const int c1 = sk_cta((long)(bid + 1) * kts - 1, tot, p.sk_ctas);
  double cv[A::NACC], acc[A::NACC];
  dmma_load_frag<T, BM, BN>(p, m0, n0, f / A::NF, f % A::NF, cv);  // in flight meanwhile
  const double* w0 = p.ws + (size_t)bid * p.sk_slots * (size_t)(NREG * kThreads) +
                     (size_t)(f * A::NACC) * kThreads + threadIdx.x;
  sum_slots<A::NACC>(w0, (size_t)NREG * kThreads, c1 - c0 + 1, acc);
  dmma_store_frag<T, BM, BN>(p, m0, n0, f / A::NF, f % A::NF, acc, cv);
}

// Split-K reduction: block (tile, fragment f) sums fragment f of the tile's
// slices in slice order (deterministic) with the GEMM kernel's
// thread-to-element map, then stores it as the unsplit epilogue does.  One
// block per (tile, fragment) spreads the reads of the slices over many SMs.
template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads) k_gemm_splitk(const GemmParams p) {
  if (p.run_if && *p.run_if == 0) return;
  using A = AccShape<T, BM, BN>;
  constexpr int NREG = A::NREG;
  const int ntiles = p.tiles_m * p.tiles_n;
  const int bid = blockIdx.x;
  const int f = blockIdx.y;  // fragment (mf, nf) = (f / NF, f % NF)
  int m0, n0;
  if (!dmma_tile<BM, BN>(p, bid, m0, n0)) return;
  double cv[A::NACC], acc[A::NACC];
  dmma_load_frag<T, BM, BN>(p, m0, n0, f / A::NF, f % A::NF, cv);  // in flight meanwhile
  const double* w0 =
      p.ws + (size_t)bid * (size_t)(NREG * kThreads) + (size_t)(f * A::NACC) * kThreads + threadIdx.x;
  sum_slots<A::NACC>(w0, (size_t)ntiles * NREG * kThreads, p.ksplit, acc);
  dmma_store_frag<T, BM, BN>(p, m0, n0, f / A::NF, f % A::NF, acc, cv);
}

// C <- beta*C on the masked part (beta == 0 writes zeros without reading).
template <class T>
__global__ void k_scale(int M, int N, double br, double bi, T* Cv, long ldc, int uplo,
                        int herm_diag, long diag) {
  using S = typename St<T>::S;
  S* C = reinterpret_cast<S*>(Cv);
  const size_t total = (size_t)M * (size_t)N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(e % (size_t)M), col = (int)(e / (size_t)M);
    if (!in_mask(uplo, diag, row, col)) continue;
    const size_t idx = (size_t)row + (size_t)col * (size_t)ldc;
    if constexpr (St<T>::CPLX) {
      double cr = 0, ci = 0;
      if (br != 0.0 || bi != 0.0) {
        const double xr = (double)C[2 * idx], xi = (double)C[2 * idx + 1];
        cr = br * xr - bi * xi;
        ci = br * xi + bi * xr;
      }
      if (herm_diag && (long)row + diag == (long)col) ci = 0.0;
      C[2 * idx] = (S)cr;
      C[2 * idx + 1] = (S)ci;
    } else {
      C[idx] = (br != 0.0) ? (S)(br * (double)C[idx]) : (S)0;
    }
  }
}

// ---------------------------------------------------------------------------
// host side
template <class T, int BM, int BN, bool A_KC, bool B_KC>
// ksplit > 1: split-K over that many slices; sk_ctas > 0: stream-K over
// that many CTAs (C full only).
static int launch_dmma(const xkb_gemm_args* a, cudaStream_t st, const int* run_if, int ksplit,
                       int sk_ctas = 0) {
  using S = typename St<T>::S;
  constexpr int W = St<T>::W;
  const int es = (int)sizeof(S);
  CUtensorMap tA, tB;
  // A stored (A_KC ? K x M : M x K), B stored (B_KC ? K x N : N x K)
  const uint64_t a_rows = A_KC ? a->K : a->M, a_cols = A_KC ? a->M : a->K;
  const uint64_t b_rows = B_KC ? a->K : a->N, b_cols = B_KC ? a->N : a->K;
  if (!encode_tmap_2d(&tA, St<T>::DT, es, a->A, a_rows * W, a_cols, (uint64_t)a->lda * W,
                      A_KC ? kBK * W : BM * W, A_KC ? BM : kBK, CU_TENSOR_MAP_SWIZZLE_NONE))
    return XKB_EINVAL;
  if (!encode_tmap_2d(&tB, St<T>::DT, es, a->B, b_rows * W, b_cols, (uint64_t)a->ldb * W,
                      B_KC ? kBK * W : BN * W, B_KC ? BN : kBK, CU_TENSOR_MAP_SWIZZLE_NONE))
    return XKB_EINVAL;
  GemmParams p;
  p.M = a->M;
  p.N = a->N;
  p.K = a->K;
  p.C = a->C;
  p.ldc = a->ldc;
  p.ar = a->alpha[0];
  p.ai = St<T>::CPLX ? a->alpha[1] : 0.0;
  p.br = a->beta[0];
  p.bi = St<T>::CPLX ? a->beta[1] : 0.0;
  p.uplo = a->uplo;
  p.herm_diag = a->herm_diag;
  p.diag = a->diag;
  p.conjA = (a->opA == XKB_OP_C);
  p.conjB = (a->opB == XKB_OP_C);
  p.tiles_m = (a->M + BM - 1) / BM;
  p.tiles_n = (a->N + BN - 1) / BN;
  p.ktiles = (a->K + kBK - 1) / kBK;
  p.run_if = run_if;
  p.ksplit = std::max(1, ksplit);
  p.kt_slice = (p.ktiles + p.ksplit - 1) / p.ksplit;
  p.ksplit = (p.ktiles + p.kt_slice - 1) / p.kt_slice;  // no empty slice
  p.ws = nullptr;
  p.sk_ctas = 0;
  p.sk_slots = 0;
  const size_t smem = kStages * (size_t)(BM + BN) * kBK * sizeof(T) + 2 * kStages * 8 + 128;
  if constexpr (BN == 128) {  // stream-K: the big tiles only
  if (sk_ctas > 0) {
    if (a->uplo != XKB_FULL) return XKB_EINVAL;
    const long ntiles = (long)p.tiles_m * p.tiles_n;
    const long tot = ntiles * p.ktiles;
    p.ksplit = 1;
    p.sk_ctas = (int)std::max<long>(1, std::min<long>(sk_ctas, tot));
    // a tile meets at most ceil(ktiles / shortest share) + 1 CTAs
    const long share = std::max<long>(1, tot / p.sk_ctas);
    p.sk_slots = (int)((p.ktiles + share - 1) / share + 1);
    auto kern = k_gemm_dmma_sk<T, BM, BN, A_KC, B_KC>;
    static bool sk_attr = false;  // one per instantiation
    if (!sk_attr) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return XKB_ECUDA;
      sk_attr = true;
    }
    const size_t ws =
        (size_t)ntiles * p.sk_slots * AccShape<T, BM, BN>::NREG * kThreads * sizeof(double);
    if (cudaMallocAsync(reinterpret_cast<void**>(&p.ws), ws, st) != cudaSuccess) {
      cudaGetLastError();
      return XKB_ENOMEM;
    }
    const long long tv = evlog_kern_begin(st, "k_gemm_dmma_sk+k_gemm_sk_reduce");
    kern<<<(unsigned)p.sk_ctas, kThreads, smem, st>>>(tA, tB, p);
    const dim3 rg((unsigned)ntiles, (unsigned)(AccShape<T, BM, BN>::MF * AccShape<T, BM, BN>::NF));
    k_gemm_sk_reduce<T, BM, BN><<<rg, kThreads, 0, st>>>(p);
    cudaFreeAsync(p.ws, st);
    evlog_kern_end(tv, st);
    count_launch(2);
    return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
  }
  }
  auto kern = k_gemm_dmma<T, BM, BN, A_KC, B_KC>;
  static bool attr_done = false;  // one per instantiation
  if (!attr_done) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return XKB_ECUDA;
    attr_done = true;
  }
  const long ntiles = (long)p.tiles_m * p.tiles_n;
  if (p.ksplit > 1) {
    const size_t ws = (size_t)p.ksplit * ntiles * AccShape<T, BM, BN>::NREG * kThreads * 8;
    if (cudaMallocAsync(reinterpret_cast<void**>(&p.ws), ws, st) != cudaSuccess) {
      cudaGetLastError();
      return XKB_ENOMEM;
    }
  }
  const long long tv = evlog_kern_begin(st, p.ksplit > 1 ? "k_gemm_dmma+k_gemm_splitk"
                                                         : "k_gemm_dmma");
  kern<<<(unsigned)(ntiles * p.ksplit), kThreads, smem, st>>>(tA, tB, p);
  if (p.ksplit > 1) {
    const dim3 rg((unsigned)ntiles, (unsigned)(AccShape<T, BM, BN>::MF * AccShape<T, BM, BN>::NF));
    k_gemm_splitk<T, BM, BN><<<rg, kThreads, 0, st>>>(p);
    cudaFreeAsync(p.ws, st);
  }
  evlog_kern_end(tv, st);
  count_launch(p.ksplit > 1 ? 2 : 1);
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

template <class T, int BM, int BN>
static int dispatch_ops(const xkb_gemm_args* a, cudaStream_t st, const int* run_if,
                        int ksplit = 1, int sk_ctas = 0) {
  const bool akc = a->opA != XKB_OP_N, bkc = a->opB == XKB_OP_N;
  if (akc && bkc) return launch_dmma<T, BM, BN, true, true>(a, st, run_if, ksplit, sk_ctas);
  if (akc && !bkc) return launch_dmma<T, BM, BN, true, false>(a, st, run_if, ksplit, sk_ctas);
  if (!akc && bkc) return launch_dmma<T, BM, BN, false, true>(a, st, run_if, ksplit, sk_ctas);
  return launch_dmma<T, BM, BN, false, false>(a, st, run_if, ksplit, sk_ctas);
}

// Split-K factor for big tiles when they alone leave SMs idle: as many
// slices as keep tiles x slices within one wave, each slice at least
// gemm_splitk_min_kt k-tiles (tuning key, default 16 = K 256); 1 = no split.
// Taken when even the small tiles cannot fill the SMs, or when every slice
// still runs gemm_splitk_long_kt k-tiles (default 16): measured on a B200,
// split-K 2 over 128x128 tiles beat the 64x64 tiles by 2.2x at
// 512x512x4096, 1.10x at 768x768x1536, 1.21x at 2048x512x2048, 1.16x at
// 1024^3 (92.5 vs 107.6 us; 32 k-tiles per slice) and 1.03x at
// 1024x1024x512 (16 k-tiles per slice).
static int splitk_factor(long tiles_big, long tiles_small, long ktiles) {
  const double on = tune("gemm_splitk", 1.0);
  if (on == 0.0 || tiles_big <= 0) return 1;
  const long sms = sm_count();
  const long min_kt = std::max(4L, (long)tune("gemm_splitk_min_kt", 16.0));
  long s = sms / tiles_big;
  s = std::min(s, ktiles / min_kt);
  s = std::max(1L, std::min(s, 32L));
  if (s > 1 && tiles_small >= sms && ktiles / s < (long)tune("gemm_splitk_long_kt", 16.0))
    return 1;
  return (int)s;
}

template <class T>
static int dispatch_type(const xkb_gemm_args* a, cudaStream_t st, const int* run_if) {
  constexpr bool CPLX = St<T>::CPLX;
  constexpr int BMb = CPLX ? 64 : 128, BNb = 128;
  const long tiles_big = (long)((a->M + BMb - 1) / BMb) * ((a->N + BNb - 1) / BNb);
  // XKBLAS_GEMM_TILE=big|small overrides the size rule (tuning sweeps); the
  // rule's threshold is the tuning table's gemm_big_min_tiles (default: more
  // big tiles than half the SMs).  Small tiles run two CTAs per SM at about
  // 0.68 of a big tile's time per SM-wave, so one wave of big tiles beats
  // them once it fills more than half the SMs (2048 x 1024 x 1024: 128 big
  // tiles 160 us, 512 small tiles 205 us); below that, split-K or the small
  // tiles.
  static const char* force = getenv("XKBLAS_GEMM_TILE");
  const bool big = force ? (force[0] == 'b')
                         : (tiles_big >= (long)tune("gemm_big_min_tiles",
                                                    (double)(sm_count() / 2 + 1)));
  if (big) return dispatch_ops<T, BMb, BNb>(a, st, run_if);
  // too few big tiles for the SMs: split their k range when K allows
  const long tiles_small =
      (long)((a->M + BMb / 2 - 1) / (BMb / 2)) * ((a->N + BNb / 2 - 1) / (BNb / 2));
  const long ktiles = (a->K + kBK - 1) / kBK;
  const int ks = force ? 1 : splitk_factor(tiles_big, tiles_small, ktiles);
  if (ks > 1) {
    // Stream-K instead when C is full (tuning key gemm_streamk, default 1)
    // and split-K's ks x tiles CTAs fill less than gemm_sk_fill (0.8) of the
    // SMs, or leave any SM idle while every tile has at least gemm_sk_long_kt
    // (64) k-steps: one CTA per SM, each with an equal share of the tiles'
    // k-steps (at least gemm_sk_min_kt of them).  Measured on a B200: 640 x
    // 1280 x 2048 (50 tiles, split-K 2 on 100 CTAs) 168 -> 136 us; 1024^3
    // (split-K 2 on 128 CTAs, 64 k-steps per tile) 97.8-98.9 -> 94.5-95.3 us
    // (alternating, same box); at 16-32 k-steps per tile and 86-97 % of the
    // SMs filled the two were within 5 % either way.
    const long min_kt = std::max(1L, (long)tune("gemm_sk_min_kt", 8.0));
    const long sk = std::min<long>(sm_count(), tiles_big * ktiles / min_kt);
    const double split_fill = (double)(tiles_big * ks) / (double)sm_count();
    if (a->uplo == XKB_FULL && tune("gemm_streamk", 1.0) != 0.0 && sk > tiles_big * ks &&
        (split_fill < tune("gemm_sk_fill", 0.8) ||
         (split_fill < 1.0 && ktiles >= (long)tune("gemm_sk_long_kt", 64.0))))
      return dispatch_ops<T, BMb, BNb>(a, st, run_if, 1, (int)sk);
    return dispatch_ops<T, BMb, BNb>(a, st, run_if, ks);
  }
  return dispatch_ops<T, BMb / 2, BNb / 2>(a, st, run_if);
}

// Copy a rows x cols column-major array (element size es) into a packed
// array with leading dimension ldd.  Used to give TMA a 16-byte aligned view
// of an operand whose base or leading dimension is not 16-byte aligned.
template <class W>
__global__ void k_repack(int rows_w, int cols, const W* __restrict__ src, long lds_w,
                         W* __restrict__ dst, long ldd_w, const int* run_if) {
  if (run_if && *run_if == 0) return;
  const size_t total = (size_t)rows_w * (size_t)cols;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e % (size_t)rows_w, j = e / (size_t)rows_w;
    dst[i + j * (size_t)ldd_w] = src[i + j * (size_t)lds_w];
  }
}

static bool tma_ok(const void* p, long ld, int es) {
  return reinterpret_cast<uintptr_t>(p) % 16 == 0 && ((size_t)ld * es) % 16 == 0;
}

// Packed copy of a stored operand (rows x cols, element size es); *out is a
// stream-ordered allocation the caller frees on the same stream.
static int repack(const void* src, long ld, int rows, int cols, int es, void** out, long* ldo,
                  cudaStream_t st, const int* run_if) {
  const long ldp = (long)(((size_t)rows * es + 15) / 16 * 16 / es);
  if (cudaMallocAsync(out, std::max<size_t>((size_t)ldp * cols * es, 16), st) != cudaSuccess)
    return XKB_ENOMEM;
  *ldo = ldp;
  const size_t total = (size_t)rows * cols;
  const unsigned grid = (unsigned)std::max<size_t>(
      1, std::min<size_t>((total + 255) / 256, (size_t)sm_count() * 16));
  const long long tv = evlog_kern_begin(st, "k_repack");
  if (es % 8 == 0 && reinterpret_cast<uintptr_t>(src) % 8 == 0)
    k_repack<double><<<grid, 256, 0, st>>>(rows * (es / 8), cols,
                                           static_cast<const double*>(src), ld * (es / 8),
                                           static_cast<double*>(*out), ldp * (es / 8), run_if);
  else
    k_repack<float><<<grid, 256, 0, st>>>(rows * (es / 4), cols, static_cast<const float*>(src),
                                          ld * (es / 4), static_cast<float*>(*out),
                                          ldp * (es / 4), run_if);
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

template <class T>
static int launch_scale(int M, int N, const double* beta, void* C, long ldc, int uplo,
                        int herm_diag, long diag, cudaStream_t st) {
  const size_t total = (size_t)M * (size_t)N;
  if (total == 0) return XKB_OK;
  long blocks = (long)((total + 255) / 256);
  if (blocks > 4L * sm_count() * 8) blocks = 4L * sm_count() * 8;
  const long long tv = evlog_kern_begin(st, "k_scale");
  k_scale<T><<<(unsigned)blocks, 256, 0, st>>>(M, N, beta[0], St<T>::CPLX ? beta[1] : 0.0,
                                               reinterpret_cast<T*>(C), ldc, uplo, herm_diag,
                                               diag);
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

}  // namespace xkb

using namespace xkb;

extern "C" int xkb_cuda_scale(int dtype, int M, int N, const double* beta, void* C, long ldc,
                              int uplo, int herm_diag, long diag, void* stream) {
  if (M < 0 || N < 0 || !beta) return XKB_EINVAL;
  if (M == 0 || N == 0) return XKB_OK;
  cudaStream_t st = resolve_stream(stream);
  switch (dtype) {
    case XKB_S: return launch_scale<float>(M, N, beta, C, ldc, uplo, herm_diag, diag, st);
    case XKB_D: return launch_scale<double>(M, N, beta, C, ldc, uplo, herm_diag, diag, st);
    case XKB_C: return launch_scale<float2>(M, N, beta, C, ldc, uplo, herm_diag, diag, st);
    case XKB_Z: return launch_scale<double2>(M, N, beta, C, ldc, uplo, herm_diag, diag, st);
  }
  return XKB_EINVAL;
}

namespace xkb {
// The whole-matrix product; run_if not null: the kernel runs only where the
// device word is non-zero (operand repacking, if any, runs regardless).
static int gemm_impl(const xkb_gemm_args* a, cudaStream_t st, const int* run_if) {
  if (!a || a->M < 0 || a->N < 0 || a->K < 0) return XKB_EINVAL;
  if (a->dtype < XKB_S || a->dtype > XKB_Z) return XKB_EINVAL;
  if (a->opA < XKB_OP_N || a->opA > XKB_OP_C || a->opB < XKB_OP_N || a->opB > XKB_OP_C)
    return XKB_EINVAL;
  if (a->M == 0 || a->N == 0) return XKB_OK;
  const bool cplx = (a->dtype == XKB_C || a->dtype == XKB_Z);
  const bool alpha_zero = a->alpha[0] == 0.0 && (!cplx || a->alpha[1] == 0.0);
  if (a->K == 0 || alpha_zero)
    return run_if ? XKB_EINVAL
                  : xkb_cuda_scale(a->dtype, a->M, a->N, a->beta, a->C, a->ldc, a->uplo,
                                   a->herm_diag, a->diag, st);
  const int slot = trace_begin(run_if ? "dmma_fallback" : "dmma_gemm", a->dtype, a->M, a->N,
                               a->K, 0, st);
  trace_mark(slot, 1, st);
  // the tensor-map loads need 16-byte aligned bases and leading dimensions:
  // other operands are first copied to packed, aligned arrays (C is read and
  // written with plain loads and stores, any alignment)
  const int es = (a->dtype == XKB_S) ? 4 : (a->dtype == XKB_Z ? 16 : 8);
  if (reinterpret_cast<uintptr_t>(a->A) % 4 || reinterpret_cast<uintptr_t>(a->B) % 4 ||
      reinterpret_cast<uintptr_t>(a->C) % 4)
    return XKB_EINVAL;
  xkb_gemm_args pa = *a;
  void* packA = nullptr;
  void* packB = nullptr;
  int r = XKB_OK;
  if (!tma_ok(a->A, a->lda, es))
    r = repack(a->A, a->lda, a->opA == XKB_OP_N ? a->M : a->K,
               a->opA == XKB_OP_N ? a->K : a->M, es, &packA, &pa.lda, st, run_if);
  if (r == XKB_OK && !tma_ok(a->B, a->ldb, es))
    r = repack(a->B, a->ldb, a->opB == XKB_OP_N ? a->K : a->N,
               a->opB == XKB_OP_N ? a->N : a->K, es, &packB, &pa.ldb, st, run_if);
  if (packA) pa.A = packA;
  if (packB) pa.B = packB;
  if (r == XKB_OK) {
    r = XKB_EINVAL;
    switch (a->dtype) {
      case XKB_S: r = dispatch_type<float>(&pa, st, run_if); break;
      case XKB_D: r = dispatch_type<double>(&pa, st, run_if); break;
      case XKB_C: r = dispatch_type<float2>(&pa, st, run_if); break;
      case XKB_Z: r = dispatch_type<double2>(&pa, st, run_if); break;
    }
  }
  if (packA) cudaFreeAsync(packA, st);
  if (packB) cudaFreeAsync(packB, st);
  trace_mark(slot, 2, st);
  trace_mark(slot, 3, st);
  return r;
}

int gemm_if(const xkb_gemm_args* a, const int* run_if, cudaStream_t st) {
  return gemm_impl(a, st, run_if);
}
}  // namespace xkb

extern "C" int xkb_cuda_gemm(const xkb_gemm_args* a, void* stream) {
  return gemm_impl(a, resolve_stream(stream), nullptr);
}
