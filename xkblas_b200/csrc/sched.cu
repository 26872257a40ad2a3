// sched.cu -- the tile-task executor: one persistent launch runs a whole
// batch of level-3 calls as a DAG of tile tasks.
//
// Replaces the reference's XKaapi machinery for this path: per-tile tasks
// (blas/ztask_gemm.c:107-158, ztask_trsm.c), their data-flow dependencies
// (kaapi/kaapi_task.c:1277-1327) and the device threads that pop ready tasks
// and launch one cuBLAS call each (kaapi/kaapi_offload_device.c:463-683,
// 852-1210).  The host builds the task graph once; persistent CTAs (as many
// as fit, two per SM) take dependency-free tasks from a bulk list and the
// others from a device-side ready queue that completing tasks append their
// successors to.  A batch of small, uneven calls thus costs one launch
// instead of one launch (or thousands of tile tasks with host round trips)
// per call.
//
// Task bodies (256 threads):
//   gemm     C[<=BM x <=BN] = alpha op(A) op(B) + beta C over the full K,
//            cp.async 3-stage shared-memory ring (16-byte copies, or 8-byte
//            L2 loads when a leading dimension is odd; zero fill at ragged
//            edges), DMMA m16n8k8; BM x BN = 64 x 64 (real), 32 x 64
//            (complex, four real MMAs per product);
//   trsm     one 64-row block X_i of a left triangular solve against up to
//            64 right-hand sides, left-looking: X_i = alpha B_i - sum_k
//            op(A)[i,k] X_k over the blocks already solved (one gemm tile
//            with the whole k range), then the diagonal solve with op(A)[i,i]
//            in the same CTA.  The reference runs the same block algorithm
//            right-looking (blas/ztrsm.c:241-372: diagonal trsm tasks, then
//            gemm updates of the trailing blocks); here each right-hand-side
//            block is one chain of mt tasks, and the sums are formed in
//            registers once instead of read-modified-written per step.
// Ordering rules: a producer stores, then __syncthreads, then thread 0
// issues __threadfence and decrements its successors' dependency counts;
// the consumer's thread 0 takes the queued task, issues __threadfence, and
// the CTA reads through L2 (cp.async.cg / ld.global.cg) -- no stale L1
// lines, no async-proxy reads.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "dmma_common.cuh"
#include "trsm_leaf.cuh"
#include "xkb_dev.cuh"

namespace xkb {
namespace sched {

enum : int { kTaskGemm = 0, kTaskTrsm = 1 };
// kFlagNarrow: an operand base or leading dimension is not 16-byte aligned,
// so the gemm tile stages it with 8-byte L2 loads instead of 16-byte copies
enum : int { kFlagSwap = 1, kFlagConj = 2, kFlagLower = 4, kFlagUnit = 8, kFlagNarrow = 16 };

// One task.  succ0 / nsucc: its successors in the batch's successor array
// (tasks whose dependency count it decrements when it completes).
//   gemm:  C = (ar,ai) op(A) op(B) + (br,bi) C, C is M x N, inner K.
//   trsm:  C = X_i (M rows, N right-hand sides); A, B = the op(A) panel and
//          the solved X rows it multiplies (K = their inner length, 0 for
//          the first block); D = the diagonal block; (ar,ai) = alpha.
struct alignas(16) Task {
  int kind, dtype, opA, opB;
  int M, N, K, call;
  const void* A;
  const void* B;
  void* C;
  const void* D;
  long lda, ldb, ldc;
  double ar, ai, br, bi;
  int succ0, nsucc, flags, pad;
};
static_assert(sizeof(Task) == 144, "task record");

// Device-side queues of one batch (ints in global memory):
//   bulk[nbulk]   tasks without dependencies (gemm tiles of gemm calls), in
//                 call order; claimed with an atomic head;
//   urq[nurg]     the solve tasks: a ready queue.  The first block of every
//                 chain is queued at launch; a task is appended (atomic
//                 tail, then the slot is written) when its last dependency
//                 completes; slots not yet written hold -1.  A CTA takes a
//                 ticket (atomic head) only while the queue shows a task it
//                 could get, then waits for its slot: one atomic per claim,
//                 no retry storms, and no deadlock (slots fill in order and
//                 every queued task's producers were queued before it).
struct Ctl {
  int head_bulk, head_urg, tail_urg, pad;
};

constexpr int kThreads = 256;
constexpr int kBK = 16;
constexpr int kSt = 3;      // cp.async stages
constexpr int kLeafS = kLeafRows;  // trsm block (trsm_leaf.cuh)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)),
               "l"(gmem), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

// Claim the next task for this CTA (thread 0 only): from the ready queue of
// the solves or from the bulk list, in the order `urgent_first` asks.  Spins
// (bounded) while every remaining task still waits for a dependency.
// Returns the task id, -1 when every task has been claimed, -2 on timeout or
// when another CTA recorded an error.
__device__ __forceinline__ int claim_task(Ctl* ctl, const int* bulk, int nbulk, const int* urq,
                                          int nurg, bool urgent_first, uint64_t wait_ns) {
  uint64_t t0 = 0;
  for (uint32_t spin = 0;; ++spin) {
    for (int pass = 0; pass < 2; ++pass) {
      if ((pass == 0) == urgent_first) {
        const int h = ld_volatile(&ctl->head_urg);
        if (h < nurg && ld_volatile(&ctl->tail_urg) > h) {
          const int tk = atomicAdd(&ctl->head_urg, 1);
          if (tk < nurg) {  // the slot fills once its task is queued
            uint64_t w0 = 0;
            for (uint32_t k = 0;; ++k) {
              const int t = ld_volatile(urq + tk);
              if (t >= 0) return t;
              __nanosleep(64);
              if ((k & 63u) == 0) {
                if (dev_error_set()) return -2;
                const uint64_t now = globaltimer();
                if (w0 == 0) w0 = now;
                else if (now - w0 > wait_ns) {
                  dev_error(kErrFullWait);
                  return -2;
                }
              }
            }
          }
        }
      } else if (ld_volatile(&ctl->head_bulk) < nbulk) {
        const int b = atomicAdd(&ctl->head_bulk, 1);
        if (b < nbulk) return bulk[b];
      }
    }
    if (ld_volatile(&ctl->head_bulk) >= nbulk && ld_volatile(&ctl->head_urg) >= nurg) return -1;
    __nanosleep(256);
    if ((spin & 31u) == 0) {
      if (dev_error_set()) return -2;
      const uint64_t now = globaltimer();
      if (t0 == 0) t0 = now;
      else if (now - t0 > wait_ns) {
        dev_error(kErrFullWait);
        return -2;
      }
    }
  }
}

// ---- gemm tile ---------------------------------------------------------------
// Shared layout of a stage: op(A) as BM x kBK, op(B) as kBK x BN, each in the
// orientation of its global storage so that 16-byte copies run along the
// contiguous dimension.  "KC" = k contiguous (row m of op(A) / column n of
// op(B) holds kBK consecutive k).  Real tiles are padded: KC rows by 8
// doubles (a lane's k-pair is one 16-byte load, conflict-free across the
// eight lanes of a phase), the other orientation by 2 (the 16 lanes of a
// phase hit 16 distinct 8-byte bank pairs).  Warp grid: real 64 x 64 tiles
// 2 x 4 warps (32 x 16 each), real 128 x 64 tiles 4 x 2 (32 x 32), complex
// 32 x 64 tiles 2 x 4 (16 x 16).
template <class T, bool A_KC, bool B_KC, int BM>
struct TileShape {
  static constexpr bool CPLX = St<T>::CPLX;
  static constexpr int BN = 64;
  static constexpr int WM = BM == 128 ? 4 : 2, WN = kThreads / 32 / WM;
  static constexpr int WTM = BM / WM, WTN = BN / WN;
  static constexpr int MF = WTM / 16, NF = WTN / 8;
  static constexpr int PKC = CPLX ? 0 : 8, PMN = CPLX ? 0 : 2;
  static constexpr int LDA = A_KC ? kBK + PKC : BM + PMN;  // smem stride (elements)
  static constexpr int LDB = B_KC ? kBK + PKC : BN + PMN;
  static constexpr int A_S = A_KC ? BM * LDA : kBK * LDA;  // smem elements per stage
  static constexpr int B_S = B_KC ? BN * LDB : kBK * LDB;
  static constexpr int ES = (int)sizeof(T);
  static constexpr int STAGE_BYTES = (A_S + B_S) * ES;
};

// Staging modes: kCopy16 16-byte cp.async.cg copies (aligned operands);
// kCopy8 8-byte cp.async.ca copies (an operand not 16-byte aligned, operands
// not written while the batch runs: L1 may keep them); kLoad8 8-byte L2 loads
// through registers, one stage ahead (not 16-byte aligned, and B holds rows
// other CTAs solved during this launch).
enum : int { kCopy16 = 0, kCopy8 = 1, kLoad8 = 2 };

// not inlined: each instantiation keeps its own register allocation
template <class T, bool A_KC, bool B_KC, int BM, int MODE>
__device__ __noinline__ void gemm_tile(const Task& t, uint8_t* smem) {
  using Sh = TileShape<T, A_KC, B_KC, BM>;
  using S = typename St<T>::S;
  constexpr bool CPLX = Sh::CPLX;
  constexpr int BN = Sh::BN, WTM = Sh::WTM, WTN = Sh::WTN, MF = Sh::MF, NF = Sh::NF;
  constexpr int LDA = Sh::LDA, LDB = Sh::LDB, ES = Sh::ES;
  constexpr int EPC = 16 / ES;  // elements per 16-byte chunk
  constexpr int A_ELEMS = BM * kBK, B_ELEMS = BN * kBK;
  constexpr int STAGE_BYTES = Sh::STAGE_BYTES;
  constexpr int NACC = CPLX ? 8 : 4;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const char* Ag = static_cast<const char*>(t.A);
  const char* Bg = static_cast<const char*>(t.B);
  const int M = t.M, N = t.N, K = t.K;
  const int KT = (K + kBK - 1) / kBK;
  // shared offset (elements) of op(A)(m, k) / op(B)(k, n)
  auto a_off = [](int m, int k) { return A_KC ? m * LDA + k : k * LDA + m; };
  auto b_off = [](int k, int n) { return B_KC ? n * LDB + k : k * LDB + n; };

  // cp.async paths: 16-byte chunks (kCopy16) or 8-byte words (kCopy8)
  auto load_stage = [&](int it, int buf) {
    uint8_t* sa = smem + buf * STAGE_BYTES;
    uint8_t* sb = sa + Sh::A_S * ES;
    const int k0 = it * kBK;
    if constexpr (MODE == kCopy8) {
      constexpr int W = ES / 8;  // words per element
      for (int w = tid; w < A_ELEMS * W; w += kThreads) {
        const int e = w / W, h = w % W;
        const int mm = A_KC ? e / kBK : e % BM, kk = A_KC ? e % kBK : e / BM;
        const int gk = k0 + kk;
        const bool v = mm < M && gk < K;
        const size_t gi =
            A_KC ? (size_t)gk + (size_t)mm * t.lda : (size_t)mm + (size_t)gk * t.lda;
        cp_async8(sa + a_off(mm, kk) * ES + h * 8, v ? Ag + gi * ES + h * 8 : Ag, v ? 8 : 0);
      }
      for (int w = tid; w < B_ELEMS * W; w += kThreads) {
        const int e = w / W, h = w % W;
        const int nn = B_KC ? e / kBK : e % BN, kk = B_KC ? e % kBK : e / BN;
        const int gk = k0 + kk;
        const bool v = nn < N && gk < K;
        const size_t gi =
            B_KC ? (size_t)gk + (size_t)nn * t.ldb : (size_t)nn + (size_t)gk * t.ldb;
        cp_async8(sb + b_off(kk, nn) * ES + h * 8, v ? Bg + gi * ES + h * 8 : Bg, v ? 8 : 0);
      }
      return;
    }
    constexpr int A_CH = A_ELEMS / EPC;
    for (int c = tid; c < A_CH; c += kThreads) {
      int mm, kk;  // first element of the chunk
      if (A_KC) {
        mm = c / (kBK / EPC);
        kk = (c % (kBK / EPC)) * EPC;
      } else {
        kk = c / (BM / EPC);
        mm = (c % (BM / EPC)) * EPC;
      }
      const int gk = k0 + kk;
      int valid;
      const char* src;
      if (A_KC) {  // element (m,k) at A[k + m*lda]; chunk runs along k
        valid = (mm < M) ? max(0, min(EPC, K - gk)) : 0;
        src = Ag + ((size_t)gk + (size_t)mm * t.lda) * ES;
      } else {     // element (m,k) at A[m + k*lda]; chunk runs along m
        valid = (gk < K) ? max(0, min(EPC, M - mm)) : 0;
        src = Ag + ((size_t)mm + (size_t)gk * t.lda) * ES;
      }
      cp_async16(sa + a_off(mm, kk) * ES, valid ? src : Ag, valid * ES);
    }
    constexpr int B_CH = B_ELEMS / EPC;
    for (int c = tid; c < B_CH; c += kThreads) {
      int nn, kk;
      if (B_KC) {
        nn = c / (kBK / EPC);
        kk = (c % (kBK / EPC)) * EPC;
      } else {
        kk = c / (BN / EPC);
        nn = (c % (BN / EPC)) * EPC;
      }
      const int gk = k0 + kk;
      int valid;
      const char* src;
      if (B_KC) {  // element (k,n) at B[k + n*ldb]
        valid = (nn < N) ? max(0, min(EPC, K - gk)) : 0;
        src = Bg + ((size_t)gk + (size_t)nn * t.ldb) * ES;
      } else {     // element (k,n) at B[n + k*ldb]
        valid = (gk < K) ? max(0, min(EPC, N - nn)) : 0;
        src = Bg + ((size_t)nn + (size_t)gk * t.ldb) * ES;
      }
      cp_async16(sb + b_off(kk, nn) * ES, valid ? src : Bg, valid * ES);
    }
  };

  // 8-byte register-staged path (an operand not 16-byte aligned): word w of
  // a stage is 8-byte word w % WPE of element w / WPE
  constexpr int WPE = ES / 8;
  constexpr int NWA = A_ELEMS * WPE / kThreads, NWB = B_ELEMS * WPE / kThreads;
  static_assert(NWA * kThreads == A_ELEMS * WPE && NWB * kThreads == B_ELEMS * WPE, "stage split");
  double ra[MODE == kLoad8 ? NWA : 1], rb[MODE == kLoad8 ? NWB : 1];
  auto a_elem = [](int e, int& mm, int& kk) {
    if (A_KC) { mm = e / kBK; kk = e % kBK; } else { kk = e / BM; mm = e % BM; }
  };
  auto b_elem = [](int e, int& nn, int& kk) {
    if (B_KC) { nn = e / kBK; kk = e % kBK; } else { kk = e / BN; nn = e % BN; }
  };
  auto fetch = [&](int it) {
    const int k0 = it * kBK;
    const double* Ad = reinterpret_cast<const double*>(Ag);
    const double* Bd = reinterpret_cast<const double*>(Bg);
#pragma unroll
    for (int q = 0; q < NWA; ++q) {
      const int w = tid + q * kThreads, e = w / WPE, h = w % WPE;
      int mm, kk;
      a_elem(e, mm, kk);
      const int gk = k0 + kk;
      const size_t gi = A_KC ? (size_t)gk + (size_t)mm * t.lda : (size_t)mm + (size_t)gk * t.lda;
      ra[q] = (mm < M && gk < K) ? __ldcg(Ad + gi * WPE + h) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < NWB; ++q) {
      const int w = tid + q * kThreads, e = w / WPE, h = w % WPE;
      int nn, kk;
      b_elem(e, nn, kk);
      const int gk = k0 + kk;
      const size_t gi = B_KC ? (size_t)gk + (size_t)nn * t.ldb : (size_t)nn + (size_t)gk * t.ldb;
      rb[q] = (nn < N && gk < K) ? __ldcg(Bd + gi * WPE + h) : 0.0;
    }
  };
  auto put = [&](int buf) {
    double* sa = reinterpret_cast<double*>(smem + buf * STAGE_BYTES);
    double* sb = sa + Sh::A_S * WPE;
#pragma unroll
    for (int q = 0; q < NWA; ++q) {
      const int w = tid + q * kThreads, e = w / WPE, h = w % WPE;
      int mm, kk;
      a_elem(e, mm, kk);
      sa[a_off(mm, kk) * WPE + h] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < NWB; ++q) {
      const int w = tid + q * kThreads, e = w / WPE, h = w % WPE;
      int nn, kk;
      b_elem(e, nn, kk);
      sb[b_off(kk, nn) * WPE + h] = rb[q];
    }
  };

  const int wm = warp / Sh::WN, wn = warp % Sh::WN;
  const int g = lane >> 2, tq = lane & 3;
  double acc[MF][NF][NACC];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int v = 0; v < NACC; ++v) acc[i][j][v] = 0.0;
  const double sgnA = (t.opA == XKB_OP_C) ? -1.0 : 1.0;
  const double sgnB = (t.opB == XKB_OP_C) ? -1.0 : 1.0;

  auto compute = [&](int buf) {
    const uint8_t* sbase = smem + buf * STAGE_BYTES;
    const S* sa = reinterpret_cast<const S*>(sbase);
    const S* sb = reinterpret_cast<const S*>(sbase + Sh::A_S * ES);
#pragma unroll
    for (int kc = 0; kc < kBK / 8; ++kc) {
      // logical k = tq and tq + 4 of the MMA are physical k0 = 2 tq, k1 = k0 + 1
      const int k0 = kc * 8 + 2 * tq, k1 = k0 + 1;
      double br[NF][2], bi[NF][2];
#pragma unroll
      for (int nf = 0; nf < NF; ++nf) {
        const int n = wn * WTN + nf * 8 + g;
        if constexpr (B_KC && !CPLX) {
          const double2 v = *reinterpret_cast<const double2*>(sb + b_off(k0, n));
          br[nf][0] = v.x;
          br[nf][1] = v.y;
        } else {
          ld_elem<T>(sb, b_off(k0, n), br[nf][0], bi[nf][0]);
          ld_elem<T>(sb, b_off(k1, n), br[nf][1], bi[nf][1]);
          if (CPLX) {
            bi[nf][0] *= sgnB;
            bi[nf][1] *= sgnB;
          }
        }
      }
#pragma unroll
      for (int mf = 0; mf < MF; ++mf) {
        const int r0 = wm * WTM + mf * 16 + g, r1 = r0 + 8;
        double ar[4], ai[4];
        if constexpr (A_KC && !CPLX) {
          const double2 v0 = *reinterpret_cast<const double2*>(sa + a_off(r0, k0));
          const double2 v1 = *reinterpret_cast<const double2*>(sa + a_off(r1, k0));
          ar[0] = v0.x;
          ar[1] = v1.x;
          ar[2] = v0.y;
          ar[3] = v1.y;
        } else {
          ld_elem<T>(sa, a_off(r0, k0), ar[0], ai[0]);
          ld_elem<T>(sa, a_off(r1, k0), ar[1], ai[1]);
          ld_elem<T>(sa, a_off(r0, k1), ar[2], ai[2]);
          ld_elem<T>(sa, a_off(r1, k1), ar[3], ai[3]);
        }
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
  };

  if constexpr (MODE != kLoad8) {
    for (int s = 0; s < kSt - 1; ++s) {
      if (s < KT) load_stage(s, s);
      cp_async_commit();
    }
    for (int it = 0; it < KT; ++it) {
      cp_async_wait<kSt - 2>();
      __syncthreads();  // stage `it` landed for everyone; stage it-1 no longer read
      if (it + kSt - 1 < KT) load_stage(it + kSt - 1, (it + kSt - 1) % kSt);
      cp_async_commit();
      compute(it % kSt);
    }
    cp_async_wait<0>();
  } else {
    // registers carry stage it+1 while stage it is computed (two buffers)
    if (KT > 0) {
      fetch(0);
      put(0);
      if (KT > 1) fetch(1);
    }
    for (int it = 0; it < KT; ++it) {
      __syncthreads();  // buffer it%2 written; buffer (it+1)%2 no longer read
      if (it + 1 < KT) put((it + 1) & 1);
      if (it + 2 < KT) fetch(it + 2);
      compute(it & 1);
    }
  }
  __syncthreads();  // smem free for the next task
  S* C = reinterpret_cast<S*>(t.C);
  const bool use_beta = (t.br != 0.0) || (t.bi != 0.0);
  // one row of fragments at a time: all of its C loads, then its stores (C
  // is read and written through one pointer; a load after a store would
  // wait for it)
#pragma unroll
  for (int mf = 0; mf < MF; ++mf) {
    double cv[NF][CPLX ? 8 : 4];
#pragma unroll
    for (int nf = 0; nf < NF; ++nf)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = wm * WTM + mf * 16 + g + ((i >> 1) << 3);
        const int col = wn * WTN + nf * 8 + 2 * tq + (i & 1);
        cv[nf][i] = 0.0;
        if (CPLX) cv[nf][CPLX ? 4 + i : i] = 0.0;
        if (!use_beta || row >= M || col >= N) continue;
        const size_t idx = (size_t)row + (size_t)col * (size_t)t.ldc;
        if constexpr (CPLX) {
          cv[nf][i] = __ldcg(C + 2 * idx);
          cv[nf][4 + i] = __ldcg(C + 2 * idx + 1);
        } else {
          cv[nf][i] = __ldcg(C + idx);
        }
      }
#pragma unroll
    for (int nf = 0; nf < NF; ++nf)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = wm * WTM + mf * 16 + g + ((i >> 1) << 3);
        const int col = wn * WTN + nf * 8 + 2 * tq + (i & 1);
        if (row >= M || col >= N) continue;
        const size_t idx = (size_t)row + (size_t)col * (size_t)t.ldc;
        if constexpr (CPLX) {
          const double xr = acc[mf][nf][i], xi = acc[mf][nf][4 + i];
          const double cr = cv[nf][i], ci = cv[nf][CPLX ? 4 + i : i];
          C[2 * idx] = t.ar * xr - t.ai * xi + (t.br * cr - t.bi * ci);
          C[2 * idx + 1] = t.ar * xi + t.ai * xr + (t.br * ci + t.bi * cr);
        } else {
          C[idx] = fma(t.br, cv[nf][i], t.ar * acc[mf][nf][i]);
        }
      }
  }
}

template <class T, int BM, int MODE>
__device__ __forceinline__ void gemm_dispatch2(const Task& t, uint8_t* smem) {
  const bool akc = t.opA != XKB_OP_N, bkc = t.opB == XKB_OP_N;
  if (akc && bkc) gemm_tile<T, true, true, BM, MODE>(t, smem);
  else if (akc) gemm_tile<T, true, false, BM, MODE>(t, smem);
  else if (bkc) gemm_tile<T, false, true, BM, MODE>(t, smem);
  else gemm_tile<T, false, false, BM, MODE>(t, smem);
}

// ---- trsm diagonal block ------------------------------------------------------
// One 64-row diagonal block against up to 64 right-hand sides: the shared
// register-resident substitution of trsm_leaf.cuh.  Not inlined: its
// register allocation stays apart from the gemm tile's.
constexpr size_t kTrsmSmem = LeafShape<double2>::SMEM;  // complex, the larger

template <class T>
__device__ __noinline__ void trsm_tile(const Task& t, uint8_t* smem, double ar, double ai) {
  using S = typename St<T>::S;
  double* sm = reinterpret_cast<double*>(smem);
  const bool swap = t.flags & kFlagSwap, conj = t.flags & kFlagConj;
  const bool lower = t.flags & kFlagLower, unit = t.flags & kFlagUnit;
  leaf_stage<T, kThreads>(static_cast<const S*>(t.D), t.lda, t.M, swap, conj, lower, unit, sm);
  S* X = static_cast<S*>(t.C);
  if (lower) leaf_solve<T, kThreads, true>(X, t.ldc, false, t.M, 0, t.N, ar, ai, sm);
  else leaf_solve<T, kThreads, false>(X, t.ldc, false, t.M, 0, t.N, ar, ai, sm);
  __syncthreads();
}

// dynamic shared memory: the largest task body (the complex solve's staging,
// 81 KB; gemm stages: real 128 x 64 3 x 26 KB, complex 3 x 24 KB) + alignment
constexpr size_t kSmemMax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kSmemBytes =
    kSmemMax(kTrsmSmem,
             kSmemMax((size_t)kSt * TileShape<double, true, true, 128>::STAGE_BYTES,
                      kSmemMax((size_t)kSt * TileShape<double, false, false, 128>::STAGE_BYTES,
                               (size_t)kSt * TileShape<double2, false, false, 32>::STAGE_BYTES))) +
    128;

__global__ void __launch_bounds__(kThreads, 2)
    k_sched(const Task* __restrict__ tasks, int* ndep, const int* __restrict__ succ,
            const int* __restrict__ bulk, int nbulk, int* urq, int nurg, Ctl* ctl,
            int urgent_first, int* call_left, unsigned long long* call_end,
            unsigned long long* t_start, unsigned long long wait_ns) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  __shared__ int s_idx;
  __shared__ Task s_task;  // the claimed task, read by every thread from here
  __shared__ Task s_sub;   // a gemm step of a solve task
  if (threadIdx.x == 0) atomicMin(t_start, (unsigned long long)globaltimer());
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = claim_task(ctl, bulk, nbulk, urq, nurg, urgent_first != 0, wait_ns);
      if (i >= 0) {
        __threadfence();  // acquire: the producers' outputs before the reads
        s_task = tasks[i];
      }
      s_idx = i;
    }
    __syncthreads();
    if (s_idx < 0) break;
    // only thread 0 rewrites s_task, after every thread is past the barrier
    // that ends this task
    const Task& t = s_task;
    if (t.kind == kTaskGemm) {  // a gemm call's tile: operands read-only here
      const bool nar = t.flags & kFlagNarrow;
      if (t.dtype == XKB_Z) {
        if (nar) gemm_dispatch2<double2, 32, kCopy8>(t, smem);
        else gemm_dispatch2<double2, 32, kCopy16>(t, smem);
      } else if (t.M > 64) {
        if (nar) gemm_dispatch2<double, 128, kCopy8>(t, smem);
        else gemm_dispatch2<double, 128, kCopy16>(t, smem);
      } else {
        if (nar) gemm_dispatch2<double, 64, kCopy8>(t, smem);
        else gemm_dispatch2<double, 64, kCopy16>(t, smem);
      }
    } else {
      // X_i = alpha B_i - op(A)[i, solved] X_solved in gemm tiles of BM rows,
      // then the diagonal solve of X_i (same CTA: the tiles' stores are
      // ordered before its loads by the barrier, both go through L2)
      const bool cplx = t.dtype == XKB_Z;
      double sar = t.ar, sai = t.ai;
      if (t.K > 0) {
        const int bm = cplx ? 32 : 64;
        const int es = cplx ? 16 : 8;
        for (int r0 = 0; r0 < t.M; r0 += bm) {
          if (threadIdx.x == 0) {
            s_sub = t;
            s_sub.M = min(bm, t.M - r0);
            s_sub.A = static_cast<const char*>(t.A) +
                      (size_t)r0 * (t.opA == XKB_OP_N ? 1 : t.lda) * es;
            s_sub.C = static_cast<char*>(t.C) + (size_t)r0 * es;
            s_sub.ar = -1.0;
            s_sub.ai = 0.0;
            s_sub.br = t.ar;
            s_sub.bi = t.ai;
          }
          __syncthreads();
          // op(B) = X rows solved by other CTAs of this launch: L2 only
          const bool nar = t.flags & kFlagNarrow;
          if (!cplx) {
            if (t.opA == XKB_OP_N) {
              if (nar) gemm_tile<double, false, true, 64, kLoad8>(s_sub, smem);
              else gemm_tile<double, false, true, 64, kCopy16>(s_sub, smem);
            } else {
              if (nar) gemm_tile<double, true, true, 64, kLoad8>(s_sub, smem);
              else gemm_tile<double, true, true, 64, kCopy16>(s_sub, smem);
            }
          } else {
            if (t.opA == XKB_OP_N) {
              if (nar) gemm_tile<double2, false, true, 32, kLoad8>(s_sub, smem);
              else gemm_tile<double2, false, true, 32, kCopy16>(s_sub, smem);
            } else {
              if (nar) gemm_tile<double2, true, true, 32, kLoad8>(s_sub, smem);
              else gemm_tile<double2, true, true, 32, kCopy16>(s_sub, smem);
            }
          }
          __syncthreads();  // s_sub is rewritten by the next row part
        }
        sar = 1.0;
        sai = 0.0;
      }
      if (!cplx) trsm_tile<double>(t, smem, sar, sai);
      else trsm_tile<double2>(t, smem, sar, sai);
    }
    __syncthreads();  // every output of the task is stored
    if (threadIdx.x == 0) {
      __threadfence();  // release the outputs before any successor is queued
      for (int k = 0; k < t.nsucc; ++k) {
        const int sidx = succ[t.succ0 + k];
        if (atomicSub(ndep + sidx, 1) == 1) {
          const int pos = atomicAdd(&ctl->tail_urg, 1);
          atomicExch(urq + pos, sidx);
        }
      }
      if (atomicSub(call_left + t.call, 1) == 1) call_end[t.call] = globaltimer();
    }
  }
}

// ---------------------------------------------------------------------------
// host: task graph construction
struct Built {
  std::vector<Task> tasks;                 // indexed by task id
  std::vector<int> ndep;                   // initial dependency count
  std::vector<std::pair<int, int>> edges;  // (producer, consumer)
  std::vector<int> bulk;                   // dependency-free gemm tiles
  std::vector<int> urg_ready;              // solve tasks ready at launch
  int nurg = 0;                            // solve tasks in total
  std::vector<int> call_tasks;
  int add(const Task& t, int ndep0) {
    tasks.push_back(t);
    ndep.push_back(ndep0);
    return (int)tasks.size() - 1;
  }
};

static int esz(int dt) { return dt == XKB_Z ? 16 : 8; }

static bool aligned_ok(const void* p, long ld, int es) {
  return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && ((ld * es) % 16 == 0);
}

static bool ptr8(const void* p) { return reinterpret_cast<uintptr_t>(p) % 8 == 0; }

static int tile128_rows() { return (int)tune("batch_tile128_min_rows", 96.0); }

static Task gemm_task(int dtype, int opA, int opB, int M, int N, int K, int call, const void* A,
                      long lda, const void* B, long ldb, void* C, long ldc, double ar, double ai,
                      double br, double bi, int flags) {
  Task t;
  std::memset(&t, 0, sizeof(t));
  t.kind = kTaskGemm;
  t.dtype = dtype;
  t.opA = opA;
  t.opB = opB;
  t.M = M;
  t.N = N;
  t.K = K;
  t.call = call;
  t.A = A;
  t.lda = lda;
  t.B = B;
  t.ldb = ldb;
  t.C = C;
  t.ldc = ldc;
  t.ar = ar;
  t.ai = ai;
  t.br = br;
  t.bi = bi;
  t.flags = flags;
  return t;
}

// A gemm call: independent C tiles (the reference's tile loop,
// blas/zgemm.c:279-367, with the whole K range in one task).
static int add_gemm(Built& b, const xkb_batch_op& o, int call) {
  const int es = esz(o.dtype);
  // real calls of at least batch_tile128_min_rows rows (tuning table,
  // default 96) use 128-row tiles (the kernel picks the 128 x 64 body for
  // any real task taller than 64 rows)
  const int BM = o.dtype == XKB_Z ? 32 : (o.M >= tile128_rows() ? 128 : 64), BN = 64;
  if (!ptr8(o.A) || !ptr8(o.B) || !ptr8(o.C)) return XKB_EINVAL;
  const int narrow =
      (aligned_ok(o.A, o.lda, es) && aligned_ok(o.B, o.ldb, es)) ? 0 : kFlagNarrow;
  const char* A = static_cast<const char*>(o.A);
  const char* B = static_cast<const char*>(o.B);
  char* C = static_cast<char*>(o.C);
  int n = 0;
  for (int n0 = 0; n0 < o.N; n0 += BN)
    for (int m0 = 0; m0 < o.M; m0 += BM) {
      const char* Ap = o.opA == XKB_OP_N ? A + (size_t)m0 * es : A + (size_t)m0 * o.lda * es;
      const char* Bp = o.opB == XKB_OP_N ? B + (size_t)n0 * o.ldb * es : B + (size_t)n0 * es;
      char* Cp = C + ((size_t)m0 + (size_t)n0 * o.ldc) * es;
      b.bulk.push_back(b.add(gemm_task(o.dtype, o.opA, o.opB, std::min(BM, o.M - m0),
                                       std::min(BN, o.N - n0), o.K, call, Ap, o.lda, Bp, o.ldb,
                                       Cp, o.ldc, o.alpha[0], o.alpha[1], o.beta[0],
                                       o.beta[1], narrow),
                             0));
      ++n;
    }
  return n;
}

// Left triangular solve: the reference's block algorithm (blas/ztrsm.c:
// 241-372; alpha applied once, its lalpha), left-looking.  Blocks are taken
// in solve order s = 0 .. mt-1 (bk = order(s): forward for an effectively
// lower op(A), backward otherwise); task (s, j) forms
//   X_bk,j = alpha B_bk,j - op(A)[bk, done] X_done,j,   done = order(0..s-1)
// and solves with op(A)[bk,bk].  The blocks already solved are contiguous
// (rows [0, bk*64) forward, [(bk+1)*64, M) backward), so the sum is one gemm
// with K = 64 s (64 (mt-1-s) backward, the last block possibly shorter).
// Task (s, j) depends on task (s-1, j) only: one chain per j.
static int add_trsm(Built& b, const xkb_batch_op& o, int call) {
  const int es = esz(o.dtype);
  if (o.side != 0) return XKB_EINVAL;  // right side: not a batch task
  if (!ptr8(o.A) || !ptr8(o.C)) return XKB_EINVAL;
  const int narrow =
      (aligned_ok(o.A, o.lda, es) && aligned_ok(o.C, o.ldc, es)) ? 0 : kFlagNarrow;
  const bool cplx = o.dtype == XKB_Z;
  const int trans = (!cplx && o.trans == XKB_OP_C) ? XKB_OP_T : o.trans;
  const bool fwd = (o.uplo == XKB_LOWER) ^ (trans != XKB_OP_N);
  const int mt = (o.M + kLeafS - 1) / kLeafS, nt = (o.N + kLeafS - 1) / kLeafS;
  const char* A = static_cast<const char*>(o.A);
  char* X = static_cast<char*>(o.C);
  const int dflags = (trans != XKB_OP_N ? kFlagSwap : 0) | (trans == XKB_OP_C ? kFlagConj : 0) |
                     (fwd ? kFlagLower : 0) | (o.diag ? kFlagUnit : 0);
  // element (r, c) of op(A) lives at A[r + c lda] (trans N) or A[c + r lda]
  auto opA_at = [&](size_t r, size_t c) {
    return trans == XKB_OP_N ? A + (r + c * o.lda) * es : A + (c + r * o.lda) * es;
  };
  int n = 0;
  for (int j = 0; j < nt; ++j) {
    const size_t c0 = (size_t)j * kLeafS;
    int prev = -1;
    for (int s = 0; s < mt; ++s) {
      const int bk = fwd ? s : mt - 1 - s;
      const size_t r0 = (size_t)bk * kLeafS;
      const int rows = std::min(kLeafS, o.M - bk * kLeafS);
      const size_t k0 = fwd ? 0 : r0 + rows;             // first solved row
      const int K = fwd ? (int)r0 : o.M - (int)(r0 + rows);  // solved rows
      Task t;
      std::memset(&t, 0, sizeof(t));
      t.kind = kTaskTrsm;
      t.dtype = o.dtype;
      t.opA = trans;
      t.opB = XKB_OP_N;
      t.M = rows;
      t.N = std::min(kLeafS, o.N - j * kLeafS);
      t.K = K;
      t.call = call;
      t.A = K > 0 ? opA_at(r0, k0) : A;
      t.lda = o.lda;
      t.B = X + (k0 + c0 * o.ldc) * es;
      t.ldb = o.ldc;
      t.C = X + (r0 + c0 * o.ldc) * es;
      t.ldc = o.ldc;
      t.D = A + (r0 + r0 * o.lda) * es;
      t.ar = o.alpha[0];
      t.ai = cplx ? o.alpha[1] : 0.0;
      t.flags = dflags | narrow;
      const int id = b.add(t, prev >= 0 ? 1 : 0);
      ++b.nurg;
      ++n;
      if (prev >= 0) b.edges.emplace_back(prev, id);
      else b.urg_ready.push_back(id);
      prev = id;
    }
  }
  return n;
}

// Device image of one batch: tasks | ndep | succ | bulk | urq | call_left |
// ctl.  tasks, succ and bulk are read-only during a launch; ndep, urq,
// call_left and ctl are consumed by it.
struct Layout {
  int ntasks = 0, nops = 0;
  size_t nbulk = 0, nurg = 0, nsucc = 0;
  size_t o_ndep = 0, o_succ = 0, o_bulk = 0, o_urq = 0, o_left = 0, o_ctl = 0, bytes = 0;
  void set(int nt, size_t ns, size_t nb, size_t nu, int no) {
    ntasks = nt;
    nsucc = ns;
    nbulk = nb;
    nurg = nu;
    nops = no;
    o_ndep = (size_t)nt * sizeof(Task);
    o_succ = o_ndep + (size_t)nt * 4;
    o_bulk = o_succ + ns * 4;
    o_urq = o_bulk + nb * 4;
    o_left = o_urq + nu * 4;
    o_ctl = (o_left + (size_t)no * 4 + 15) & ~size_t(15);
    bytes = o_ctl + sizeof(Ctl);
  }
};

// A batch seen before, kept as a CUDA graph: reset the consumed state from
// the pristine image (two device-to-device copies), clear the timestamps,
// run k_sched.  Replaying skips the host-side task construction and the
// upload of the task list.
struct GraphEntry {
  uint64_t key = 0;
  int schedule = 0;
  std::vector<xkb_batch_op> ops;  // the op list, compared on lookup
  Layout L;
  uint8_t* d_img = nullptr;       // pristine image
  uint8_t* d_run = nullptr;       // image the launch consumes
  unsigned long long* d_times = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int> call_tasks;
  uint64_t last_use = 0;
  size_t bytes() const { return 2 * L.bytes + ((size_t)L.nops + 1) * 8; }
};

struct Batch {
  uint8_t* h_stage = nullptr;  // pinned: the image of the batch being launched
  size_t h_cap = 0;
  uint8_t* d_buf = nullptr;    // device image of uncached batches
  size_t d_cap = 0;
  unsigned long long* d_times = nullptr;  // call_end[ncalls], t_start
  size_t d_cap_times = 0;
  // the last launch (read by xkb_cuda_batch_latency)
  int ncalls = 0;
  std::vector<int> call_tasks;
  unsigned long long* cur_times = nullptr;
  // graph cache (XKBLAS_BATCH_GRAPHS=0 disables)
  std::vector<GraphEntry*> graphs;
  std::vector<uint64_t> seen;  // keys of recent uncached batches
  uint64_t tick = 0;
  size_t graph_bytes = 0;
};

constexpr size_t kGraphMaxEntries = 8;
constexpr size_t kGraphMaxBytes = size_t(2) << 30;

static void free_entry(GraphEntry* e, cudaStream_t st) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->d_img) cudaFreeAsync(e->d_img, st);
  if (e->d_run) cudaFreeAsync(e->d_run, st);
  if (e->d_times) cudaFreeAsync(e->d_times, st);
  delete e;
}

// field-wise (the struct has padding bytes, which callers need not clear)
static bool same_op(const xkb_batch_op& a, const xkb_batch_op& b) {
  return a.kind == b.kind && a.dtype == b.dtype && a.opA == b.opA && a.opB == b.opB &&
         a.side == b.side && a.uplo == b.uplo && a.trans == b.trans && a.diag == b.diag &&
         a.M == b.M && a.N == b.N && a.K == b.K && a.A == b.A && a.lda == b.lda && a.B == b.B &&
         a.ldb == b.ldb && a.C == b.C && a.ldc == b.ldc && a.alpha[0] == b.alpha[0] &&
         a.alpha[1] == b.alpha[1] && a.beta[0] == b.beta[0] && a.beta[1] == b.beta[1];
}

static uint64_t op_key(const xkb_batch_op* ops, int nops, int schedule) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)(unsigned)schedule;
  auto mix = [&](uint64_t v) {
    for (int i = 0; i < 8; ++i) h = (h ^ ((v >> (8 * i)) & 0xffu)) * 1099511628211ull;
  };
  auto bits = [](double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
  };
  for (int c = 0; c < nops; ++c) {
    const xkb_batch_op& o = ops[c];
    mix(((uint64_t)(unsigned)o.kind << 32) ^ (uint64_t)(unsigned)o.dtype);
    mix(((uint64_t)(unsigned)o.opA << 48) ^ ((uint64_t)(unsigned)o.opB << 32) ^
        ((uint64_t)(unsigned)o.side << 16) ^ (uint64_t)(unsigned)o.uplo);
    mix(((uint64_t)(unsigned)o.trans << 32) ^ (uint64_t)(unsigned)o.diag);
    mix(((uint64_t)(unsigned)o.M << 32) ^ (uint64_t)(unsigned)o.N);
    mix((uint64_t)(unsigned)o.K);
    mix(reinterpret_cast<uintptr_t>(o.A));
    mix((uint64_t)o.lda);
    mix(reinterpret_cast<uintptr_t>(o.B));
    mix((uint64_t)o.ldb);
    mix(reinterpret_cast<uintptr_t>(o.C));
    mix((uint64_t)o.ldc);
    mix(bits(o.alpha[0]));
    mix(bits(o.alpha[1]));
    mix(bits(o.beta[0]));
    mix(bits(o.beta[1]));
  }
  return h ^ (uint64_t)nops;
}

// kernel arguments of one launch on image d
// How long a CTA of the executor waits for a task whose dependencies are
// not yet resolved before it records kErrFullWait and the launch ends: the
// tuning key sched_wait_ms (default 4000 ms), a kernel parameter.
static unsigned long long wait_limit_ns() {
  const double ms = tune("sched_wait_ms", (double)(kWaitLimitNs / 1000000ull));
  return (unsigned long long)(std::max(1.0, ms) * 1e6);
}

struct KArgs {
  const Task* tasks;
  int* ndep;
  const int* succ;
  const int* bulk;
  int nbulk;
  int* urq;
  int nurg;
  Ctl* ctl;
  int urgent_first;
  int* left;
  unsigned long long* call_end;
  unsigned long long* t_start;
  unsigned long long wait_ns;
  KArgs(uint8_t* d, const Layout& L, int schedule, unsigned long long* times)
      : tasks(reinterpret_cast<const Task*>(d)),
        ndep(reinterpret_cast<int*>(d + L.o_ndep)),
        succ(reinterpret_cast<const int*>(d + L.o_succ)),
        bulk(reinterpret_cast<const int*>(d + L.o_bulk)),
        nbulk((int)L.nbulk),
        urq(reinterpret_cast<int*>(d + L.o_urq)),
        nurg((int)L.nurg),
        ctl(reinterpret_cast<Ctl*>(d + L.o_ctl)),
        urgent_first(schedule == 0 ? 1 : 0),
        left(reinterpret_cast<int*>(d + L.o_left)),
        call_end(times),
        t_start(times + L.nops),
        wait_ns(wait_limit_ns()) {}
  void* params[13] = {&tasks, &ndep, &succ,         &bulk, &nbulk,    &urq,    &nurg,
                      &ctl,   &urgent_first, &left, &call_end, &t_start, &wait_ns};
};

static Batch& batch() {
  static Batch b;
  return b;
}
static std::mutex g_batch_mu;

static int grid_size() {
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sched, kThreads, kSmemBytes);
  if (per <= 0) per = 1;
  return per * sm_count();
}

static int set_smem_attr() {
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_sched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSmemBytes) != cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  return XKB_OK;
}

// Per-call rows of an executor launch in the event trace (recording on).
static void trace_calls(long long tv, cudaStream_t st, const unsigned long long* d_times,
                        const xkb_batch_op* ops, int n) {
  if (tv < 0) return;
  static const char* const kNames[2][2] = {{"dgemm", "zgemm"}, {"dtrsm", "ztrsm"}};
  std::vector<const char*> names((size_t)n);
  for (int i = 0; i < n; ++i)
    names[i] = kNames[ops[i].kind == XKB_BATCH_TRSM][ops[i].dtype == XKB_Z];
  evlog_kern_calls(tv, st, d_times, n, names.data());
}

static int launch_entry(Batch& B, GraphEntry* e, cudaStream_t st) {
  e->last_use = ++B.tick;
  B.ncalls = e->L.nops;
  B.call_tasks = e->call_tasks;
  B.cur_times = e->d_times;
  const long long tv = evlog_kern_begin(st, "k_sched(graph)");
  const cudaError_t le = cudaGraphLaunch(e->exec, st);
  evlog_kern_end(tv, st);
  if (le != cudaSuccess) return XKB_ECUDA;
  trace_calls(tv, st, e->d_times, e->ops.data(), e->L.nops);
  count_launch();
  return XKB_OK;
}

// Build the graph of a cached batch whose image is in e->d_img.
static int build_graph(GraphEntry* e) {
  const Layout& L = e->L;
  if (cudaGraphCreate(&e->graph, 0) != cudaSuccess) return XKB_ECUDA;
  cudaGraphNode_t cp, m0, m1, kn;
  if (cudaGraphAddMemcpyNode1D(&cp, e->graph, nullptr, 0, e->d_run, e->d_img, L.bytes,
                               cudaMemcpyDeviceToDevice) != cudaSuccess)
    return XKB_ECUDA;
  cudaMemsetParams ms{};
  ms.dst = e->d_times;
  ms.value = 0;
  ms.elementSize = 1;
  ms.width = (size_t)L.nops * 8;
  ms.height = 1;
  ms.pitch = ms.width;
  if (cudaGraphAddMemsetNode(&m0, e->graph, nullptr, 0, &ms) != cudaSuccess) return XKB_ECUDA;
  ms.dst = e->d_times + L.nops;
  ms.value = 0xff;
  ms.width = 8;
  ms.pitch = 8;
  if (cudaGraphAddMemsetNode(&m1, e->graph, nullptr, 0, &ms) != cudaSuccess) return XKB_ECUDA;
  KArgs a(e->d_run, L, e->schedule, e->d_times);
  cudaKernelNodeParams kp{};
  kp.func = reinterpret_cast<void*>(k_sched);
  kp.gridDim = dim3((unsigned)std::min(grid_size(), std::max(1, L.ntasks)));
  kp.blockDim = dim3(kThreads);
  kp.sharedMemBytes = (unsigned)kSmemBytes;
  kp.kernelParams = a.params;
  const cudaGraphNode_t deps[3] = {cp, m0, m1};
  if (cudaGraphAddKernelNode(&kn, e->graph, deps, 3, &kp) != cudaSuccess) return XKB_ECUDA;
  if (cudaGraphInstantiate(&e->exec, e->graph, 0) != cudaSuccess) return XKB_ECUDA;
  return XKB_OK;
}

}  // namespace sched
}  // namespace xkb

using namespace xkb;
using namespace xkb::sched;

extern "C" int xkb_cuda_batch(const xkb_batch_op* ops, int nops, int schedule, void* stream) {
  if (!ops || nops < 0) return XKB_EINVAL;
  if (nops == 0) return XKB_OK;
  std::lock_guard<std::mutex> g(g_batch_mu);
  cudaStream_t st = resolve_stream(stream);
  Batch& B = batch();
  if (int e = set_smem_attr()) return e;
  static const bool use_graphs = [] {
    const char* v = getenv("XKBLAS_BATCH_GRAPHS");
    return !(v && v[0] == '0');
  }();
  const uint64_t key = use_graphs ? op_key(ops, nops, schedule) : 0;
  if (use_graphs) {
    for (GraphEntry* e : B.graphs) {
      if (e->key != key || e->schedule != schedule || (int)e->ops.size() != nops) continue;
      bool same = true;
      for (int c = 0; c < nops && same; ++c) same = same_op(e->ops[(size_t)c], ops[c]);
      if (same) return launch_entry(B, e, st);
    }
  }
  Built b;
  b.call_tasks.assign(nops, 0);
  {  // size every list once: the task build is a hot host path for big batches
    size_t nt = 0, ne = 0, nb = 0;
    for (int c = 0; c < nops; ++c) {
      const xkb_batch_op& o = ops[c];
      if (o.M <= 0 || o.N <= 0) continue;
      if (o.kind == XKB_BATCH_GEMM) {
        const size_t bm = o.dtype == XKB_Z ? 32 : (o.M >= tile128_rows() ? 128 : 64);
        const size_t t = ((size_t)o.M + bm - 1) / bm * (((size_t)o.N + 63) / 64);
        nt += t;
        nb += t;
      } else {
        const size_t t = ((size_t)o.M + kLeafS - 1) / kLeafS * (((size_t)o.N + kLeafS - 1) / kLeafS);
        nt += t;
        ne += t;
      }
    }
    b.tasks.reserve(nt);
    b.ndep.reserve(nt);
    b.bulk.reserve(nb);
    b.edges.reserve(ne);
  }
  for (int c = 0; c < nops; ++c) {
    const xkb_batch_op& o = ops[c];
    if ((o.dtype != XKB_D && o.dtype != XKB_Z) || o.M < 0 || o.N < 0 || o.K < 0) return XKB_EINVAL;
    if (o.M == 0 || o.N == 0) continue;
    int n;
    if (o.kind == XKB_BATCH_GEMM) {
      if (o.K == 0) return XKB_EINVAL;  // beta-only calls are not batch tasks
      n = add_gemm(b, o, c);
    } else if (o.kind == XKB_BATCH_TRSM) {
      n = add_trsm(b, o, c);
    } else {
      return XKB_EINVAL;
    }
    if (n < 0) return n;
    b.call_tasks[c] = n;
  }
  const int ntasks = (int)b.tasks.size();
  B.ncalls = nops;
  B.call_tasks = b.call_tasks;
  if (ntasks == 0) return XKB_OK;
  // successor lists (CSR over producers)
  std::vector<int> succ0((size_t)ntasks + 1, 0);
  for (auto& e : b.edges) ++succ0[(size_t)e.first + 1];
  for (int i = 0; i < ntasks; ++i) succ0[(size_t)i + 1] += succ0[(size_t)i];
  std::vector<int> succ(b.edges.size());
  {
    std::vector<int> fill(succ0.begin(), succ0.end() - 1);
    for (auto& e : b.edges) succ[(size_t)fill[(size_t)e.first]++] = e.second;
  }
  for (int i = 0; i < ntasks; ++i) {
    b.tasks[(size_t)i].succ0 = succ0[(size_t)i];
    b.tasks[(size_t)i].nsucc = succ0[(size_t)i + 1] - succ0[(size_t)i];
  }
  Layout L;
  L.set(ntasks, succ.size(), b.bulk.size(), (size_t)b.nurg, nops);
  // the previous batch may still read the pinned staging buffer
  if (B.h_stage) cudaStreamSynchronize(st);
  if (L.bytes > B.h_cap) {
    if (B.h_stage) cudaFreeHost(B.h_stage);
    B.h_cap = L.bytes * 2;
    if (cudaHostAlloc(&B.h_stage, B.h_cap, cudaHostAllocDefault) != cudaSuccess) {
      B.h_stage = nullptr;
      B.h_cap = 0;
      return XKB_ENOMEM;
    }
  }
  uint8_t* h = B.h_stage;
  std::memcpy(h, b.tasks.data(), L.o_ndep);
  std::memcpy(h + L.o_ndep, b.ndep.data(), (size_t)ntasks * 4);
  if (!succ.empty()) std::memcpy(h + L.o_succ, succ.data(), succ.size() * 4);
  if (L.nbulk) std::memcpy(h + L.o_bulk, b.bulk.data(), L.nbulk * 4);
  int* urq = reinterpret_cast<int*>(h + L.o_urq);
  for (size_t i = 0; i < L.nurg; ++i) urq[i] = i < b.urg_ready.size() ? b.urg_ready[i] : -1;
  std::memcpy(h + L.o_left, b.call_tasks.data(), (size_t)nops * 4);
  Ctl ctl{0, 0, (int)b.urg_ready.size(), 0};
  std::memcpy(h + L.o_ctl, &ctl, sizeof(ctl));

  // a batch seen before (recently, uncached) becomes a cached graph
  bool cache = false;
  if (use_graphs) {
    auto it = std::find(B.seen.begin(), B.seen.end(), key);
    if (it != B.seen.end()) {
      B.seen.erase(it);
      cache = 2 * L.bytes <= kGraphMaxBytes;
    } else {
      B.seen.push_back(key);
      if (B.seen.size() > 32) B.seen.erase(B.seen.begin());
    }
  }
  if (cache) {
    GraphEntry* e = new GraphEntry;
    e->key = key;
    e->schedule = schedule;
    e->ops.assign(ops, ops + nops);
    e->L = L;
    e->call_tasks = b.call_tasks;
    if (cudaMallocAsync(&e->d_img, L.bytes, st) != cudaSuccess ||
        cudaMallocAsync(&e->d_run, L.bytes, st) != cudaSuccess ||
        cudaMallocAsync(&e->d_times, ((size_t)nops + 1) * 8, st) != cudaSuccess) {
      cudaGetLastError();
      free_entry(e, st);
      return XKB_ENOMEM;
    }
    cudaMemcpyAsync(e->d_img, h, L.bytes, cudaMemcpyHostToDevice, st);
    if (int r = build_graph(e)) {
      free_entry(e, st);
      return r;
    }
    // evict least recently used entries beyond the limits
    while (!B.graphs.empty() && (B.graphs.size() >= kGraphMaxEntries ||
                                 B.graph_bytes + e->bytes() > kGraphMaxBytes)) {
      auto lru = std::min_element(B.graphs.begin(), B.graphs.end(),
                                  [](GraphEntry* x, GraphEntry* y) { return x->last_use < y->last_use; });
      B.graph_bytes -= (*lru)->bytes();
      free_entry(*lru, st);
      B.graphs.erase(lru);
    }
    B.graphs.push_back(e);
    B.graph_bytes += e->bytes();
    return launch_entry(B, e, st);
  }

  if (L.bytes > B.d_cap) {
    if (B.d_buf) cudaFreeAsync(B.d_buf, st);
    B.d_cap = L.bytes * 2;
    if (cudaMallocAsync(&B.d_buf, B.d_cap, st) != cudaSuccess) {
      B.d_buf = nullptr;
      B.d_cap = 0;
      return XKB_ENOMEM;
    }
  }
  if ((size_t)nops + 1 > B.d_cap_times) {
    if (B.d_times) cudaFreeAsync(B.d_times, st);
    B.d_cap_times = ((size_t)nops + 1) * 2;
    if (cudaMallocAsync(&B.d_times, B.d_cap_times * sizeof(unsigned long long), st) !=
        cudaSuccess) {
      B.d_times = nullptr;
      B.d_cap_times = 0;
      return XKB_ENOMEM;
    }
  }
  uint8_t* d = B.d_buf;
  cudaMemcpyAsync(d, h, L.bytes, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(B.d_times, 0, (size_t)nops * sizeof(unsigned long long), st);
  cudaMemsetAsync(B.d_times + nops, 0xff, sizeof(unsigned long long), st);
  B.cur_times = B.d_times;
  KArgs a(d, L, schedule, B.d_times);
  const int grid = std::min(grid_size(), std::max(1, ntasks));
  const long long tv = evlog_kern_begin(st, "k_sched");
  k_sched<<<grid, kThreads, kSmemBytes, st>>>(a.tasks, a.ndep, a.succ, a.bulk, a.nbulk, a.urq,
                                              a.nurg, a.ctl, a.urgent_first, a.left,
                                              a.call_end, a.t_start, a.wait_ns);
  evlog_kern_end(tv, st);
  trace_calls(tv, st, B.d_times, ops, nops);
  count_launch();
  // the pinned staging buffer must outlive the copy: the copy is ordered
  // before the kernel, and the next batch synchronises before reusing it
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

extern "C" int xkb_cuda_batch_latency(double* ms, int n) {
  Batch& B = batch();
  std::lock_guard<std::mutex> g(g_batch_mu);
  if (!ms || n < 0 || n > B.ncalls || !B.cur_times) return XKB_EINVAL;
  if (cudaDeviceSynchronize() != cudaSuccess) return XKB_ECUDA;
  std::vector<unsigned long long> t((size_t)B.ncalls + 1);
  if (cudaMemcpy(t.data(), B.cur_times, t.size() * sizeof(unsigned long long),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return XKB_ECUDA;
  const unsigned long long t0 = t[B.ncalls];
  for (int i = 0; i < n; ++i)
    ms[i] = (B.call_tasks[i] && t[i] >= t0) ? (double)(t[i] - t0) * 1e-6 : 0.0;
  return XKB_OK;
}

extern "C" int xkb_cuda_batch_release(void) {
  Batch& B = batch();
  std::lock_guard<std::mutex> g(g_batch_mu);
  if (cudaDeviceSynchronize() != cudaSuccess) return XKB_ECUDA;
  for (GraphEntry* e : B.graphs) free_entry(e, nullptr);
  B.graphs.clear();
  B.seen.clear();
  B.graph_bytes = 0;
  if (B.cur_times && B.cur_times != B.d_times) B.cur_times = nullptr;
  return XKB_OK;
}

extern "C" int xkb_cuda_batch_cached(void) {
  Batch& B = batch();
  std::lock_guard<std::mutex> g(g_batch_mu);
  return (int)B.graphs.size();
}

// Exercises the bounded wait on the device: one CTA of the executor is
// launched on a ready queue whose only slot claims a task (the queue's tail
// was advanced) that no producer ever writes -- as if the task's last
// dependency never resolved.  The CTA waits wait_ms, records kErrFullWait
// and ends; the launch returns normally and the context stays usable.  The
// caller reads the outcome with xkb_cuda_take_device_error (or xkblas_sync).
extern "C" int xkb_cuda_sched_wait_test(int wait_ms, void* stream) {
  if (wait_ms < 1 || wait_ms > 10000) return XKB_EINVAL;
  cudaStream_t st = resolve_stream(stream);
  if (int e = set_smem_attr()) return e;
  // layout: ctl | urq[1] | ndep[1] | left[1] | times[2] | task[1]
  const size_t o_urq = 16, o_ndep = 32, o_left = 48, o_times = 64, o_task = 128;
  const size_t bytes = o_task + sizeof(Task);
  uint8_t* d = nullptr;
  if (cudaMallocAsync(&d, bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return XKB_ENOMEM;
  }
  uint8_t h[o_task + sizeof(Task)];
  std::memset(h, 0, sizeof h);
  const Ctl ctl{0, 0, 1, 0};  // no bulk work; one queued ticket ...
  std::memcpy(h, &ctl, sizeof ctl);
  const int unset = -1;       // ... whose slot is never written
  std::memcpy(h + o_urq, &unset, sizeof unset);
  const int one = 1;
  std::memcpy(h + o_ndep, &one, sizeof one);
  std::memcpy(h + o_left, &one, sizeof one);
  cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
  auto* times = reinterpret_cast<unsigned long long*>(d + o_times);
  cudaMemsetAsync(times + 1, 0xff, sizeof(unsigned long long), st);
  const long long tv = evlog_kern_begin(st, "k_sched");
  k_sched<<<1, kThreads, kSmemBytes, st>>>(
      reinterpret_cast<const Task*>(d + o_task), reinterpret_cast<int*>(d + o_ndep), nullptr,
      nullptr, 0, reinterpret_cast<int*>(d + o_urq), 1, reinterpret_cast<Ctl*>(d), 1,
      reinterpret_cast<int*>(d + o_left), times, times + 1, (unsigned long long)wait_ms * 1000000ull);
  evlog_kern_end(tv, st);
  count_launch();
  cudaFreeAsync(d, st);
  // the staging array h is copied by the time the host can return: pageable
  // memory makes cudaMemcpyAsync stage it synchronously
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}
