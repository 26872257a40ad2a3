// sched.cu -- the tile-task executor: one persistent launch runs a whole
// batch of level-3 calls as a DAG of tile tasks.
//
// Replaces the reference's XKaapi machinery for this path: per-tile tasks
// (blas/ztask_gemm.c:107-158, ztask_trsm.c), their data-flow dependencies
// (kaapi/kaapi_task.c:1277-1327) and the device threads that pop ready tasks
// and launch one cuBLAS call each (kaapi/kaapi_offload_device.c:463-683,
// 852-1210).  Here the host builds the task list once, in a topological
// order; persistent CTAs claim tasks in that order with an atomic counter,
// wait (bounded) on per-tile dependency counters, run the tile body on the
// FP64 tensor cores, and bump the counters of the tiles they produced.  A
// batch of small, uneven calls thus costs one launch instead of one launch
// (or thousands of tile tasks with host round trips) per call.
//
// Tile bodies (256 threads):
//   gemm   C[<=BM x <=BN] = alpha op(A) op(B) + beta C over the full K,
//          cp.async 3-stage shared-memory ring (16-byte copies, or 8-byte
//          ones when a leading dimension is odd; zero fill at ragged
//          edges), DMMA m16n8k8; BM x BN = 64 x 64 (real), 32 x 64 (complex,
//          four real MMAs per product);
//   trsm   one 64-row diagonal block of a left triangular solve against up
//          to 64 right-hand sides (the reference's tile body ztask_trsm.c);
//          the trailing updates of the tile algorithm (blas/ztrsm.c:241-372)
//          are gemm tasks.
// Ordering rules: a producer stores, then __syncthreads, then thread 0
// issues __threadfence and increments the counter; a consumer's thread 0
// observes the counter, issues __threadfence, and the CTA reads through L2
// (cp.async.cg / ld.global.cg) -- no stale L1 lines, no async-proxy reads.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "dmma_common.cuh"
#include "xkb_dev.cuh"

namespace xkb {
namespace sched {

enum : int { kTaskGemm = 0, kTaskTrsmDiag = 1 };
// kFlagNarrow: an operand base or leading dimension is not 16-byte aligned,
// so the gemm tile stages it with 8-byte copies instead of 16-byte ones
enum : int { kFlagSwap = 1, kFlagConj = 2, kFlagLower = 4, kFlagUnit = 8, kFlagNarrow = 16 };

struct alignas(16) Task {
  int kind, dtype, opA, opB;
  int M, N, K, call;
  const void* A;
  const void* B;
  void* C;
  long lda, ldb, ldc;
  double ar, ai, br, bi;
  int wait0, target0, wait1, target1;
  int signal, flags, pad0, pad1;
};

constexpr int kThreads = 256;
constexpr int kBK = 16;
constexpr int kSt = 3;      // cp.async stages
constexpr int kLeafS = 64;  // trsm block

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

// Bounded wait: *c >= target.  Returns false (error recorded) after the
// time limit or when another CTA already recorded an error.
__device__ __forceinline__ bool wait_ge(const int* c, int target) {
  const volatile int* v = c;
  if (*v >= target) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t i = 1;; ++i) {
    if (*v >= target) return true;
    __nanosleep(64);
    if ((i & 63u) == 0) {
      if (dev_error_set()) return false;
      if (globaltimer() - t0 > kWaitLimitNs) {
        dev_error(kErrFullWait);
        return false;
      }
    }
  }
}

// ---- gemm tile ---------------------------------------------------------------
template <class T, bool A_KC, bool B_KC>
__device__ __forceinline__ void gemm_tile(const Task& t, uint8_t* smem) {
  using S = typename St<T>::S;
  constexpr bool CPLX = St<T>::CPLX;
  constexpr int BM = CPLX ? 32 : 64, BN = 64;
  constexpr int WTM = BM / 2, WTN = BN / 4;
  constexpr int MF = WTM / 16, NF = WTN / 8;
  constexpr int ES = (int)sizeof(T);
  constexpr int EPC = 16 / ES;  // elements per 16-byte chunk
  constexpr int A_ELEMS = BM * kBK, B_ELEMS = BN * kBK;
  constexpr int STAGE_BYTES = (A_ELEMS + B_ELEMS) * ES;
  constexpr int NACC = CPLX ? 8 : 4;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const char* Ag = static_cast<const char*>(t.A);
  const char* Bg = static_cast<const char*>(t.B);
  const int M = t.M, N = t.N, K = t.K;
  const int KT = (K + kBK - 1) / kBK;

  const bool narrow = t.flags & kFlagNarrow;
  auto load_stage = [&](int it, int buf) {
    uint8_t* sa = smem + buf * STAGE_BYTES;
    uint8_t* sb = sa + A_ELEMS * ES;
    const int k0 = it * kBK;
    if (narrow) {  // same shared layout, one 8-byte word per copy
      constexpr int WPE = ES / 8;
      for (int w = tid; w < A_ELEMS * WPE; w += kThreads) {
        const int e = w / WPE, h = w % WPE;
        const int mm = A_KC ? e / kBK : e % BM, kk = A_KC ? e % kBK : e / BM;
        const int gk = k0 + kk;
        const bool v = mm < M && gk < K;
        const size_t gi =
            A_KC ? (size_t)gk + (size_t)mm * t.lda : (size_t)mm + (size_t)gk * t.lda;
        const int soff = A_KC ? (mm * kBK + kk) : (kk * BM + mm);
        cp_async8(sa + soff * ES + h * 8, v ? Ag + gi * ES + h * 8 : Ag, v ? 8 : 0);
      }
      for (int w = tid; w < B_ELEMS * WPE; w += kThreads) {
        const int e = w / WPE, h = w % WPE;
        const int nn = B_KC ? e / kBK : e % BN, kk = B_KC ? e % kBK : e / BN;
        const int gk = k0 + kk;
        const bool v = nn < N && gk < K;
        const size_t gi =
            B_KC ? (size_t)gk + (size_t)nn * t.ldb : (size_t)nn + (size_t)gk * t.ldb;
        const int soff = B_KC ? (nn * kBK + kk) : (kk * BN + nn);
        cp_async8(sb + soff * ES + h * 8, v ? Bg + gi * ES + h * 8 : Bg, v ? 8 : 0);
      }
      return;
    }
    // A chunks
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
      const int gm = mm, gk = k0 + kk;
      int valid;
      const char* src;
      if (A_KC) {  // element (m,k) at A[k + m*lda]; chunk runs along k
        valid = (gm < M) ? max(0, min(EPC, K - gk)) : 0;
        src = Ag + ((size_t)gk + (size_t)gm * t.lda) * ES;
      } else {     // element (m,k) at A[m + k*lda]; chunk runs along m
        valid = (gk < K) ? max(0, min(EPC, M - gm)) : 0;
        src = Ag + ((size_t)gm + (size_t)gk * t.lda) * ES;
      }
      const int soff = A_KC ? (mm * kBK + kk) : (kk * BM + mm);
      cp_async16(sa + soff * ES, valid ? src : Ag, valid * ES);
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
      const int gn = nn, gk = k0 + kk;
      int valid;
      const char* src;
      if (B_KC) {  // element (k,n) at B[k + n*ldb]
        valid = (gn < N) ? max(0, min(EPC, K - gk)) : 0;
        src = Bg + ((size_t)gk + (size_t)gn * t.ldb) * ES;
      } else {     // element (k,n) at B[n + k*ldb]
        valid = (gk < K) ? max(0, min(EPC, N - gn)) : 0;
        src = Bg + ((size_t)gn + (size_t)gk * t.ldb) * ES;
      }
      const int soff = B_KC ? (nn * kBK + kk) : (kk * BN + nn);
      cp_async16(sb + soff * ES, valid ? src : Bg, valid * ES);
    }
  };

  const int wm = warp >> 2, wn = warp & 3;
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

  for (int s = 0; s < kSt - 1; ++s) {
    if (s < KT) load_stage(s, s);
    cp_async_commit();
  }
  for (int it = 0; it < KT; ++it) {
    cp_async_wait<kSt - 2>();
    __syncthreads();  // stage `it` landed for everyone; stage it-1 no longer read
    if (it + kSt - 1 < KT) load_stage(it + kSt - 1, (it + kSt - 1) % kSt);
    cp_async_commit();
    const uint8_t* sbase = smem + (it % kSt) * STAGE_BYTES;
    const S* sa = reinterpret_cast<const S*>(sbase);
    const S* sb = reinterpret_cast<const S*>(sbase + A_ELEMS * ES);
#pragma unroll
    for (int kc = 0; kc < kBK / 8; ++kc) {
      const int k0 = kc * 8 + 2 * tq, k1 = k0 + 1;
      double br[NF][2], bi[NF][2];
#pragma unroll
      for (int nf = 0; nf < NF; ++nf) {
        const int n = wn * WTN + nf * 8 + g;
        ld_elem<T>(sb, B_KC ? n * kBK + k0 : k0 * BN + n, br[nf][0], bi[nf][0]);
        ld_elem<T>(sb, B_KC ? n * kBK + k1 : k1 * BN + n, br[nf][1], bi[nf][1]);
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
  cp_async_wait<0>();
  __syncthreads();  // smem free for the next task
  S* C = reinterpret_cast<S*>(t.C);
  const bool use_beta = (t.br != 0.0) || (t.bi != 0.0);
#pragma unroll
  for (int mf = 0; mf < MF; ++mf)
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
          double vr = t.ar * xr - t.ai * xi;
          double vi = t.ar * xi + t.ai * xr;
          if (use_beta) {
            const double cr = __ldcg(C + 2 * idx), ci = __ldcg(C + 2 * idx + 1);
            vr += t.br * cr - t.bi * ci;
            vi += t.br * ci + t.bi * cr;
          }
          C[2 * idx] = vr;
          C[2 * idx + 1] = vi;
        } else {
          double v = t.ar * acc[mf][nf][i];
          if (use_beta) v = fma(t.br, __ldcg(C + idx), v);
          C[idx] = v;
        }
      }
}

// ---- trsm diagonal block ------------------------------------------------------
template <class T>
__device__ __forceinline__ void trsm_tile(const Task& t, uint8_t* smem) {
  constexpr bool CP = St<T>::CPLX;
  using S = typename St<T>::S;
  double (*Tr)[kLeafS + 1] = reinterpret_cast<double (*)[kLeafS + 1]>(smem);
  double (*Ti)[kLeafS + 1] =
      reinterpret_cast<double (*)[kLeafS + 1]>(smem + sizeof(double) * kLeafS * (kLeafS + 1));
  const int n = t.M, nrhs = t.N;
  const bool swap = t.flags & kFlagSwap, conj = t.flags & kFlagConj;
  const bool lower = t.flags & kFlagLower, unit = t.flags & kFlagUnit;
  const S* A = static_cast<const S*>(t.A);
  S* B = static_cast<S*>(t.C);
  for (int e = threadIdx.x; e < n * n; e += kThreads) {
    const int i = e % n, j = e / n;
    double re = 0, im = 0;
    if (lower ? (j <= i) : (j >= i)) {
      const size_t idx = swap ? (size_t)j + (size_t)i * t.lda : (size_t)i + (size_t)j * t.lda;
      if (CP) {
        re = __ldcg(A + 2 * idx);
        im = __ldcg(A + 2 * idx + 1);
        if (conj) im = -im;
      } else {
        re = __ldcg(A + idx);
      }
      if (i == j && unit) {
        re = 1.0;
        im = 0.0;
      }
    }
    Tr[i][j] = re;
    if (CP) Ti[i][j] = im;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = warp; c < nrhs; c += kThreads / 32) {
    double xr[2], xi[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = lane + 32 * h;
      xr[h] = xi[h] = 0.0;
      if (r < n) {
        const size_t idx = (size_t)r + (size_t)c * t.ldc;
        const double br = CP ? __ldcg(B + 2 * idx) : __ldcg(B + idx);
        const double bi = CP ? __ldcg(B + 2 * idx + 1) : 0.0;
        xr[h] = t.ar * br - t.ai * bi;
        xi[h] = CP ? (t.ar * bi + t.ai * br) : 0.0;
      }
    }
    for (int s = 0; s < n; ++s) {
      const int i = lower ? s : n - 1 - s;
      const int h = i >> 5, src = i & 31;
      double vr = __shfl_sync(0xffffffffu, h ? xr[1] : xr[0], src);
      double vi = CP ? __shfl_sync(0xffffffffu, h ? xi[1] : xi[0], src) : 0.0;
      const double dr = Tr[i][i], di = CP ? Ti[i][i] : 0.0;
      if (CP) {
        const double den = dr * dr + di * di;
        const double qr = (vr * dr + vi * di) / den, qi = (vi * dr - vr * di) / den;
        vr = qr;
        vi = qi;
      } else {
        vr = vr / dr;
      }
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int r = lane + 32 * hh;
        if (r == i) {
          xr[hh] = vr;
          xi[hh] = vi;
        } else if (r < n && (lower ? r > i : r < i)) {
          const double tr = Tr[r][i];
          if (CP) {
            const double ti = Ti[r][i];
            xr[hh] -= tr * vr - ti * vi;
            xi[hh] -= tr * vi + ti * vr;
          } else {
            xr[hh] -= tr * vr;
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = lane + 32 * h;
      if (r < n) {
        const size_t idx = (size_t)r + (size_t)c * t.ldc;
        if (CP) {
          B[2 * idx] = xr[h];
          B[2 * idx + 1] = xi[h];
        } else {
          B[idx] = xr[h];
        }
      }
    }
  }
  __syncthreads();
}

// smem: max(complex gemm 3 x 24 KB, complex trsm 2 x 33 KB) + alignment
constexpr size_t kSmemBytes = 3 * (32 + 64) * kBK * 16 + 128 > 2 * 8 * kLeafS * (kLeafS + 1) + 128
                                  ? 3 * (32 + 64) * kBK * 16 + 128
                                  : 2 * 8 * kLeafS * (kLeafS + 1) + 128;

__global__ void __launch_bounds__(kThreads) k_sched(const Task* __restrict__ tasks, int ntasks,
                                                    int* counters, int* next, int* call_left,
                                                    unsigned long long* call_end,
                                                    unsigned long long* t_start) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  __shared__ int s_idx, s_ok;
  if (threadIdx.x == 0) atomicMin(t_start, (unsigned long long)globaltimer());
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = atomicAdd(next, 1);
      int ok = 1;
      if (i < ntasks) {
        const Task* tp = tasks + i;
        if (tp->wait0 >= 0 && !wait_ge(counters + tp->wait0, tp->target0)) ok = 0;
        if (ok && tp->wait1 >= 0 && !wait_ge(counters + tp->wait1, tp->target1)) ok = 0;
        __threadfence();
      }
      s_idx = i;
      s_ok = ok;
    }
    __syncthreads();
    const int i = s_idx;
    if (i >= ntasks || !s_ok) break;
    const Task t = tasks[i];
    if (t.kind == kTaskGemm) {
      const bool akc = t.opA != XKB_OP_N, bkc = t.opB == XKB_OP_N;
      if (t.dtype == XKB_D) {
        if (akc && bkc) gemm_tile<double, true, true>(t, smem);
        else if (akc) gemm_tile<double, true, false>(t, smem);
        else if (bkc) gemm_tile<double, false, true>(t, smem);
        else gemm_tile<double, false, false>(t, smem);
      } else {
        if (akc && bkc) gemm_tile<double2, true, true>(t, smem);
        else if (akc) gemm_tile<double2, true, false>(t, smem);
        else if (bkc) gemm_tile<double2, false, true>(t, smem);
        else gemm_tile<double2, false, false>(t, smem);
      }
    } else {
      if (t.dtype == XKB_D) trsm_tile<double>(t, smem);
      else trsm_tile<double2>(t, smem);
    }
    __syncthreads();  // every output of the task is stored
    if (threadIdx.x == 0) {
      __threadfence();
      if (t.signal >= 0) atomicAdd(counters + t.signal, 1);
      if (atomicSub(call_left + t.call, 1) == 1) call_end[t.call] = globaltimer();
    }
  }
}

// ---------------------------------------------------------------------------
// host: task list construction
struct Built {
  std::vector<Task> tasks;
  std::vector<int> call_tasks;
  int ncounters = 0;
};

static int esz(int dt) { return dt == XKB_Z ? 16 : 8; }

static bool aligned_ok(const void* p, long ld, int es) {
  return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && ((ld * es) % 16 == 0);
}

static bool ptr8(const void* p) { return reinterpret_cast<uintptr_t>(p) % 8 == 0; }

static int add_gemm(Built& b, const xkb_batch_op& o, int call) {
  const int es = esz(o.dtype);
  const int BM = o.dtype == XKB_Z ? 32 : 64, BN = 64;
  if (!ptr8(o.A) || !ptr8(o.B) || !ptr8(o.C)) return XKB_EINVAL;
  const int narrow =
      (aligned_ok(o.A, o.lda, es) && aligned_ok(o.B, o.ldb, es)) ? 0 : kFlagNarrow;
  const char* A = static_cast<const char*>(o.A);
  const char* B = static_cast<const char*>(o.B);
  char* C = static_cast<char*>(o.C);
  int n = 0;
  for (int n0 = 0; n0 < o.N; n0 += BN)
    for (int m0 = 0; m0 < o.M; m0 += BM) {
      Task t;
      std::memset(&t, 0, sizeof(t));
      t.kind = kTaskGemm;
      t.dtype = o.dtype;
      t.opA = o.opA;
      t.opB = o.opB;
      t.M = std::min(BM, o.M - m0);
      t.N = std::min(BN, o.N - n0);
      t.K = o.K;
      t.call = call;
      t.A = o.opA == XKB_OP_N ? A + (size_t)m0 * es : A + (size_t)m0 * o.lda * es;
      t.B = o.opB == XKB_OP_N ? B + (size_t)n0 * o.ldb * es : B + (size_t)n0 * es;
      t.C = C + ((size_t)m0 + (size_t)n0 * o.ldc) * es;
      t.lda = o.lda;
      t.ldb = o.ldb;
      t.ldc = o.ldc;
      t.ar = o.alpha[0];
      t.ai = o.alpha[1];
      t.br = o.beta[0];
      t.bi = o.beta[1];
      t.flags = narrow;
      t.wait0 = t.wait1 = -1;
      t.signal = -1;
      b.tasks.push_back(t);
      ++n;
    }
  return n;
}

// Left triangular solve as the reference's tile algorithm (blas/ztrsm.c):
// diagonal solves + trailing gemm updates with lalpha on the first step.
static int add_trsm(Built& b, const xkb_batch_op& o, int call,
                    std::vector<std::vector<Task>>& steps) {
  const int es = esz(o.dtype);
  if (o.side != 0) return XKB_EINVAL;  // right side: not a batch task
  if (!ptr8(o.A) || !ptr8(o.C)) return XKB_EINVAL;
  const int narrow =
      (aligned_ok(o.A, o.lda, es) && aligned_ok(o.C, o.ldc, es)) ? 0 : kFlagNarrow;
  const bool cplx = o.dtype == XKB_Z;
  const int trans = (!cplx && o.trans == XKB_OP_C) ? XKB_OP_T : o.trans;
  const bool lower_eff = (o.uplo == XKB_LOWER) ^ (trans != XKB_OP_N);
  const int mt = (o.M + kLeafS - 1) / kLeafS, nt = (o.N + kLeafS - 1) / kLeafS;
  const int cb = b.ncounters;
  b.ncounters += mt * nt;
  auto cnt = [&](int blk, int j) { return cb + blk + j * mt; };
  auto order = [&](int s) { return lower_eff ? s : mt - 1 - s; };
  auto rows = [&](int blk) { return std::min(kLeafS, o.M - blk * kLeafS); };
  const char* A = static_cast<const char*>(o.A);
  char* X = static_cast<char*>(o.C);
  int n = 0;
  for (int s = 0; s < mt; ++s) {
    const int bk = order(s);
    steps.emplace_back();
    std::vector<Task>& out = steps.back();
    for (int j = 0; j < nt; ++j) {
      Task t;
      std::memset(&t, 0, sizeof(t));
      t.kind = kTaskTrsmDiag;
      t.dtype = o.dtype;
      t.M = rows(bk);
      t.N = std::min(kLeafS, o.N - j * kLeafS);
      t.call = call;
      t.A = A + ((size_t)bk * kLeafS + (size_t)bk * kLeafS * o.lda) * es;
      t.C = X + ((size_t)bk * kLeafS + (size_t)j * kLeafS * o.ldc) * es;
      t.lda = o.lda;
      t.ldc = o.ldc;
      t.ar = s == 0 ? o.alpha[0] : 1.0;
      t.ai = s == 0 ? o.alpha[1] : 0.0;
      t.flags = (trans != XKB_OP_N ? kFlagSwap : 0) | (trans == XKB_OP_C ? kFlagConj : 0) |
                (lower_eff ? kFlagLower : 0) | (o.diag ? kFlagUnit : 0);
      t.wait0 = cnt(bk, j);
      t.target0 = s;  // the s updates from earlier steps are in
      t.wait1 = -1;
      t.signal = cnt(bk, j);
      out.push_back(t);
      ++n;
    }
    for (int p = s + 1; p < mt; ++p) {  // next diagonal block first (look-ahead)
      const int bi = order(p);
      for (int j = 0; j < nt; ++j) {
        Task t;
        std::memset(&t, 0, sizeof(t));
        t.kind = kTaskGemm;
        t.dtype = o.dtype;
        t.M = rows(bi);
        t.N = std::min(kLeafS, o.N - j * kLeafS);
        t.K = rows(bk);
        t.call = call;
        // op(A)[bi rows, bk cols] = trans N: A[bi, bk]; else op(A[bk, bi])
        if (trans == XKB_OP_N) {
          t.opA = XKB_OP_N;
          t.A = A + ((size_t)bi * kLeafS + (size_t)bk * kLeafS * o.lda) * es;
        } else {
          t.opA = trans;
          t.A = A + ((size_t)bk * kLeafS + (size_t)bi * kLeafS * o.lda) * es;
        }
        t.opB = XKB_OP_N;
        t.B = X + ((size_t)bk * kLeafS + (size_t)j * kLeafS * o.ldc) * es;
        t.C = X + ((size_t)bi * kLeafS + (size_t)j * kLeafS * o.ldc) * es;
        t.lda = o.lda;
        t.ldb = o.ldc;
        t.ldc = o.ldc;
        t.ar = -1.0;
        t.ai = 0.0;
        t.br = s == 0 ? o.alpha[0] : 1.0;
        t.bi = s == 0 ? o.alpha[1] : 0.0;
        t.wait0 = cnt(bk, j);
        t.target0 = s + 1;  // X_bk solved
        t.wait1 = cnt(bi, j);
        t.target1 = s;      // earlier updates of this block applied
        t.signal = cnt(bi, j);
        t.flags = narrow;
        out.push_back(t);
        ++n;
      }
    }
  }
  return n;
}

struct Batch {
  Task* h_tasks = nullptr;  // pinned
  size_t cap = 0;
  Task* d_tasks = nullptr;
  int* d_counters = nullptr;  // counters, next, call_left (contiguous)
  unsigned long long* d_times = nullptr;  // call_end[ncalls], t_start
  size_t d_cap_tasks = 0, d_cap_ints = 0, d_cap_times = 0;
  int ntasks = 0, ncalls = 0, nctr = 0;
  std::vector<int> call_tasks;
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

}  // namespace sched
}  // namespace xkb

using namespace xkb;
using namespace xkb::sched;

extern "C" int xkb_cuda_batch(const xkb_batch_op* ops, int nops, int schedule, void* stream) {
  if (!ops || nops < 0) return XKB_EINVAL;
  if (nops == 0) return XKB_OK;
  std::lock_guard<std::mutex> g(g_batch_mu);
  cudaStream_t st = resolve_stream(stream);
  Built b;
  b.call_tasks.assign(nops, 0);
  std::vector<std::vector<std::vector<Task>>> solves;  // per solve: its steps
  for (int c = 0; c < nops; ++c) {
    const xkb_batch_op& o = ops[c];
    if ((o.dtype != XKB_D && o.dtype != XKB_Z) || o.M < 0 || o.N < 0 || o.K < 0) return XKB_EINVAL;
    if (o.M == 0 || o.N == 0) continue;
    if (o.kind == XKB_BATCH_GEMM) {
      if (o.K == 0) return XKB_EINVAL;  // beta-only calls are not batch tasks
      const int n = add_gemm(b, o, c);
      if (n < 0) return n;
      b.call_tasks[c] = n;
    } else if (o.kind == XKB_BATCH_TRSM) {
      std::vector<std::vector<Task>> st_steps;
      const int n = add_trsm(b, o, c, st_steps);
      if (n < 0) return n;
      b.call_tasks[c] = n;
      solves.push_back(std::move(st_steps));
    } else {
      return XKB_EINVAL;
    }
  }
  // schedule 0: gemm tiles in call order, then the solves step by step;
  // schedule 1: interleave -- step s of every solve, then an equal share of
  // the gemm tiles, so dependent steps sit far apart in the claim order
  std::vector<Task> gemms;
  gemms.swap(b.tasks);
  std::vector<Task>& out = b.tasks;
  size_t longest = 0;
  for (auto& sv : solves) longest = std::max(longest, sv.size());
  if (schedule == 0 || solves.empty()) {
    out = gemms;
    for (size_t st2 = 0; st2 < longest; ++st2)
      for (auto& sv : solves)
        if (st2 < sv.size()) out.insert(out.end(), sv[st2].begin(), sv[st2].end());
  } else {
    const size_t chunk = (gemms.size() + longest) / (longest + 1);
    size_t gi = 0;
    for (size_t st2 = 0; st2 < longest; ++st2) {
      for (auto& sv : solves)
        if (st2 < sv.size()) out.insert(out.end(), sv[st2].begin(), sv[st2].end());
      const size_t ge = std::min(gemms.size(), gi + chunk);
      out.insert(out.end(), gemms.begin() + gi, gemms.begin() + ge);
      gi = ge;
    }
    out.insert(out.end(), gemms.begin() + gi, gemms.end());
  }
  Batch& B = batch();
  const int ntasks = (int)out.size();
  B.ntasks = ntasks;
  B.ncalls = nops;
  B.call_tasks = b.call_tasks;
  if (ntasks == 0) return XKB_OK;
  // the previous batch may still read the pinned staging buffer
  if (B.h_tasks) cudaStreamSynchronize(st);
  if ((size_t)ntasks > B.cap) {
    if (B.h_tasks) cudaFreeHost(B.h_tasks);
    B.cap = (size_t)ntasks * 2;
    if (cudaHostAlloc(&B.h_tasks, B.cap * sizeof(Task), cudaHostAllocDefault) != cudaSuccess) {
      B.h_tasks = nullptr;
      B.cap = 0;
      return XKB_ENOMEM;
    }
  }
  std::memcpy(B.h_tasks, out.data(), (size_t)ntasks * sizeof(Task));
  const size_t nints = (size_t)b.ncounters + 1 + (size_t)nops;
  if ((size_t)ntasks > B.d_cap_tasks) {
    if (B.d_tasks) cudaFreeAsync(B.d_tasks, st);
    B.d_cap_tasks = (size_t)ntasks * 2;
    if (cudaMallocAsync(&B.d_tasks, B.d_cap_tasks * sizeof(Task), st) != cudaSuccess) {
      B.d_tasks = nullptr;
      B.d_cap_tasks = 0;
      return XKB_ENOMEM;
    }
  }
  if (nints > B.d_cap_ints) {
    if (B.d_counters) cudaFreeAsync(B.d_counters, st);
    B.d_cap_ints = nints * 2;
    if (cudaMallocAsync(&B.d_counters, B.d_cap_ints * sizeof(int), st) != cudaSuccess) {
      B.d_counters = nullptr;
      B.d_cap_ints = 0;
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
  int* d_next = B.d_counters + b.ncounters;
  int* d_left = d_next + 1;
  cudaMemcpyAsync(B.d_tasks, B.h_tasks, (size_t)ntasks * sizeof(Task), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(B.d_counters, 0, (size_t)(b.ncounters + 1) * sizeof(int), st);
  cudaMemcpyAsync(d_left, b.call_tasks.data(), (size_t)nops * sizeof(int), cudaMemcpyHostToDevice,
                  st);
  cudaMemsetAsync(B.d_times, 0, (size_t)nops * sizeof(unsigned long long), st);
  cudaMemsetAsync(B.d_times + nops, 0xff, sizeof(unsigned long long), st);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_sched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSmemBytes) != cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  const int grid = std::min(grid_size(), std::max(1, ntasks));
  k_sched<<<grid, kThreads, kSmemBytes, st>>>(B.d_tasks, ntasks, B.d_counters, d_next, d_left,
                                              B.d_times, B.d_times + nops);
  count_launch();
  // the pinned staging buffer must outlive the copy: the copy is ordered
  // before the kernel, and the next batch synchronises before reusing it
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

extern "C" int xkb_cuda_batch_latency(double* ms, int n) {
  Batch& B = batch();
  std::lock_guard<std::mutex> g(g_batch_mu);
  if (!ms || n < 0 || n > B.ncalls || !B.d_times) return XKB_EINVAL;
  if (cudaDeviceSynchronize() != cudaSuccess) return XKB_ECUDA;
  std::vector<unsigned long long> t((size_t)B.ncalls + 1);
  if (cudaMemcpy(t.data(), B.d_times, t.size() * sizeof(unsigned long long),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return XKB_ECUDA;
  const unsigned long long t0 = t[B.ncalls];
  for (int i = 0; i < n; ++i)
    ms[i] = (B.call_tasks[i] && t[i] >= t0) ? (double)(t[i] - t0) * 1e-6 : 0.0;
  return XKB_OK;
}
