// ozaki.cu -- FP64-accurate contraction on INT8 tensor cores (Ozaki scheme II).
//
// No counterpart in the reference (whose tile bodies call cuBLAS DGEMM,
// blas/ztask_gemm.c:206); selected by xkblas_set_modemath(XKBLAS_TENSOR_OP_MATH)
// or XKBLAS_DEFAULT_MATH=TC, the reference's switch for tensor-core math
// (blas/xkblas.h:100-107, blas/ztask_gemm.c:182-196).
//
// Method (Ozaki, Uchino, Imamura, "Ozaki Scheme II: a GEMM-oriented emulation
// of floating-point matrix multiplication using an integer modular
// technique", 2025), restated:
//   1. each row i of op(A) is scaled by 2^mu_i and each column j of op(B) by
//      2^nu_j and rounded to integers A', B' (|A'|,|B'| < 2^62), with the
//      shifts chosen from the 2-norms so that |A' B'| (Cauchy-Schwarz) stays
//      below P/2, P = p_1 ... p_n the product of the moduli;
//   2. for every modulus p_l (pairwise coprime, <= 256) the symmetric
//      residues A' mod p_l, B' mod p_l fit in int8 and their product is
//      computed EXACTLY on the tensor cores (tcgen05.mma kind::i8, INT32
//      accumulation in TMEM; K * 128^2 < 2^31 for K <= 131072), then reduced
//      mod p_l;
//   3. the n residues of each C entry are recombined by the Chinese remainder
//      theorem on the FP64 pipe (CRT weights split into an exact high part
//      and a rounded low part, the quotient by P exact; see crt_value),
//      mapped to the symmetric range and scaled back by 2^-(mu_i + nu_j);
//      alpha/beta are applied in FP64.
// With n = 16 moduli P ~ 2^125.4, so each operand keeps ~61 bits relative to
// its row / column 2-norm: the contraction error is below FP64 DGEMM's.
//
// Kernels: k_oz_norm (per-row / per-column scaling), k_oz_residues (scale,
// round, reduce to int8 planes in the K-major layout TMA reads), k_oz_gemm
// (TMA -> 4-stage smem ring -> tcgen05.mma -> TMEM -> mod-p epilogue, one
// launch for all moduli), k_oz_crt (reconstruction + alpha/beta + mask).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "xkb_dev.cuh"

namespace xkb {
namespace oz {

constexpr int kMaxMod = 16;

struct Consts {
  int nmod;
  int H;                       // scaled operands stay below 2^H in 2-norm
  int p[kMaxMod];
  float invp_f[kMaxMod];
  double invp_d[kMaxMod];
  uint32_t wlo[kMaxMod], whi[kMaxMod];  // bytes of 2^(8t) mod p, t = 0..3, 4..7
  uint32_t off[kMaxMod];                // p - (2^62 mod p): undoes the +2^62 offset
  uint32_t offh[kMaxMod];               // off + floor(p/2): symmetric residues
  uint32_t magic[kMaxMod];              // ceil(2^32 / p): exact quotients below 2^21
  int half[kMaxMod];                    // floor(p/2)
  // CRT weights w = (P/p)((P/p)^-1 mod p) mod P split as w = w1 + w2: w1 the
  // bits of w from 2^csplit up (exact double, <= 41 significant bits), w2
  // the rest rounded to double; P = P1 + P2 the same way
  double w1[kMaxMod], w2[kMaxMod];
  double P1d, P2d, Pd, invPd;
};

// ---------------------------------------------------------------------------
// host: moduli and CRT constants
typedef unsigned __int128 u128;

static std::vector<int> moduli_list() {
  std::vector<int> m;
  for (int c = 256; c >= 2 && (int)m.size() < kMaxMod; --c) {
    bool ok = true;
    for (int q : m) {
      int a = c, b = q;
      while (b) {
        int t = a % b;
        a = b;
        b = t;
      }
      if (a != 1) {
        ok = false;
        break;
      }
    }
    if (ok) m.push_back(c);
  }
  return m;
}

static u128 mulmod(u128 a, u128 b, u128 m) {  // a, b < m < 2^127
  u128 r = 0;
  a %= m;
  while (b) {
    if (b & 1) {
      r += a;
      if (r >= m) r -= m;
    }
    a += a;
    if (a >= m) a -= m;
    b >>= 1;
  }
  return r;
}

static int inv_mod(int a, int p) {  // a^-1 mod p, gcd(a,p) = 1
  int t = 0, nt = 1, r = p, nr = ((a % p) + p) % p;
  while (nr) {
    int q = r / nr, tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return t < 0 ? t + p : t;
}

static double log2P(int n) {
  std::vector<int> m = moduli_list();
  double s = 0;
  for (int i = 0; i < n; ++i) s += std::log2((double)m[i]);
  return s;
}

static bool make_consts(int n, Consts* c) {
  if (n < 2 || n > kMaxMod) return false;
  std::vector<int> m = moduli_list();
  std::memset(c, 0, sizeof(*c));
  c->nmod = n;
  u128 P = 1;
  for (int i = 0; i < n; ++i) P *= (u128)m[i];
  // budget: ||A'_i||_2 ||B'_j||_2 <= 2^(2H) (1+tiny) < P/2
  c->H = (int)std::floor((log2P(n) - 1.0) / 2.0) - 1;
  // split point of the CRT weights: sum_l r_l w1_l < 4080 P < 2^(bits(P)+12)
  // must be an integer multiple of 2^csplit below 2^(53+csplit)
  int bitsP = 0;
  for (u128 t = P; t; t >>= 1) ++bitsP;
  const int csplit = std::max(0, bitsP + 12 - 53);
  const u128 low = csplit ? (((u128)1 << csplit) - 1) : 0;
  for (int i = 0; i < n; ++i) {
    const int p = m[i];
    c->p[i] = p;
    c->invp_f[i] = std::nextafter(1.0f / (float)p, 0.0f);  // <= 1/p (see k_oz_residues)
    c->invp_d[i] = 1.0 / (double)p;
    uint32_t lo = 0, hi = 0;
    for (int t = 0; t < 8; ++t) {
      uint64_t w = 1;
      for (int s = 0; s < 8 * t; ++s) w = (w * 2) % (uint64_t)p;
      if (t < 4) lo |= (uint32_t)w << (8 * t);
      else hi |= (uint32_t)w << (8 * (t - 4));
    }
    c->wlo[i] = lo;
    c->whi[i] = hi;
    uint64_t t62 = 1;
    for (int s2 = 0; s2 < 62; ++s2) t62 = (t62 * 2) % (uint64_t)p;
    c->off[i] = (uint32_t)((uint64_t)p - t62);
    c->half[i] = p / 2;
    c->offh[i] = c->off[i] + (uint32_t)(p / 2);
    c->magic[i] = (uint32_t)(((1ull << 32) + (uint64_t)p - 1) / (uint64_t)p);
    const u128 Mi = P / (u128)p;
    const int inv = inv_mod((int)(Mi % (u128)p), p);
    const u128 w = mulmod(Mi, (u128)inv, P);
    c->w1[i] = std::ldexp((double)(uint64_t)(w >> csplit), csplit);  // < 2^41 units: exact
    c->w2[i] = (double)(w & low);
  }
  c->P1d = std::ldexp((double)(uint64_t)(P >> csplit), csplit);
  c->P2d = (double)(P & low);
  c->Pd = (double)P;
  c->invPd = 1.0 / c->Pd;
  return true;
}

// ---------------------------------------------------------------------------
// 1. scaling exponents and the moduli count.  View the operand as L "rows"
//    of length K, element (l,k) at X[l*sl + k*sk] (one of sl, sk is 1).
//    Partial sums over k-chunks go to part[chunk][l] = (sum of squares,
//    max |x|, sum |x|, nonzero count); k_oz_stat finalises each row.
constexpr int kNormChunk = 512;

// The moduli count of a call, chosen on the device (k_oz_pick) and read by
// every later kernel of the call: n moduli (0: the plain FP64 kernel runs
// instead), H the exponent budget of the scaled operands for that count.
struct OzSel {
  int n, H, fallback, pad;
};

// Counters over all contractions of the process (xkb_ozaki_counts).
static __device__ unsigned long long g_oz_calls, g_oz_mod_sum, g_oz_fallbacks;
static __device__ int g_oz_last = -1;

template <bool KC>  // KC: k contiguous (sk == 1)
__global__ void __launch_bounds__(256) k_oz_norm(int L, int K, const double* X, long ld, int cplx,
                                                  double4* part) {
  // block: 32 rows x 8 lanes along k (KC: warp-cooperative along k instead)
  const int chunk = blockIdx.y;
  const int k0 = chunk * kNormChunk, k1 = min(K, k0 + kNormChunk);
  double ss = 0.0, mx = 0.0, s1 = 0.0, nz = 0.0;
  auto acc = [&](double v) {
    ss = fma(v, v, ss);
    mx = fmax(mx, fabs(v));
    s1 += fabs(v);
    nz += (v != 0.0) ? 1.0 : 0.0;
  };
  if constexpr (KC) {
    // one warp per row: lanes stride along contiguous k
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * 8 + warp;
    if (l < L) {
      for (int k = k0 + lane; k < k1; k += 32) {
        if (cplx) {
          acc(X[2 * ((size_t)k + (size_t)l * ld)]);
          acc(X[2 * ((size_t)k + (size_t)l * ld) + 1]);
        } else {
          acc(X[(size_t)k + (size_t)l * ld]);
        }
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      ss += __shfl_xor_sync(0xffffffffu, ss, o);
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    if (lane == 0 && l < L) part[(size_t)chunk * L + l] = make_double4(ss, mx, s1, nz);
  } else {
    // l contiguous: 32 consecutive rows per warp-row, 8 k-lanes
    __shared__ double4 red[8][32];
    const int tl = threadIdx.x & 31, tk = threadIdx.x >> 5;
    const int l = blockIdx.x * 32 + tl;
    if (l < L) {
      for (int k = k0 + tk; k < k1; k += 8) {
        if (cplx) {
          acc(X[2 * ((size_t)l + (size_t)k * ld)]);
          acc(X[2 * ((size_t)l + (size_t)k * ld) + 1]);
        } else {
          acc(X[(size_t)l + (size_t)k * ld]);
        }
      }
    }
    red[tk][tl] = make_double4(ss, mx, s1, nz);
    __syncthreads();
    if (tk == 0 && l < L) {
      double4 t = red[0][tl];
      for (int i = 1; i < 8; ++i) {
        t.x += red[i][tl].x;
        t.y = fmax(t.y, red[i][tl].y);
        t.z += red[i][tl].z;
        t.w += red[i][tl].w;
      }
      part[(size_t)chunk * L + l] = t;
    }
  }
}

// 2^e as a double for -1022 <= e <= 1023 (exact, no libm call)
__device__ __forceinline__ double pow2(int e) {
  return __longlong_as_double((long long)(1023 + e) << 52);
}

// Row codes written by k_oz_stat: the exponent e of a bound nrm < 2^e of the
// row's 2-norm, or one of two sentinels.  The shift of the row is H - e.
constexpr int kShiftNonFinite = -100000;  // the row holds Inf/NaN: results NaN
constexpr int kCodeZero = 100000;         // all-zero row: shift 0

__device__ __forceinline__ int shift_of(int code, int H) {
  if (code == kShiftNonFinite) return kShiftNonFinite;
  if (code == kCodeZero) return 0;
  return max(-1000, min(1000, H - code));  // scaled values stay finite
}

// Per row: the code above, and the row's concentration
// rho = sqrt(nnz) ||x||_2 / ||x||_1 (1 for entries of one magnitude, up to
// sqrt(nnz) for one dominant entry), whose maximum over the rows goes to
// *rmax (a non-negative float compared as its bits).
__global__ void k_oz_stat(int L, int K, int nchunks, const double4* part, int* code,
                          unsigned* rmax) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  float rho = 0.0f;
  if (l < L) {
    double ss = 0.0, mx = 0.0, s1 = 0.0, nz = 0.0;
    for (int c = 0; c < nchunks; ++c) {  // fixed order: deterministic
      const double4 v = part[(size_t)c * L + l];
      ss += v.x;
      mx = fmax(mx, v.y);
      s1 += v.z;
      nz += v.w;
    }
    if (!isfinite(mx) || isnan(ss)) {
      code[l] = kShiftNonFinite;
    } else if (mx == 0.0) {
      code[l] = kCodeZero;
    } else {
      // bound on the row 2-norm (the sum of squares may overflow for huge entries)
      double nrm = isfinite(ss) ? sqrt(ss) : mx * sqrt((double)K);
      nrm = fmax(nrm, mx) * (1.0 + 1e-12);
      int e;
      frexp(nrm, &e);  // nrm < 2^e
      code[l] = e;
      // scale-free form: sqrt(nnz) * (nrm / mx) / (s1 / mx), all ratios <= nnz
      const double r = sqrt(nz) * (nrm / mx) / fmax(s1 / mx, 1.0);
      rho = (float)fmin(r, 3.0e38);
    }
  }
  // warp maximum, one atomic per warp
#pragma unroll
  for (int o = 16; o; o >>= 1) rho = fmaxf(rho, __shfl_xor_sync(0xffffffffu, rho, o));
  if ((threadIdx.x & 31) == 0 && rho > 0.0f) atomicMax(rmax, __float_as_uint(rho));
}

// Moduli-count rule.  The scaled, rounded operands lose at most half a unit
// per nonzero entry; with errors of random sign the contraction error
// relative to sum_k |a_ik||b_kj| is about 0.58 rho_i sigma_j 2^-H, and its
// maximum over many entries about four times that (rho, sigma: the
// concentrations of row i of op(A) and column j of op(B)).  The smallest
// count with 2.31 rho_max sigma_max 2^-H <= 2^-53 keeps the result within
// FP64 rounding; if the largest count cannot, the call runs the plain FP64
// kernel instead (fallback = 1), or, where that is not allowed, the largest
// count.  fixed > 0: that count, no data rule.
struct PickP {
  int fixed, lo, hi, allow_fallback;
  int H[kMaxMod + 1];  // exponent budget per count
};

__global__ void k_oz_pick(const unsigned* rmax, OzSel* sel, const PickP q) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n = q.fixed, fb = 0;
  if (n <= 0) {
    const double ra = fmax(1.0, (double)__uint_as_float(rmax[0]));
    const double rb = fmax(1.0, (double)__uint_as_float(rmax[1]));
    const double need = 53.0 + log2(2.31 * ra * rb);
    n = 0;
#pragma unroll
    for (int c = kMaxMod; c >= 2; --c)  // constant indices: no local copy of q.H
      if (c >= q.lo && c <= q.hi && (double)q.H[c] >= need) n = c;
    if (n == 0) {
      if (q.allow_fallback) fb = 1;
      else n = q.hi;
    }
  }
  sel->n = n;
  sel->H = n ? q.H[n] : 0;
  sel->fallback = fb;
  sel->pad = 0;
  atomicAdd(&g_oz_calls, 1ull);
  atomicAdd(&g_oz_mod_sum, (unsigned long long)n);
  if (fb) atomicAdd(&g_oz_fallbacks, 1ull);
  g_oz_last = n;
}

// ---------------------------------------------------------------------------
// 2. residues: planes[m][l][k] (int8, row stride Kpad) for l < Lpad, k < Kpad
//    (zero padding), from X (L x K view, KC: k contiguous).  Complex operands
//    (cplx = 1) are handled by the caller through the concatenated views.
// Residue planes 1 .. min(CNT, n) - 1 of four consecutive elements whose
// offset values a' = a + 2^62 have 32-bit halves lo, hi (plane 0 is written
// by the caller).
template <int CNT>
__device__ __forceinline__ void res_planes(const Consts& c, const uint32_t (&lo)[4],
                                           const uint32_t (&hi)[4], int8_t* dst, size_t plane,
                                           int n) {
#pragma unroll
  for (int m = 1; m < CNT; ++m) {
    if (m >= n) break;
    const uint32_t p = (uint32_t)c.p[m];
    uint32_t r[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      // s = a' mod p + h (mod p) from the bytes of a': offh + sum_t byte_t
      // (2^(8t) mod p) < 2^21; q = floor(s / p) exactly by the 32-bit
      // reciprocal ceil(2^32 / p) (error s * 2^-32 < 1/p); s - q p - h is
      // the symmetric residue in [-h, h]
      uint32_t sacc = __dp4a(lo[v], c.wlo[m], c.offh[m]);
      sacc = __dp4a(hi[v], c.whi[m], sacc);
      const uint32_t q = __umulhi(sacc, c.magic[m]);
      r[v] = sacc - q * p - (uint32_t)c.half[m];
    }
    *reinterpret_cast<uint32_t*>(dst + (size_t)m * plane) =
        __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
  }
}

template <bool KC, int NM>
__global__ void __launch_bounds__(256) k_oz_residues(int L, int K, const double* X, long ld,
                                                      long estride, long eoff, double esign,
                                                      const int* code, const OzSel* sel,
                                                      const Consts c, int8_t* planes, long Lpad,
                                                      long Kpad, long kofs) {
  // X element (l,k) = esign * X[eoff + estride*(KC ? k + l*ld : l + k*ld)];
  // planes 0 .. sel->n - 1 are written (NM: the most the call may use)
  const int nm = sel->n, H = sel->H;
  if (nm == 0) return;  // the plain kernel computes this call
  __shared__ double tile[64][65];
  const int l0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  {
    // all 16 loads of a thread in flight before the shared stores
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = threadIdx.x + q * 256;
      const int ll = KC ? e >> 6 : e & 63, kk = KC ? e & 63 : e >> 6;
      const int l = l0 + ll, k = k0 + kk;
      v[q] = 0.0;
      if (l < L && k < K) {
        const size_t idx = KC ? (size_t)k + (size_t)l * ld : (size_t)l + (size_t)k * ld;
        v[q] = esign * X[eoff + estride * idx];
      }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = threadIdx.x + q * 256;
      const int ll = KC ? e >> 6 : e & 63, kk = KC ? e & 63 : e >> 6;
      tile[ll][kk] = v[q];
    }
  }
  __syncthreads();
  const size_t plane = (size_t)Lpad * (size_t)Kpad;
  for (int it = threadIdx.x; it < 64 * 16; it += 256) {
    const int ll = it >> 4, kq = (it & 15) * 4;
    const int l = l0 + ll;
    const int s = (l < L) ? shift_of(code[l], H) : 0;
    // a' = a + 2^62 >= 0 (|a| < 2^62); residues of a' are shifted back by the
    // per-modulus constant folded into c.off (no sign handling per modulus)
    const double sc = (s == kShiftNonFinite) ? 0.0 : pow2(s / 2) * pow2(s - s / 2);
    long long a[4];
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double x = tile[ll][kq + v] * sc;  // exact power-of-two scaling
      a[v] = llrint(x);
      const unsigned long long u = (unsigned long long)a[v] + (1ull << 62);
      lo[v] = (uint32_t)u;
      hi[v] = (uint32_t)(u >> 32);
    }
    int8_t* dst = planes + (size_t)l * Kpad + kofs + k0 + kq;
    // p_0 = 256: the two's complement low byte (the offset 2^62 is 0 mod 256)
    *reinterpret_cast<uint32_t*>(dst) =
        __byte_perm(__byte_perm(lo[0], lo[1], 0x0040), __byte_perm(lo[2], lo[3], 0x0040), 0x5410);
    // planes 1 .. nm-1, unrolled for the plan's largest count and the one
    // below it (the data rule's two counts); other counts take a loop
    if (nm == NM) res_planes<NM>(c, lo, hi, dst, plane, NM);
    else if (NM > 2 && nm == NM - 1)
      res_planes<(NM > 2 ? NM - 1 : NM)>(c, lo, hi, dst, plane, NM - 1);
    else res_planes<NM>(c, lo, hi, dst, plane, nm);
  }
}

// ---------------------------------------------------------------------------
// 3. INT8 tensor-core GEMM: persistent CTAs (one per SM) walking the
//    (modulus, 128 x 256 C tile) list.  Warp 0: TMA producer into a 4-stage
//    ring; warp 1: TMEM allocator (512 columns = two 256-column accumulators)
//    and single-thread MMA issuer; warps 2-5: epilogue.  The accumulator is
//    double buffered, so the epilogue of tile i (TMEM -> registers -> mod p ->
//    uint8 plane) runs while the MMAs of tile i+1 fill the other buffer.
constexpr int BM = 128, BN = 256, BKB = 128;  // BKB: k bytes per stage
constexpr int S = 4;
constexpr uint32_t A_STAGE = BM * BKB, B_STAGE = BN * BKB;
constexpr int kGemmThreads = 192;
constexpr uint32_t kTmemCols = 512;  // two accumulators of BN columns
constexpr int kEpiWarps = 4;

struct GemmP {
  int tiles_m, tiles_n, kblocks, nmod;  // nmod: planes of the operand buffers (the most used)
  const OzSel* sel;                     // moduli multiplied: sel->n (<= nmod)
  int group;  // raster: M tiles per group (tiles in flight share A / B panels in L2)
  uint8_t* R;
  long Mpad, Npad;
  int uplo;
  long diag;
  int p[kMaxMod];
  double invp[kMaxMod];
};

__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused, K-major swizzled)
  d |= (uint64_t)(1024 >> 4) << 32;          // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                    // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                    // 128-byte swizzle
  return d;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_mma_i8(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                          uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* m, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// tile t of the (modulus-major, grouped raster) list; false if the tile lies
// wholly outside the written triangle
__device__ __forceinline__ bool oz_tile(const GemmP& p, int t, int& mod, int& m0, int& n0) {
  const int tiles_mn = p.tiles_m * p.tiles_n;
  mod = t / tiles_mn;
  const int r = t - mod * tiles_mn;
  const int GROUP = p.group;
  const int span = GROUP * p.tiles_n;
  const int first_m = (r / span) * GROUP;
  const int gsz = min(p.tiles_m - first_m, GROUP);
  const int tm = first_m + (r % span) % gsz;
  const int tn = (r % span) / gsz;
  m0 = tm * BM;
  n0 = tn * BN;
  if (p.uplo == XKB_LOWER && (long)(m0 + BM - 1) + p.diag < (long)n0) return false;
  if (p.uplo == XKB_UPPER && (long)m0 + p.diag > (long)(n0 + BN - 1)) return false;
  return true;
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_oz_gemm(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
              const GemmP p) {
  extern __shared__ uint8_t sm_raw[];
  uint8_t* sm =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = sm;
  uint8_t* sB = sm + S * A_STAGE;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + S * B_STAGE);
  uint64_t* empty = full + S;
  uint64_t* accf = empty + S;  // [2] accumulator ready
  uint64_t* acce = accf + 2;   // [2] accumulator drained
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);

  const int total = p.tiles_m * p.tiles_n * min(p.sel->n, p.nmod);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], kEpiWarps);
    }
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tslot);
  const int KB = p.kblocks;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer
      tma_prefetch(&tA);
      tma_prefetch(&tB);
      uint32_t it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        int mod, m0, n0;
        if (!oz_tile(p, t, mod, m0, n0)) continue;
        for (int kb = 0; kb < KB; ++kb, ++it) {
          const int s = it % S;
          const uint32_t ph = (it / S) & 1;
          if (!mbar_wait(&empty[s], ph ^ 1, kErrEmptyWait)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], A_STAGE + B_STAGE);
          tma_load_3d(sA + s * A_STAGE, &tA, kb * BKB, m0, mod, &full[s]);
          tma_load_3d(sB + s * B_STAGE, &tB, kb * BKB, n0, mod, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      // kind::i8: D s32 (2 << 4), A s8 (1 << 7), B s8 (1 << 10), K-major A/B,
      // N >> 3 at bit 17, M >> 4 at bit 24
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(BM >> 4) << 24);
      uint32_t it = 0, tl = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        int mod, m0, n0;
        if (!oz_tile(p, t, mod, m0, n0)) continue;
        const int b = tl & 1;
        const uint32_t aph = (tl >> 1) & 1;
        if (!mbar_wait(&acce[b], aph ^ 1, kErrAccWait)) break;  // buffer drained
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * BN);
        for (int kb = 0; kb < KB; ++kb, ++it) {
          const int s = it % S;
          const uint32_t ph = (it / S) & 1;
          if (!mbar_wait(&full[s], ph, kErrFullWait)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * A_STAGE), b0 = smem_u32(sB + s * B_STAGE);
#pragma unroll
          for (int k = 0; k < BKB / 32; ++k)
            tc_mma_i8(d, desc_sw128(a0 + 32 * k), desc_sw128(b0 + 32 * k), idesc,
                      (kb | k) != 0 ? 1u : 0u);
          tc_commit(&empty[s]);  // stage s free once these MMAs have read it
        }
        tc_commit(&accf[b]);  // accumulator b complete (also drains an aborted loop)
        ++tl;
      }
    }
  } else {
    // ---- epilogue: warps 2..5, TMEM lanes 32*(warp%4) .. +31
    const int q = warp & 3;
    uint32_t tl = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
      int mod, m0, n0;
      if (!oz_tile(p, t, mod, m0, n0)) continue;
      const int b = tl & 1;
      const uint32_t aph = (tl >> 1) & 1;
      const bool got = mbar_wait(&accf[b], aph, kErrAccWait);
      if (!__all_sync(0xffffffffu, got)) break;  // uniform and converged for tcgen05.ld
      tc_fence_after();
      const int row = m0 + q * 32 + lane;
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN);
      const int pm = p.p[mod];
      const double ip = p.invp[mod];
      uint8_t* plane = p.R + (size_t)mod * (size_t)p.Mpad * (size_t)p.Npad;
      for (int c = 0; c < BN / 16; ++c) {
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
            "%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tbase + (uint32_t)(c * 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (c == BN / 16 - 1) {
          // every column of buffer b is in registers: hand it back to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[b]);
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int acc = (int)v[e];
          const int qq = (int)floor((double)acc * ip);
          int r = acc - qq * pm;
          if (r < 0) r += pm;
          else if (r >= pm) r -= pm;
          const size_t col = (size_t)(n0 + c * 16 + e);
          // streaming store: the residue planes are read once, by the CRT
          // kernel; they should not evict the operand panels from L2
          __stcs(plane + col * (size_t)p.Mpad + (size_t)row, (unsigned char)r);
        }
      }
      ++tl;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// 3b. The same product on CTA pairs (a cluster of 2): tcgen05.mma.cta_group::2
//     computes a 256 x 256 tile per pair, each CTA holding 128 rows of A and
//     128 rows of B (its half of N) in shared memory and 128 rows of the
//     accumulator in its TMEM.  Per CTA and stage: 16 KB of A + 16 KB of B
//     for the work that takes 16 + 32 KB in the single-CTA kernel, so a third
//     less operand traffic from L2 per MMA.  Both CTAs load their halves with
//     TMA; the loads signal the even CTA's stage barrier, the even CTA
//     issues the MMAs and commits to the barriers of both CTAs, and
//     the odd CTA's epilogue warps release the accumulator on the even CTA's
//     barrier.
constexpr int BM2 = 256, BN2 = 256;                 // pair tile
constexpr int S2 = 6;                               // stages
constexpr uint32_t H_STAGE = 128 * BKB;             // one 128-row operand half per stage
constexpr uint32_t kPeerMask = 0xFEFFFFFFu;         // shared::cluster address of the even CTA

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t mapa_rank(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx_cluster(uint32_t cluster_addr, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cluster.shared::cluster.b64 _, [%0], %1;" ::"r"(
                   cluster_addr),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_3d_pair(void* dst, const CUtensorMap* m, int x, int y,
                                                 int z, uint32_t bar_even) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(z), "r"(bar_even)
      : "memory");
}
__device__ __forceinline__ void tc_mma_i8_pair(uint32_t tmem, uint64_t ad, uint64_t bd,
                                               uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
// commit the MMAs issued so far to the barrier at this offset in both CTAs
// (one commit per CTA, addressed through the cluster window)
__device__ __forceinline__ void tc_commit_pair(uint64_t* bar) {
#pragma unroll
  for (uint32_t r = 0; r < 2; ++r)
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::
                     "r"(mapa_rank(smem_u32(bar), r))
                 : "memory");
}

__device__ __forceinline__ bool oz_tile2(const GemmP& p, int t, int& mod, int& m0, int& n0) {
  const int tiles_mn = p.tiles_m * p.tiles_n;
  mod = t / tiles_mn;
  const int r = t - mod * tiles_mn;
  const int GROUP = p.group;
  const int span = GROUP * p.tiles_n;
  const int first_m = (r / span) * GROUP;
  const int gsz = min(p.tiles_m - first_m, GROUP);
  const int tm = first_m + (r % span) % gsz;
  const int tn = (r % span) / gsz;
  m0 = tm * BM2;
  n0 = tn * BN2;
  if (p.uplo == XKB_LOWER && (long)(m0 + BM2 - 1) + p.diag < (long)n0) return false;
  if (p.uplo == XKB_UPPER && (long)m0 + p.diag > (long)(n0 + BN2 - 1)) return false;
  return true;
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_oz_gemm2(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
               const GemmP p) {
  extern __shared__ uint8_t sm_raw[];
  uint8_t* sm =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = sm;
  uint8_t* sB = sm + S2 * H_STAGE;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + S2 * H_STAGE);
  uint64_t* empty = full + S2;
  uint64_t* accf = empty + S2;  // [2] accumulator ready (both CTAs)
  uint64_t* acce = accf + 2;    // [2] accumulator drained (even CTA: both epilogues)
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);

  const uint32_t rank = cluster_rank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int total = p.tiles_m * p.tiles_n * min(p.sel->n, p.nmod);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S2; ++s) {
      mbar_init(&full[s], 2);  // one arrive.expect_tx per CTA of the pair
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 2 * kEpiWarps);
    }
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    tc_fence_before();
  }
  __syncthreads();
  cluster_sync();  // barriers of both CTAs initialised before any cross-CTA signal
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tslot);
  const int KB = p.kblocks;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer (both CTAs): this CTA's halves of A and B
      tma_prefetch(&tA);
      tma_prefetch(&tB);
      uint32_t it = 0;
      bool ok = true;
      for (int t = pair; t < total && ok; t += npairs) {
        int mod, m0, n0;
        if (!oz_tile2(p, t, mod, m0, n0)) continue;
        for (int kb = 0; kb < KB; ++kb, ++it) {
          const int s = it % S2;
          const uint32_t ph = (it / S2) & 1;
          if (!mbar_wait(&empty[s], ph ^ 1, kErrEmptyWait)) {
            ok = false;
            break;
          }
          // the even CTA's stage barrier: arrive through its cluster address,
          // the pair-form TMA names it with the peer bit cleared
          mbar_expect_tx_cluster(mapa_rank(smem_u32(&full[s]), 0), 2 * H_STAGE);
          const uint32_t fe = smem_u32(&full[s]) & kPeerMask;
          tma_load_3d_pair(sA + s * H_STAGE, &tA, kb * BKB, m0 + 128 * (int)rank, mod, fe);
          tma_load_3d_pair(sB + s * H_STAGE, &tB, kb * BKB, n0 + 128 * (int)rank, mod, fe);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {  // ---- MMA issuer (even CTA)
      // kind::i8: D s32, A s8, B s8, K-major; N = 256, M = 256 (the pair)
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN2 >> 3) << 17) |
                             ((uint32_t)(BM2 >> 4) << 24);
      uint32_t it = 0, tl = 0;
      bool ok = true;
      for (int t = pair; t < total && ok; t += npairs) {
        int mod, m0, n0;
        if (!oz_tile2(p, t, mod, m0, n0)) continue;
        const int b = tl & 1;
        const uint32_t aph = (tl >> 1) & 1;
        if (!mbar_wait(&acce[b], aph ^ 1, kErrAccWait)) break;  // drained in both CTAs
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * BN2);
        for (int kb = 0; kb < KB; ++kb, ++it) {
          const int s = it % S2;
          const uint32_t ph = (it / S2) & 1;
          if (!mbar_wait(&full[s], ph, kErrFullWait)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * H_STAGE), b0 = smem_u32(sB + s * H_STAGE);
#pragma unroll
          for (int k = 0; k < BKB / 32; ++k)
            tc_mma_i8_pair(d, desc_sw128(a0 + 32 * k), desc_sw128(b0 + 32 * k), idesc,
                           (kb | k) != 0 ? 1u : 0u);
          tc_commit_pair(&empty[s]);  // stage s free in both CTAs once read
        }
        tc_commit_pair(&accf[b]);  // accumulator b complete in both CTAs
        ++tl;
      }
    }
  } else {
    // ---- epilogue (both CTAs): warps 2..5, TMEM lanes 32*(warp%4) .. +31
    const int q = warp & 3;
    const uint32_t ae0 = mapa_rank(smem_u32(&acce[0]), 0), ae1 = mapa_rank(smem_u32(&acce[1]), 0);
    uint32_t tl = 0;
    for (int t = pair; t < total; t += npairs) {
      int mod, m0, n0;
      if (!oz_tile2(p, t, mod, m0, n0)) continue;
      const int b = tl & 1;
      const uint32_t aph = (tl >> 1) & 1;
      const bool got = mbar_wait(&accf[b], aph, kErrAccWait);
      if (!__all_sync(0xffffffffu, got)) break;  // uniform and converged for tcgen05.ld
      tc_fence_after();
      const int row = m0 + 128 * (int)rank + q * 32 + lane;
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN2);
      const int pm = p.p[mod];
      const double ip = p.invp[mod];
      uint8_t* plane = p.R + (size_t)mod * (size_t)p.Mpad * (size_t)p.Npad;
      for (int c = 0; c < BN2 / 16; ++c) {
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
            "%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tbase + (uint32_t)(c * 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (c == BN2 / 16 - 1) {
          // every column of buffer b is in registers: release it to the even CTA
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_cluster(b ? ae1 : ae0);
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int acc = (int)v[e];
          const int qq = (int)floor((double)acc * ip);
          int r = acc - qq * pm;
          if (r < 0) r += pm;
          else if (r >= pm) r -= pm;
          const size_t col = (size_t)(n0 + c * 16 + e);
          __stcs(plane + col * (size_t)p.Mpad + (size_t)row, (unsigned char)r);
        }
      }
      ++tl;
    }
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs done with the pair's TMEM and barriers
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// 4. CRT reconstruction + scaling + alpha/beta, 4 consecutive rows per thread.
struct CrtP {
  int M, N;
  const uint8_t* R;
  long Mpad, Npad;
  const int* mu;     // row codes of op(A) (k_oz_stat)
  const int* nu;     // column codes of op(B)
  const OzSel* sel;  // the call's moduli count and exponent budget
  double* C;         // interleaved complex when cplx: writes part `part` (0 re, 1 im)
  long ldc;
  int cplx, part;
  double ar, ai, br, bi;  // real: ar, br used
  const double* other;    // complex: the other part's integer result, see host
  int uplo, herm_diag;
  long diag;
};

// Recombination on the FP64 pipe.  S = sum_l r_l w_l < 4080 P; the shifts
// keep |C'| <= P/8, so the wanted value is S - qP with q = round(S / P).
// With w = w1 + w2 (w1: multiples of 2^csplit, <= 41 significant bits):
//  - S1 = sum r_l w1_l is exact (8-bit x 41-bit products, multiples of
//    2^csplit, sum below 2^(53+csplit));
//  - q = rint(S1 / P) is exact: S2 / P < 2^-28 and S / P lies within 1/8 of
//    an integer (q < 2^12);
//  - S1 - q P1 is exact (a 53-bit product, the difference a multiple of
//    2^csplit below 2^(42+csplit));
//  - S2 - q P2 carries absolute errors of order 2^(csplit-37) plus the
//    rounding of w2 (2^43 at 16 moduli), far below the 2^(2H-61) sqrt(K)
//    already left by rounding the scaled operands to integers.
// 2 FP64 FMAs per modulus and element (a 128-bit integer sum would take 4
// 64-bit integer multiply-adds): the kernel runs on the FP64 pipe, which
// nothing else here uses.
template <int NM>
__device__ __forceinline__ double crt_value(const uint32_t (&r)[NM], const Consts& c) {
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int m = 0; m < NM; ++m) {
    const double rv = (double)r[m];
    s1 = fma(rv, c.w1[m], s1);
    s2 = fma(rv, c.w2[m], s2);
  }
  const double q = rint(s1 * c.invPd);
  return fma(-q, c.P1d, s1) + fma(-q, c.P2d, s2);
}

// x * 2^e for the shift range used here (|e| <= 2000), exact unless the
// result under/overflows
__device__ __forceinline__ double scale2(double x, int e) {
  // x normal and x 2^e normal: add e to the exponent field
  const int hi = __double2hiint(x);
  const int ex = (hi >> 20) & 0x7ff;
  if (ex != 0 && (unsigned)(ex + e - 1) < 2046u)
    return __hiloint2double(hi + (int)((unsigned)e << 20), __double2loint(x));
  const int e1 = e / 2, e2 = e - e1;
  return x * pow2(e1) * pow2(e2);
}

// The four rows of a thread are reconstructed unconditionally (rows past M
// reuse the last row's shift and are not stored), so their independent
// integer chains interleave; the stores are predicated afterwards.
template <int NM>
__device__ __forceinline__ void crt_quad(const CrtP& p, const Consts& c, int H, long i0, int j,
                                         double (&y)[4]) {
  const size_t plane = (size_t)p.Mpad * (size_t)p.Npad;
  uint32_t words[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m)
    words[m] = *reinterpret_cast<const uint32_t*>(p.R + (size_t)m * plane + (size_t)j * p.Mpad + i0);
  const int nuj = shift_of(p.nu[j], H);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    uint32_t r[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) r[m] = __byte_perm(words[m], 0u, 0x4440 + v);
    const int mui = shift_of(p.mu[min(i0 + v, (long)p.M - 1)], H);
    if (mui == kShiftNonFinite || nuj == kShiftNonFinite) y[v] = __longlong_as_double(0x7ff8000000000000ll);
    else y[v] = scale2(crt_value<NM>(r, c), -(mui + nuj));
  }
}

template <int NM>
__device__ __forceinline__ void crt_body(const CrtP& p, const Consts& c, int H) {
  const long iq = (long)blockIdx.x * blockDim.x + threadIdx.x;  // row quad
  const long i0 = iq * 4;
  if (i0 >= p.M) return;
  for (int j = blockIdx.y; j < p.N; j += gridDim.y) {
    double y[4];
    crt_quad<NM>(p, c, H, i0, j, y);
    const size_t idx0 = (size_t)i0 + (size_t)j * p.ldc;
    if (!p.cplx) {
      const bool full = i0 + 3 < p.M && p.uplo == XKB_FULL &&
                        (reinterpret_cast<uintptr_t>(p.C + idx0) & 15) == 0;
      if (full) {  // two 16-byte loads / stores for the quad
        double2* cp2 = reinterpret_cast<double2*>(p.C + idx0);
        double2 o0 = make_double2(p.ar * y[0], p.ar * y[1]);
        double2 o1 = make_double2(p.ar * y[2], p.ar * y[3]);
        if (p.br != 0.0) {
          const double2 c0 = cp2[0], c1 = cp2[1];
          o0.x = fma(p.br, c0.x, o0.x);
          o0.y = fma(p.br, c0.y, o0.y);
          o1.x = fma(p.br, c1.x, o1.x);
          o1.y = fma(p.br, c1.y, o1.y);
        }
        cp2[0] = o0;
        cp2[1] = o1;
        continue;
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const long i = i0 + v;
      if (i >= p.M) break;
      if (p.uplo == XKB_LOWER && i + p.diag < j) continue;
      if (p.uplo == XKB_UPPER && i + p.diag > j) continue;
      const size_t idx = (size_t)i + (size_t)j * p.ldc;
      if (!p.cplx) {
        double out = p.ar * y[v];
        if (p.br != 0.0) out = fma(p.br, p.C[idx], out);
        p.C[idx] = out;
      } else {
        // complex: the first pass wrote Re(AB) into p.other[i + j*M]; this
        // pass reconstructs Im(AB) and writes the (Re, Im) pairs of C
        const double xr = p.other[(size_t)i + (size_t)j * p.M], xi = y[v];
        double vr = p.ar * xr - p.ai * xi;
        double vi = p.ar * xi + p.ai * xr;
        if (p.br != 0.0 || p.bi != 0.0) {
          const double cr = p.C[2 * idx], ci = p.C[2 * idx + 1];
          vr += p.br * cr - p.bi * ci;
          vi += p.br * ci + p.bi * cr;
        }
        if (p.herm_diag && i + p.diag == j) vi = 0.0;
        p.C[2 * idx] = vr;
        p.C[2 * idx + 1] = vi;
      }
    }
  }
}

// Complex first pass: Re(op(A)op(B)) (unscaled by alpha) into a scratch M x N.
template <int NM>
__device__ __forceinline__ void crt_store_body(const CrtP& p, const Consts& c, int H,
                                               double* out) {
  const long iq = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long i0 = iq * 4;
  if (i0 >= p.M) return;
  for (int j = blockIdx.y; j < p.N; j += gridDim.y) {
    double y[4];
    crt_quad<NM>(p, c, H, i0, j, y);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const long i = i0 + v;
      if (i >= p.M) break;
      if (p.uplo == XKB_LOWER && i + p.diag < j) continue;
      if (p.uplo == XKB_UPPER && i + p.diag > j) continue;
      out[(size_t)i + (size_t)j * p.M] = y[v];
    }
  }
}

// CRT kernels.  A fixed count: one instance per count.  A count chosen on the
// device between 15 and 16 (the data rule's range, k_oz_pick): one kernel
// holding both reconstructions, each block taking the one sel->n names.  A
// call the pick sent to the plain kernel (sel->n == 0) writes nothing here.
template <int NM>
__global__ void __launch_bounds__(256, 4) k_oz_crt(const CrtP p, const Consts c) {
  const OzSel s = *p.sel;
  if (s.n != NM) return;
  crt_body<NM>(p, c, s.H);
}
template <int NM>
__global__ void __launch_bounds__(256, 4) k_oz_crt_store(const CrtP p, const Consts c, double* out) {
  const OzSel s = *p.sel;
  if (s.n != NM) return;
  crt_store_body<NM>(p, c, s.H, out);
}
__global__ void __launch_bounds__(256, 4) k_oz_crt_15_16(const CrtP p, const Consts c15,
                                                         const Consts c16) {
  const OzSel s = *p.sel;
  if (s.n == 15) crt_body<15>(p, c15, s.H);
  else if (s.n == 16) crt_body<16>(p, c16, s.H);
}
__global__ void __launch_bounds__(256, 4) k_oz_crt_store_15_16(const CrtP p, const Consts c15,
                                                               const Consts c16, double* out) {
  const OzSel s = *p.sel;
  if (s.n == 15) crt_store_body<15>(p, c15, s.H, out);
  else if (s.n == 16) crt_store_body<16>(p, c16, s.H, out);
}

template <int NM>
static void crt_launch(dim3 g, cudaStream_t st, const CrtP& cp, const Consts& c, double* store) {
  if (store) k_oz_crt_store<NM><<<g, 256, 0, st>>>(cp, c, store);
  else k_oz_crt<NM><<<g, 256, 0, st>>>(cp, c);
}
// lo == hi: that count; (lo, hi) == (15, 16): the count the device chose.
static int launch_crt(dim3 g, cudaStream_t st, const CrtP& cp, const Consts* lo,
                      const Consts* hi, double* store) {
  if (!lo || !hi) return XKB_EINVAL;
  const long long tv = evlog_kern_begin(st, store ? "k_oz_crt_store" : "k_oz_crt");
  if (lo->nmod != hi->nmod) {
    if (lo->nmod != 15 || hi->nmod != 16) return XKB_EINVAL;
    if (store) k_oz_crt_store_15_16<<<g, 256, 0, st>>>(cp, *lo, *hi, store);
    else k_oz_crt_15_16<<<g, 256, 0, st>>>(cp, *lo, *hi);
  } else {
    switch (hi->nmod) {
#define XKB_CRT_CASE(NM) \
  case NM:               \
    crt_launch<NM>(g, st, cp, *hi, store); break;
      XKB_CRT_CASE(2) XKB_CRT_CASE(3) XKB_CRT_CASE(4) XKB_CRT_CASE(5) XKB_CRT_CASE(6)
      XKB_CRT_CASE(7) XKB_CRT_CASE(8) XKB_CRT_CASE(9) XKB_CRT_CASE(10) XKB_CRT_CASE(11)
      XKB_CRT_CASE(12) XKB_CRT_CASE(13) XKB_CRT_CASE(14) XKB_CRT_CASE(15) XKB_CRT_CASE(16)
#undef XKB_CRT_CASE
      default: return XKB_EINVAL;
    }
  }
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

// ---------------------------------------------------------------------------
// host orchestration
static size_t rup(size_t v, size_t a) { return (v + a - 1) / a * a; }

static const Consts* consts_for(int n) {
  static Consts cache[kMaxMod + 1];
  static bool have[kMaxMod + 1] = {false};
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  if (n < 2 || n > kMaxMod) return nullptr;
  if (!have[n]) {
    if (!make_consts(n, &cache[n])) return nullptr;
    have[n] = true;
  }
  return &cache[n];
}

// Operand descriptor: an L x K "row" view (rows of op(A), or columns of
// op(B)) of a real matrix, or of one part of a complex one.
struct View {
  const double* X;  // base (double units)
  long ld;          // leading dimension in elements (complex: complex elements)
  bool kc;          // k contiguous
  long estride;     // 1 real, 2 complex
  long eoff;        // 0 real part, 1 imaginary part
  double sign;
};

// Device words of one call: the moduli selection and the two concentration
// maxima (rows of op(A), columns of op(B)); zeroed before the norms.
struct CallWords {
  OzSel sel;
  unsigned rmax[2];
  unsigned pad[2];
};

// The counts a call may use: a fixed count (lo = hi), or the data rule's
// range [lo, 16] with lo = max(15, the tuning table's count for K's band).
struct ModPlan {
  int lo = 0, hi = 0;
  bool fixed = true;
  const Consts* clo = nullptr;
  const Consts* chi = nullptr;
};

static bool plan_moduli(int nmod, long K, ModPlan* pl) {
  if (nmod > 0) {
    pl->lo = pl->hi = nmod;
    pl->fixed = true;
  } else {
    const int tuned = tune_band("ozaki_moduli_k<=", K);
    pl->lo = std::min(kMaxMod, std::max(15, (tuned >= 2 && tuned <= kMaxMod) ? tuned : 0));
    pl->hi = kMaxMod;
    pl->fixed = false;
  }
  pl->clo = consts_for(pl->lo);
  pl->chi = consts_for(pl->hi);
  return pl->clo && pl->chi;
}

// Row statistics of an L x K operand view: codes (k_oz_stat) and the
// concentration maximum into *rmax.
static int launch_norm(const View& v, int L, int K, int cplx, double4* part, int* code,
                       unsigned* rmax, cudaStream_t st) {
  const int nch = (K + kNormChunk - 1) / kNormChunk;
  const long long tv = evlog_kern_begin(st, "k_oz_norm+k_oz_stat");
  if (v.kc) {
    dim3 g((unsigned)((L + 7) / 8), (unsigned)nch);
    k_oz_norm<true><<<g, 256, 0, st>>>(L, K, v.X, v.ld, cplx, part);
  } else {
    dim3 g((unsigned)((L + 31) / 32), (unsigned)nch);
    k_oz_norm<false><<<g, 256, 0, st>>>(L, K, v.X, v.ld, cplx, part);
  }
  k_oz_stat<<<(unsigned)((L + 255) / 256), 256, 0, st>>>(L, K, nch, part, code, rmax);
  evlog_kern_end(tv, st);
  count_launch(2);
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static int launch_pick(CallWords* w, const ModPlan& pl, bool allow_fallback, cudaStream_t st) {
  PickP q;
  std::memset(&q, 0, sizeof(q));
  q.fixed = pl.fixed ? pl.hi : 0;
  q.lo = pl.lo;
  q.hi = pl.hi;
  q.allow_fallback = allow_fallback ? 1 : 0;
  for (int n = 2; n <= kMaxMod; ++n) {
    const Consts* c = consts_for(n);
    if (!c) return XKB_EINVAL;
    q.H[n] = c->H;
  }
  const long long tv = evlog_kern_begin(st, "k_oz_pick");
  k_oz_pick<<<1, 32, 0, st>>>(w->rmax, &w->sel, q);
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

// Residue planes 0 .. sel->n - 1 of an operand view (c: the constants of the
// plan's largest count; the per-modulus constants are those of every count).
static int launch_res(const View& v, int L, int K, const int* code, const OzSel* sel,
                      const Consts* c, int8_t* planes, long Lpad, long Kpad, long kofs,
                      cudaStream_t st, long grid_rows = 0) {
  // grid covers Lpad (or grid_rows, for a block of rows of larger planes:
  // planes stay Lpad rows apart) x (K rounded to 64); kofs places the block
  // at column kofs; rows from L to the grid's end are written as zeros
  dim3 g((unsigned)((grid_rows ? grid_rows : Lpad) / 64), (unsigned)(rup((size_t)K, 64) / 64));
#define XKB_RES_CASE(NM)                                                                     \
  case NM:                                                                                   \
    if (v.kc)                                                                                \
      k_oz_residues<true, NM><<<g, 256, 0, st>>>(L, K, v.X, v.ld, v.estride, v.eoff, v.sign, \
                                                 code, sel, *c, planes, Lpad, Kpad, kofs);   \
    else                                                                                     \
      k_oz_residues<false, NM><<<g, 256, 0, st>>>(L, K, v.X, v.ld, v.estride, v.eoff,       \
                                                  v.sign, code, sel, *c, planes, Lpad, Kpad, \
                                                  kofs);                                     \
    break;
  if (c->nmod < 2 || c->nmod > kMaxMod) return XKB_EINVAL;
  const long long tv = evlog_kern_begin(st, "k_oz_residues");
  switch (c->nmod) {
    XKB_RES_CASE(2) XKB_RES_CASE(3) XKB_RES_CASE(4) XKB_RES_CASE(5) XKB_RES_CASE(6)
    XKB_RES_CASE(7) XKB_RES_CASE(8) XKB_RES_CASE(9) XKB_RES_CASE(10) XKB_RES_CASE(11)
    XKB_RES_CASE(12) XKB_RES_CASE(13) XKB_RES_CASE(14) XKB_RES_CASE(15) XKB_RES_CASE(16)
    default: break;
  }
#undef XKB_RES_CASE
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

static bool encode_planes(CUtensorMap* m, const int8_t* base, long Kpad, long Lpad, int nmod,
                          uint32_t box_rows, long plane_rows = 0) {
  return encode_tmap_3d_u8(m, base, (uint64_t)Kpad, (uint64_t)Lpad, (uint64_t)nmod, 128,
                           box_rows, (uint64_t)plane_rows);
}

// a_rows / b_rows: rows per plane of the A / B residue buffers (>= Mpad /
// Npad; equal when one buffer serves both operands).  a_stride / b_stride
// (0: the same): rows between consecutive planes, when Ap / Bp point at a
// block of rows of larger planes.
static int launch_gemm(const int8_t* Ap, long a_rows, const int8_t* Bp, long b_rows, long Mpad,
                       long Npad, long Kpad, const Consts* c, const OzSel* sel, uint8_t* R,
                       int uplo, long diag, cudaStream_t st, long a_stride = 0,
                       long b_stride = 0) {
  CUtensorMap tA, tB;
  if (a_rows < Mpad || b_rows < Npad) return XKB_EINVAL;
  if (!encode_planes(&tA, Ap, Kpad, a_rows, c->nmod, BM, a_stride)) return XKB_EINVAL;
  if (!encode_planes(&tB, Bp, Kpad, b_rows, c->nmod, BN, b_stride)) return XKB_EINVAL;
  GemmP p;
  std::memset(&p, 0, sizeof(p));
  p.tiles_m = (int)(Mpad / BM);
  p.tiles_n = (int)(Npad / BN);
  p.kblocks = (int)(Kpad / BKB);
  p.nmod = c->nmod;
  p.sel = sel;
  // raster group (tuning table oz_group_m, default 8 M tiles)
  p.group = std::max(1, std::min(p.tiles_m, (int)tune("oz_group_m", 8.0)));
  p.R = R;
  p.Mpad = Mpad;
  p.Npad = Npad;
  p.uplo = uplo;
  p.diag = diag;
  for (int m = 0; m < c->nmod; ++m) {
    p.p[m] = c->p[m];
    p.invp[m] = c->invp_d[m];
  }
  const long total2 = (Mpad % BM2 == 0 && Npad % BN2 == 0)
                         ? (Mpad / BM2) * (Npad / BN2) * (long)c->nmod : 0;
  if (total2 > 0 && tune("oz_2cta", 0.0) != 0.0 && sm_count() >= 2) {
    // CTA pairs: 256 x 256 tiles, each CTA loading 128-row halves of A and B
    CUtensorMap tB2;
    if (!encode_planes(&tB2, Bp, Kpad, b_rows, c->nmod, 128, b_stride)) return XKB_EINVAL;
    p.tiles_m = (int)(Mpad / BM2);
    p.tiles_n = (int)(Npad / BN2);
    p.group = std::max(1, std::min(p.tiles_m, (int)tune("oz_group_m", 8.0)));
    const size_t smem2 = 1024 + S2 * (size_t)(2 * H_STAGE) + (2 * S2 + 4) * 8 + 16;
    static bool attr2 = false;
    if (!attr2) {
      if (cudaFuncSetAttribute(k_oz_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem2) != cudaSuccess)
        return XKB_ECUDA;
      attr2 = true;
    }
    const long pairs = std::min<long>(total2, sm_count() / 2);
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(2 * pairs));
    cfg.blockDim = dim3(kGemmThreads);
    cfg.dynamicSmemBytes = smem2;
    cfg.stream = st;
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeClusterDimension;
    la[0].val.clusterDim.x = 2;
    la[0].val.clusterDim.y = 1;
    la[0].val.clusterDim.z = 1;
    cfg.attrs = la;
    cfg.numAttrs = 1;
    const long long tv = evlog_kern_begin(st, "k_oz_gemm2");
    const cudaError_t le = cudaLaunchKernelEx(&cfg, k_oz_gemm2, tA, tB2, p);
    evlog_kern_end(tv, st);
    if (le != cudaSuccess) return XKB_ECUDA;
    count_launch();
    return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
  }
  const size_t smem = 1024 + S * (size_t)(A_STAGE + B_STAGE) + (2 * S + 4) * 8 + 16;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return XKB_ECUDA;
    attr = true;
  }
  const long total = (long)p.tiles_m * p.tiles_n * c->nmod;
  const unsigned grid = (unsigned)std::min<long>(total, sm_count());  // persistent
  const long long tv = evlog_kern_begin(st, "k_oz_gemm");
  k_oz_gemm<<<grid, kGemmThreads, smem, st>>>(tA, tB, p);
  evlog_kern_end(tv, st);
  count_launch();
  return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
}

int default_moduli(long K) {
  if (K <= 0 || K > 131072) return 0;  // exact INT32 accumulation limit
  // a count the autotuner measured for this K band (tuning table keys
  // "ozaki_moduli_k<=<K>"), when one covers K
  const int tuned = tune_band("ozaki_moduli_k<=", K);
  if (tuned >= 2 && tuned <= kMaxMod) return tuned;
  // keep >= 53 bits for the largest entry of a row whose entries are all of
  // the same magnitude: H - log2(K)/2 >= 53
  for (int n = 8; n <= kMaxMod; ++n) {
    const int H = (int)std::floor((log2P(n) - 1.0) / 2.0) - 1;
    if ((double)H - 0.5 * std::log2((double)K) >= 53.0) return n;
  }
  return kMaxMod;
}

}  // namespace oz
}  // namespace xkb

using namespace xkb;
using namespace xkb::oz;

extern "C" int xkb_ozaki_default_moduli(long K) { return default_moduli(K); }

extern "C" int xkb_ozaki_counts(unsigned long long* out, int* last, int reset) {
  if (!out) return XKB_EINVAL;
  // the counters are written by kernels on the library's non-blocking streams
  if (cudaDeviceSynchronize() != cudaSuccess) return XKB_ECUDA;
  if (cudaMemcpyFromSymbol(&out[0], g_oz_calls, sizeof(out[0])) != cudaSuccess ||
      cudaMemcpyFromSymbol(&out[1], g_oz_mod_sum, sizeof(out[1])) != cudaSuccess ||
      cudaMemcpyFromSymbol(&out[2], g_oz_fallbacks, sizeof(out[2])) != cudaSuccess)
    return XKB_ECUDA;
  if (last && cudaMemcpyFromSymbol(last, g_oz_last, sizeof(int)) != cudaSuccess) return XKB_ECUDA;
  if (reset) {
    const unsigned long long z = 0;
    const int none = -1;
    if (cudaMemcpyToSymbol(g_oz_calls, &z, sizeof z) != cudaSuccess ||
        cudaMemcpyToSymbol(g_oz_mod_sum, &z, sizeof z) != cudaSuccess ||
        cudaMemcpyToSymbol(g_oz_fallbacks, &z, sizeof z) != cudaSuccess ||
        cudaMemcpyToSymbol(g_oz_last, &none, sizeof none) != cudaSuccess)
      return XKB_ECUDA;
  }
  return XKB_OK;
}

// Real or complex Ozaki GEMM.  nmod > 0: that many moduli.  nmod == 0: the
// count is chosen on the device from the operands (k_oz_pick: 15 or 16, at
// least the tuning table's count for K's band); operands whose spread 16
// moduli cannot carry to FP64 accuracy are computed by the plain FP64
// kernel instead, launched here and predicated on the device's choice.
// Scratch (stream-ordered, from the pool): residue planes of op(A) and
// op(B) for the largest count the call may use (nmod x Mpad x Kpad,
// nmod x Npad x Kpad int8), residue planes of C (nmod x Mpad x Npad uint8),
// row codes, norm partials and the call's device words.
extern "C" int xkb_cuda_ozaki_gemm(const xkb_gemm_args* a, int nmod, void* stream) {
  if (!a || (a->dtype != XKB_D && a->dtype != XKB_Z)) return XKB_EINVAL;
  if (a->M < 0 || a->N < 0 || a->K < 0) return XKB_EINVAL;
  if (a->M == 0 || a->N == 0) return XKB_OK;
  const bool cplx = a->dtype == XKB_Z;
  const long Keff = cplx ? 2L * a->K : (long)a->K;
  if (a->K == 0 || (a->alpha[0] == 0.0 && a->alpha[1] == 0.0))
    return xkb_cuda_gemm(a, stream);
  if (Keff > 131072) return XKB_ERANGE;
  ModPlan pl;
  if (!plan_moduli(nmod, Keff, &pl)) return XKB_ERANGE;
  const int nmax = pl.hi;
  cudaStream_t st = resolve_stream(stream);
  const int M = a->M, N = a->N, K = a->K;
  // complex operands are laid out [Re | pad | Im | pad] along k, each block
  // starting on a 64-column boundary (aligned 4-byte stores in the residue
  // kernel); the zero pads contribute nothing to the products
  const long kofs2 = (long)rup(K, 64);
  const long Kpad = cplx ? (long)rup(2 * kofs2, BKB) : (long)rup(K, BKB);
  const long Mpad = (long)rup(M, BM2), Npad = (long)rup(N, BN);  // BM2: CTA-pair tiles
  const bool akc = a->opA != XKB_OP_N, bkc = a->opB == XKB_OP_N;
  // C = A A^T (or A^T A): op(B)^T's rows are op(A)'s rows, one residue buffer
  // serves both operands; it then holds max(Mpad, Npad) rows per plane
  const bool same = (a->A == a->B) && (a->lda == a->ldb) && (akc == bkc) && !cplx && M == N;
  const long Arows = same ? std::max(Mpad, Npad) : Mpad;
  const size_t szA = (size_t)nmax * Arows * Kpad, szB = (size_t)nmax * Npad * Kpad;
  const size_t szR = (size_t)nmax * Mpad * Npad;
  const int nch = (int)((Keff + kNormChunk - 1) / kNormChunk);
  const size_t szPart = 256 + sizeof(double4) * (size_t)nch * (size_t)std::max(M, N) * 2;
  const size_t szRe = cplx ? sizeof(double) * (size_t)M * N : 0;
  int8_t *Ap = nullptr, *Bp = nullptr;
  uint8_t* R = nullptr;
  int *mu = nullptr, *nu = nullptr;
  unsigned char* pw = nullptr;  // CallWords, then the norm partials from byte 256
  double* re = nullptr;
  auto alloc = [&](void** p, size_t n) {
    return cudaMallocAsync(p, std::max<size_t>(n, 256), st) == cudaSuccess;
  };
  bool ok = alloc((void**)&Ap, szA) && alloc((void**)&Bp, cplx ? 2 * szB : szB) &&
            alloc((void**)&R, szR) && alloc((void**)&mu, sizeof(int) * M) &&
            alloc((void**)&nu, sizeof(int) * N) && alloc((void**)&pw, szPart) &&
            (!cplx || alloc((void**)&re, szRe));
  int err = ok ? XKB_OK : XKB_ENOMEM;
  if (!ok) cudaGetLastError();
  CallWords* w = reinterpret_cast<CallWords*>(pw);
  double4* part = reinterpret_cast<double4*>(pw + 256);
  const OzSel* sel = w ? &w->sel : nullptr;
  // operand views ----------------------------------------------------------
  // rows of op(A): opA == N -> A is M x K, row i = A[i + k*lda] (i contiguous)
  //                else     -> A is K x M, row i = A[k + i*lda] (k contiguous)
  // columns of op(B): opB == N -> B is K x N, col j = B[k + j*ldb] (k contig.)
  //                   else     -> B is N x K, col j = B[j + k*ldb]
  const double* Ad = static_cast<const double*>(a->A);
  const double* Bd = static_cast<const double*>(a->B);
  const double sa = (a->opA == XKB_OP_C) ? -1.0 : 1.0;  // conj: negate Im
  const double sb = (a->opB == XKB_OP_C) ? -1.0 : 1.0;
  const int slot = trace_begin("ozaki_gemm", a->dtype, M, N, K, pl.fixed ? nmax : 0, st);
  if (err == XKB_OK) {
    // scaling: complex rows use the norm over (re, im) = the concatenated row
    View va{Ad, a->lda, akc, 1, 0, 1.0}, vb{Bd, a->ldb, bkc, 1, 0, 1.0};
    if (cudaMemsetAsync(w, 0, sizeof(CallWords), st) != cudaSuccess) err = XKB_ECUDA;
    if (!err) err = launch_norm(va, M, K, cplx, part, mu, &w->rmax[0], st);
    if (!err)
      err = launch_norm(vb, N, K, cplx, part + (size_t)nch * std::max(M, N), nu, &w->rmax[1], st);
    if (!err) err = launch_pick(w, pl, !pl.fixed, st);
  }
  if (err == XKB_OK) {
    if (!cplx) {
      View va{Ad, a->lda, akc, 1, 0, 1.0}, vb{Bd, a->ldb, bkc, 1, 0, 1.0};
      err = launch_res(va, M, K, mu, sel, pl.chi, Ap, Arows, Kpad, 0, st);
      if (!err && !same) err = launch_res(vb, N, K, nu, sel, pl.chi, Bp, Npad, Kpad, 0, st);
      if (!err && Kpad > (long)rup(K, 64)) {
        // zero the k padding beyond the last 64-column block
        const size_t kz = rup(K, 64);
        err = cudaMemset2DAsync(Ap + kz, Kpad, 0, Kpad - kz, (size_t)nmax * Arows, st) == cudaSuccess
                  ? XKB_OK : XKB_ECUDA;
        if (!err && !same)
          err = cudaMemset2DAsync(Bp + kz, Kpad, 0, Kpad - kz, (size_t)nmax * Npad, st) == cudaSuccess
                    ? XKB_OK : XKB_ECUDA;
      }
    } else {
      // A' = [Re op(A) | Im op(A)] (K' = 2K);  B1 = [Re op(B); -Im op(B)],
      // B2 = [Im op(B); Re op(B)]:  Re(AB) = A' B1,  Im(AB) = A' B2.
      View ar{Ad, a->lda, akc, 2, 0, 1.0}, ai{Ad, a->lda, akc, 2, 1, sa};
      View br{Bd, a->ldb, bkc, 2, 0, 1.0}, bi{Bd, a->ldb, bkc, 2, 1, sb};
      View bin{Bd, a->ldb, bkc, 2, 1, -sb};
      int8_t* B1 = Bp;
      int8_t* B2 = Bp + szB;
      err = launch_res(ar, M, K, mu, sel, pl.chi, Ap, Mpad, Kpad, 0, st);
      if (!err) err = launch_res(ai, M, K, mu, sel, pl.chi, Ap, Mpad, Kpad, kofs2, st);
      if (!err) err = launch_res(br, N, K, nu, sel, pl.chi, B1, Npad, Kpad, 0, st);
      if (!err) err = launch_res(bin, N, K, nu, sel, pl.chi, B1, Npad, Kpad, kofs2, st);
      if (!err) err = launch_res(bi, N, K, nu, sel, pl.chi, B2, Npad, Kpad, 0, st);
      if (!err) err = launch_res(br, N, K, nu, sel, pl.chi, B2, Npad, Kpad, kofs2, st);
      if (!err && Kpad > 2 * kofs2) {
        const size_t kz = 2 * (size_t)kofs2;
        if (cudaMemset2DAsync(Ap + kz, Kpad, 0, Kpad - kz, (size_t)nmax * Mpad, st) != cudaSuccess ||
            cudaMemset2DAsync(Bp + kz, Kpad, 0, Kpad - kz, (size_t)2 * nmax * Npad, st) != cudaSuccess)
          err = XKB_ECUDA;
      }
    }
  }
  CrtP cp;
  std::memset(&cp, 0, sizeof(cp));
  cp.M = M;
  cp.N = N;
  cp.R = R;
  cp.Mpad = Mpad;
  cp.Npad = Npad;
  cp.mu = mu;
  cp.nu = nu;
  cp.sel = sel;
  cp.C = static_cast<double*>(a->C);
  cp.ldc = a->ldc;
  cp.cplx = cplx;
  cp.ar = a->alpha[0];
  cp.ai = cplx ? a->alpha[1] : 0.0;
  cp.br = a->beta[0];
  cp.bi = cplx ? a->beta[1] : 0.0;
  cp.uplo = a->uplo;
  cp.herm_diag = a->herm_diag;
  cp.diag = a->diag;
  const dim3 cg((unsigned)(((M + 3) / 4 + 255) / 256), (unsigned)std::min(N, 65535));
  trace_mark(slot, 1, st);
  if (err == XKB_OK) {
    err = same ? launch_gemm(Ap, Arows, Ap, Arows, Mpad, Npad, Kpad, pl.chi, sel, R, a->uplo,
                             a->diag, st)
               : launch_gemm(Ap, Mpad, Bp, Npad, Mpad, Npad, Kpad, pl.chi, sel, R, a->uplo,
                             a->diag, st);
    if (!err) {
      if (!cplx) {
        trace_mark(slot, 2, st);
        err = launch_crt(cg, st, cp, pl.clo, pl.chi, nullptr);
      } else {
        err = launch_crt(cg, st, cp, pl.clo, pl.chi, re);
        if (!err)
          err = launch_gemm(Ap, Mpad, Bp + szB, Npad, Mpad, Npad, Kpad, pl.chi, sel, R, a->uplo,
                            a->diag, st);
        trace_mark(slot, 2, st);
        if (!err) {
          cp.other = re;
          err = launch_crt(cg, st, cp, pl.clo, pl.chi, nullptr);
        }
      }
    }
    // the data rule may have sent the call to the plain FP64 kernel
    if (!err && !pl.fixed) err = gemm_if(a, &w->sel.fallback, st);
    if (!err && cudaPeekAtLastError() != cudaSuccess) err = XKB_ECUDA;
  }
  trace_mark(slot, 3, st);
  if (Ap) cudaFreeAsync(Ap, st);
  if (Bp) cudaFreeAsync(Bp, st);
  if (R) cudaFreeAsync(R, st);
  if (mu) cudaFreeAsync(mu, st);
  if (nu) cudaFreeAsync(nu, st);
  if (pw) cudaFreeAsync(pw, st);
  if (re) cudaFreeAsync(re, st);
  return err;
}

// ===========================================================================
// Column-panel form of the real contraction, for callers that move op(B)
// and C across the host link panel by panel: op(A) is scaled and converted
// once; then for each column panel [n0, n1) of op(B) / C the stream waits on
// wait_ev[p] (the panel's operands are on the device), the panel's column
// shifts and residue planes are formed, multiplied on the INT8 tensor cores
// and recombined into C[:, n0:n1), and done_ev[p] is recorded (the panel's
// result is final).  Transfers of later panels and of finished results then
// overlap the arithmetic.  The caller orders op(A) before the call.
// Real, C full (no triangle mask); other calls use xkb_cuda_ozaki_gemm.
extern "C" int xkb_cuda_ozaki_gemm_panels(const xkb_gemm_args* a, int nmod, void* stream,
                                          int npanel, const long* bounds,
                                          void* const* wait_ev, void* const* done_ev) {
  if (!a || a->dtype != XKB_D || a->uplo != XKB_FULL || npanel < 1 || !bounds)
    return XKB_EINVAL;
  if (a->M < 0 || a->N < 0 || a->K < 0) return XKB_EINVAL;
  if (bounds[0] != 0 || bounds[npanel] != a->N) return XKB_EINVAL;
  for (int q = 0; q < npanel; ++q)
    if (bounds[q + 1] <= bounds[q]) return XKB_EINVAL;
  cudaStream_t st = resolve_stream(stream);
  auto wait = [&](int q) {
    if (wait_ev && wait_ev[q]) cudaStreamWaitEvent(st, static_cast<cudaEvent_t>(wait_ev[q]), 0);
  };
  auto done = [&](int q) {
    if (done_ev && done_ev[q]) cudaEventRecord(static_cast<cudaEvent_t>(done_ev[q]), st);
  };
  if (a->M == 0) {
    for (int q = 0; q < npanel; ++q) done(q);
    return XKB_OK;
  }
  if (a->K == 0 || a->alpha[0] == 0.0 || a->K > 131072) {  // no split product to pipeline
    for (int q = 0; q < npanel; ++q) wait(q);
    const int r = a->K > 131072 ? XKB_ERANGE : xkb_cuda_gemm(a, st);
    for (int q = 0; q < npanel; ++q) done(q);
    return r;
  }
  // op(A) is converted before op(B) arrives: the count is fixed for the call
  // (the tuning table's or the K rule's when nmod == 0)
  if (nmod == 0) nmod = default_moduli(a->K);
  ModPlan pl;
  if (!plan_moduli(nmod, a->K, &pl)) return XKB_ERANGE;
  const Consts* c = pl.chi;
  const int M = a->M, K = a->K;
  const long Kpad = (long)rup(K, BKB), Mpad = (long)rup(M, BM2);
  long wmax = 0;
  for (int q = 0; q < npanel; ++q) wmax = std::max(wmax, bounds[q + 1] - bounds[q]);
  const long Wpad = (long)rup((size_t)wmax, BN);
  const bool akc = a->opA != XKB_OP_N, bkc = a->opB == XKB_OP_N;
  const int nch = (int)((K + kNormChunk - 1) / kNormChunk);
  int8_t *Ap = nullptr, *Bp = nullptr;
  uint8_t* R = nullptr;
  int *mu = nullptr, *nu = nullptr;
  unsigned char* pw = nullptr;  // CallWords, then the norm partials from byte 256
  auto alloc = [&](void** p, size_t n) {
    return cudaMallocAsync(p, std::max<size_t>(n, 256), st) == cudaSuccess;
  };
  bool ok = alloc((void**)&Ap, (size_t)nmod * Mpad * Kpad) &&
            alloc((void**)&Bp, (size_t)nmod * Wpad * Kpad) &&
            alloc((void**)&R, (size_t)nmod * Mpad * Wpad) && alloc((void**)&mu, sizeof(int) * M) &&
            alloc((void**)&nu, sizeof(int) * a->N) &&
            alloc((void**)&pw, 256 + sizeof(double4) * (size_t)nch * (size_t)std::max<long>(M, wmax));
  int err = ok ? XKB_OK : XKB_ENOMEM;
  if (!ok) cudaGetLastError();
  CallWords* w = reinterpret_cast<CallWords*>(pw);
  double4* part = reinterpret_cast<double4*>(pw + 256);
  const OzSel* sel = w ? &w->sel : nullptr;
  const double* Ad = static_cast<const double*>(a->A);
  const double* Bd = static_cast<const double*>(a->B);
  const int slot = trace_begin("ozaki_panels", a->dtype, M, a->N, K, nmod, st);
  if (!err) {
    View va{Ad, a->lda, akc, 1, 0, 1.0};
    if (cudaMemsetAsync(w, 0, sizeof(CallWords), st) != cudaSuccess) err = XKB_ECUDA;
    if (!err) err = launch_norm(va, M, K, 0, part, mu, &w->rmax[0], st);
    if (!err) err = launch_pick(w, pl, false, st);
    if (!err) err = launch_res(va, M, K, mu, sel, c, Ap, Mpad, Kpad, 0, st);
    if (!err && Kpad > (long)rup(K, 64)) {
      const size_t kz = rup(K, 64);
      if (cudaMemset2DAsync(Ap + kz, Kpad, 0, Kpad - kz, (size_t)nmod * Mpad, st) != cudaSuccess)
        err = XKB_ECUDA;
    }
  }
  trace_mark(slot, 1, st);
  for (int q = 0; q < npanel; ++q) {
    wait(q);
    const long n0 = bounds[q], nw = bounds[q + 1] - bounds[q];
    const long npad = (long)rup((size_t)nw, BN);
    if (!err) {
      // columns n0.. of op(B): opB == N -> B[k + j ldb]; else B[j + k ldb]
      View vb{bkc ? Bd + n0 * a->ldb : Bd + n0, a->ldb, bkc, 1, 0, 1.0};
      err = launch_norm(vb, (int)nw, K, 0, part, nu + n0, &w->rmax[1], st);
      if (!err) err = launch_res(vb, (int)nw, K, nu + n0, sel, c, Bp, npad, Kpad, 0, st);
      if (!err && Kpad > (long)rup(K, 64)) {
        const size_t kz = rup(K, 64);
        if (cudaMemset2DAsync(Bp + kz, Kpad, 0, Kpad - kz, (size_t)nmod * npad, st) != cudaSuccess)
          err = XKB_ECUDA;
      }
      if (!err)
        err = launch_gemm(Ap, Mpad, Bp, npad, Mpad, npad, Kpad, c, sel, R, XKB_FULL, 0, st);
      if (!err) {
        CrtP cp;
        std::memset(&cp, 0, sizeof(cp));
        cp.M = M;
        cp.N = (int)nw;
        cp.R = R;
        cp.Mpad = Mpad;
        cp.Npad = npad;
        cp.mu = mu;
        cp.nu = nu + n0;
        cp.sel = sel;
        cp.C = static_cast<double*>(a->C) + n0 * a->ldc;
        cp.ldc = a->ldc;
        cp.ar = a->alpha[0];
        cp.br = a->beta[0];
        cp.uplo = XKB_FULL;
        const dim3 cg((unsigned)(((M + 3) / 4 + 255) / 256), (unsigned)std::min<long>(nw, 65535));
        err = launch_crt(cg, st, cp, c, c, nullptr);
      }
    }
    done(q);  // recorded on every path: waiters never hang on an error
  }
  trace_mark(slot, 2, st);
  trace_mark(slot, 3, st);
  if (Ap) cudaFreeAsync(Ap, st);
  if (Bp) cudaFreeAsync(Bp, st);
  if (R) cudaFreeAsync(R, st);
  if (mu) cudaFreeAsync(mu, st);
  if (nu) cudaFreeAsync(nu, st);
  if (pw) cudaFreeAsync(pw, st);
  return err;
}

// Row blocks of op(A) and column panels of op(B) landing in the order `seq`
// names; see include/xkb_cuda.h.  Every block is converted once, when it
// lands, into residue planes that hold all of op(A) (all of op(B)); the
// products of the newly landed block with all the blocks of the other
// operand converted before it form one rectangle of C -- one INT8 launch,
// one CRT -- whose completion is recorded on done_ev[k].  Row blocks and
// column panels each land in increasing order, so those rectangles are
// [row block i] x [0, the columns landed so far) or [0, the rows landed so
// far) x [panel j], and together they cover C once.
extern "C" int xkb_cuda_ozaki_gemm_blocks(const xkb_gemm_args* a, int nmod, void* stream, int nr,
                                          const long* rb, int nc, const long* cb, const int* seq,
                                          void* const* a_ev, void* const* b_ev,
                                          void* const* done_ev) {
  if (!a || a->dtype != XKB_D || a->uplo != XKB_FULL || nr < 1 || nc < 1 || !rb || !cb || !seq)
    return XKB_EINVAL;
  if (a->M < 0 || a->N < 0 || a->K < 0) return XKB_EINVAL;
  if (rb[0] != 0 || rb[nr] != a->M || cb[0] != 0 || cb[nc] != a->N) return XKB_EINVAL;
  // interior bounds on multiples of 256: block and panel offsets then fall on
  // INT8 tile and TMA boundaries of the residue planes
  for (int i = 0; i < nr; ++i)
    if (rb[i + 1] <= rb[i] || (i > 0 && rb[i] % 256 != 0)) return XKB_EINVAL;
  for (int j = 0; j < nc; ++j)
    if (cb[j + 1] <= cb[j] || (j > 0 && cb[j] % 256 != 0)) return XKB_EINVAL;
  {
    int ni = 0, nj = 0;  // each block once, row blocks and panels in increasing order
    for (int k = 0; k < nr + nc; ++k) {
      if (seq[k] < 0) {
        if (-1 - seq[k] != ni) return XKB_EINVAL;
        ++ni;
      } else {
        if (seq[k] != nj) return XKB_EINVAL;
        ++nj;
      }
    }
    if (ni != nr || nj != nc) return XKB_EINVAL;
  }
  cudaStream_t st = resolve_stream(stream);
  const int nseq = nr + nc;
  auto wait = [&](void* const* evs, int q) {
    if (evs && evs[q]) cudaStreamWaitEvent(st, static_cast<cudaEvent_t>(evs[q]), 0);
  };
  auto done = [&](int k) {
    if (done_ev && done_ev[k]) cudaEventRecord(static_cast<cudaEvent_t>(done_ev[k]), st);
  };
  if (a->M == 0 || a->K == 0 || a->alpha[0] == 0.0 || a->K > 131072) {
    // nothing to pipeline: every operand, then one plain product
    for (int k = 0; k < nseq; ++k) wait(seq[k] < 0 ? a_ev : b_ev, seq[k] < 0 ? -1 - seq[k] : seq[k]);
    const int r = a->K > 131072 ? XKB_ERANGE : (a->M == 0 ? XKB_OK : xkb_cuda_gemm(a, st));
    for (int k = 0; k < nseq; ++k) done(k);
    return r;
  }
  // blocks are converted before the other operand has landed: the count is
  // fixed for the call (the tuning table's or the K rule's when nmod == 0)
  if (nmod == 0) nmod = default_moduli(a->K);
  ModPlan pl;
  if (!plan_moduli(nmod, a->K, &pl)) return XKB_ERANGE;
  const Consts* c = pl.chi;
  const int M = a->M, N = a->N, K = a->K;
  const long Kpad = (long)rup(K, BKB), Mpad = (long)rup(M, BM2), Npad = (long)rup(N, BN2);
  long rmax = 0, cmax = 0;
  for (int i = 0; i < nr; ++i) rmax = std::max(rmax, rb[i + 1] - rb[i]);
  for (int j = 0; j < nc; ++j) cmax = std::max(cmax, cb[j + 1] - cb[j]);
  const bool akc = a->opA != XKB_OP_N, bkc = a->opB == XKB_OP_N;
  const int nch = (int)((K + kNormChunk - 1) / kNormChunk);
  int8_t *Ap = nullptr, *Bp = nullptr;
  uint8_t* R = nullptr;
  int *mu = nullptr, *nu = nullptr;
  unsigned char* pw = nullptr;  // CallWords, then the norm partials from byte 256
  auto alloc = [&](void** p, size_t n) {
    return cudaMallocAsync(p, std::max<size_t>(n, 256), st) == cudaSuccess;
  };
  // the largest rectangle: all rows x one panel, or one row block x all columns
  const size_t rsz = std::max((size_t)Mpad * rup((size_t)cmax, BN), rup((size_t)rmax, BM) * (size_t)Npad);
  bool ok = alloc((void**)&Ap, (size_t)nmod * Mpad * Kpad) &&
            alloc((void**)&Bp, (size_t)nmod * Npad * Kpad) && alloc((void**)&R, (size_t)nmod * rsz) &&
            alloc((void**)&mu, sizeof(int) * M) && alloc((void**)&nu, sizeof(int) * N) &&
            alloc((void**)&pw, 256 + sizeof(double4) * (size_t)nch * (size_t)std::max(rmax, cmax));
  int err = ok ? XKB_OK : XKB_ENOMEM;
  if (!ok) cudaGetLastError();
  CallWords* w = reinterpret_cast<CallWords*>(pw);
  double4* part = reinterpret_cast<double4*>(pw + 256);
  const OzSel* sel = w ? &w->sel : nullptr;
  const double* Ad = static_cast<const double*>(a->A);
  const double* Bd = static_cast<const double*>(a->B);
  const int slot = trace_begin("ozaki_blocks", a->dtype, M, N, K, nmod, st);
  if (!err) {
    if (cudaMemsetAsync(w, 0, sizeof(CallWords), st) != cudaSuccess) err = XKB_ECUDA;
    if (!err) err = launch_pick(w, pl, false, st);
    // k columns past K (to the INT8 k-block) are zero in every plane
    const size_t kz = rup(K, 64);
    if (!err && Kpad > (long)kz &&
        (cudaMemset2DAsync(Ap + kz, Kpad, 0, Kpad - kz, (size_t)nmod * Mpad, st) != cudaSuccess ||
         cudaMemset2DAsync(Bp + kz, Kpad, 0, Kpad - kz, (size_t)nmod * Npad, st) != cudaSuccess))
      err = XKB_ECUDA;
  }
  trace_mark(slot, 1, st);
  int ra = 0, cn = 0;  // row blocks / panels landed so far
  for (int k = 0; k < nseq; ++k) {
    long r0, r1, c0, c1;  // the rectangle of C this landing completes
    if (seq[k] < 0) {
      const int i = -1 - seq[k];
      wait(a_ev, i);
      r0 = rb[i];
      r1 = rb[i + 1];
      c0 = 0;
      c1 = cb[cn];
      if (!err) {
        // rows r0.. of op(A): opA == N -> A[i + k lda]; else A[k + i lda]
        View va{akc ? Ad + r0 * a->lda : Ad + r0, a->lda, akc, 1, 0, 1.0};
        const int L = (int)(r1 - r0);
        err = launch_norm(va, L, K, 0, part, mu + r0, &w->rmax[0], st);
        if (!err)
          err = launch_res(va, L, K, mu + r0, sel, c, Ap + r0 * Kpad, Mpad, Kpad, 0, st,
                           (long)rup((size_t)L, 64));
      }
      ++ra;
    } else {
      const int j = seq[k];
      wait(b_ev, j);
      r0 = 0;
      r1 = rb[ra];
      c0 = cb[j];
      c1 = cb[j + 1];
      if (!err) {
        // columns c0.. of op(B): opB == N -> B[k + j ldb]; else B[j + k ldb]
        View vb{bkc ? Bd + c0 * a->ldb : Bd + c0, a->ldb, bkc, 1, 0, 1.0};
        const int L = (int)(c1 - c0);
        err = launch_norm(vb, L, K, 0, part, nu + c0, &w->rmax[1], st);
        if (!err)
          err = launch_res(vb, L, K, nu + c0, sel, c, Bp + c0 * Kpad, Npad, Kpad, 0, st,
                           (long)rup((size_t)L, 64));
      }
      ++cn;
    }
    if (!err && r1 > r0 && c1 > c0) {
      const long mp = (long)rup((size_t)(r1 - r0), BM), np = (long)rup((size_t)(c1 - c0), BN);
      err = launch_gemm(Ap + r0 * Kpad, mp, Bp + c0 * Kpad, np, mp, np, Kpad, c, sel, R, XKB_FULL,
                        0, st, Mpad, Npad);
      if (!err) {
        CrtP cp;
        std::memset(&cp, 0, sizeof(cp));
        cp.M = (int)(r1 - r0);
        cp.N = (int)(c1 - c0);
        cp.R = R;
        cp.Mpad = mp;
        cp.Npad = np;
        cp.mu = mu + r0;
        cp.nu = nu + c0;
        cp.sel = sel;
        cp.C = static_cast<double*>(a->C) + r0 + c0 * a->ldc;
        cp.ldc = a->ldc;
        cp.ar = a->alpha[0];
        cp.br = a->beta[0];
        cp.uplo = XKB_FULL;
        const dim3 cg((unsigned)(((cp.M + 3) / 4 + 255) / 256), (unsigned)std::min<long>(cp.N, 65535));
        err = launch_crt(cg, st, cp, c, c, nullptr);
      }
    }
    done(k);  // recorded on every path: waiters never hang on an error
  }
  trace_mark(slot, 2, st);
  trace_mark(slot, 3, st);
  if (Ap) cudaFreeAsync(Ap, st);
  if (Bp) cudaFreeAsync(Bp, st);
  if (R) cudaFreeAsync(R, st);
  if (mu) cudaFreeAsync(mu, st);
  if (nu) cudaFreeAsync(nu, st);
  if (pw) cudaFreeAsync(pw, st);
  return err;
}

// ===========================================================================
// Scratch-free variant of the real Ozaki contraction.
//
// Who needs it: callers that cannot ask the CUDA allocator for memory at call
// time -- for example a program that has already handed all free device
// memory to its own caching allocator (cudaMallocAsync would then fail), or a
// latency-bound loop that must not risk an allocation stalling or failing in
// the middle of a step.  xkb_cuda_ozaki_gemm takes its scratch (residue
// planes, shifts, norm partials) from the stream-ordered pool on every call;
// this entry point takes it from one fixed device array compiled into the
// library instead, and allocates nothing.
//
// Limits and rules:
//   * real double (XKB_D) only, M, N, K <= kNoAllocMaxDim (512); larger sizes
//     are refused with XKB_ERANGE before anything is launched;
//   * the array (kNoAllocBytes, about 12.6 MiB) lives in every GPU that
//     loads this library, for the life of the process;
//   * all calls share it: two calls whose kernels overlap on the GPU (other
//     streams, other host threads) race on it and corrupt each other --
//     serialise them;
//   * the array is placed in device memory when this file's CUDA module is
//     loaded, which with lazy module loading (the CUDA 12 default) happens
//     at its first use, not when the library is opened.  noalloc_prepare()
//     -- run by xkblas_init() for its device, or else by the first call of
//     this entry point on a device -- looks the array's address up with
//     cudaGetSymbolAddress (that device current), which loads the module, and
//     loads every kernel this entry point launches.  A caller that is about
//     to hand the free device memory to its own allocator therefore calls
//     xkblas_init() (or this entry point once) first; that first call should
//     also come before any stream capture;
//   * the address is cached per device together with the CUDA context's
//     unique ID; after cudaDeviceReset() the next call sees a new context and
//     looks the (reloaded) array up again.
// Nothing in the array has to start at zero: every byte a call reads is
// written earlier in the same call (planes padded by the residue kernel and a
// 2-D memset, row codes and partials fully rewritten, the call's moduli
// selection words cleared by a memset first).
namespace xkb {
namespace oz {
constexpr int kNoAllocMaxDim = 512;
// per-plane rows and k extent at the limit: max(rup(512,128), rup(512,256))
constexpr size_t kNoAllocRows = 512, kNoAllocK = 512;
constexpr size_t kNoAllocPlane = kNoAllocRows * kNoAllocK;              // bytes
constexpr size_t kNoAllocA = kMaxMod * kNoAllocPlane;                  // A planes
constexpr size_t kNoAllocB = kMaxMod * kNoAllocPlane;                  // B planes
constexpr size_t kNoAllocR = kMaxMod * kNoAllocRows * kNoAllocRows;    // C residues
constexpr size_t kNoAllocShift = 2 * 4 * kNoAllocRows;                 // mu, nu
constexpr size_t kNoAllocPart = sizeof(double4) * 2 * kNoAllocRows;    // 1 k-chunk
constexpr size_t kNoAllocBytes =
    kNoAllocA + kNoAllocB + kNoAllocR + kNoAllocShift + kNoAllocPart + 4096;

static __device__ __align__(256) unsigned char g_oz_noalloc_scratch[kNoAllocBytes];

// C <- beta C on the masked part (beta == 0 writes zeros without reading),
// for K == 0 or alpha == 0: kept in this file so that the scratch-free path
// launches only kernels of this module (loaded by noalloc_prepare).
__global__ void k_oz_beta(int M, int N, double beta, double* C, long ldc, int uplo, long diag) {
  const size_t total = (size_t)M * (size_t)N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const long i = (long)(e % (size_t)M), j = (long)(e / (size_t)M);
    if (uplo == XKB_LOWER && i + diag < j) continue;
    if (uplo == XKB_UPPER && i + diag > j) continue;
    double* c = C + (size_t)i + (size_t)j * (size_t)ldc;
    *c = beta != 0.0 ? beta * *c : 0.0;
  }
}

typedef CUresult (*PFN_ctxGetCurrent)(CUcontext*);
typedef CUresult (*PFN_ctxGetId)(CUcontext, unsigned long long*);

// Unique ID of the calling thread's current CUDA context (0 if unknown or
// none is current).
static unsigned long long current_ctx_id() {
  static PFN_ctxGetCurrent get_cur = nullptr;
  static PFN_ctxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<PFN_ctxGetCurrent>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_ctxGetId>(p);
    cudaGetLastError();
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Kernels the scratch-free path launches, loaded up front (with lazy loading
// a kernel's code is otherwise placed in device memory at its first launch).
template <int NM>
static bool load_nm_kernels() {
  cudaFuncAttributes fa;
  return cudaFuncGetAttributes(&fa, k_oz_residues<true, NM>) == cudaSuccess &&
         cudaFuncGetAttributes(&fa, k_oz_residues<false, NM>) == cudaSuccess &&
         cudaFuncGetAttributes(&fa, k_oz_crt<NM>) == cudaSuccess;
}
static bool load_noalloc_kernels() {
  cudaFuncAttributes fa;
  bool ok = cudaFuncGetAttributes(&fa, k_oz_norm<true>) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_norm<false>) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_stat) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_pick) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_crt_15_16) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_gemm) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, k_oz_beta) == cudaSuccess;
  ok = ok && load_nm_kernels<2>() && load_nm_kernels<3>() && load_nm_kernels<4>() &&
       load_nm_kernels<5>() && load_nm_kernels<6>() && load_nm_kernels<7>() &&
       load_nm_kernels<8>() && load_nm_kernels<9>() && load_nm_kernels<10>() &&
       load_nm_kernels<11>() && load_nm_kernels<12>() && load_nm_kernels<13>() &&
       load_nm_kernels<14>() && load_nm_kernels<15>() && load_nm_kernels<16>();
  return ok;
}

// Device address of the array for the current device, looked up when the
// device's context is seen for the first time (once per device, unless the
// context is reset).
static int noalloc_base(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* ptr[64] = {nullptr};
  static unsigned long long ctx_of[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return XKB_ECUDA;
  std::lock_guard<std::mutex> g(mu);
  const unsigned long long id = current_ctx_id();
  if (!ptr[dev] || id == 0 || id != ctx_of[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_oz_noalloc_scratch) != cudaSuccess || !p ||
        !load_noalloc_kernels()) {
      cudaGetLastError();
      ptr[dev] = nullptr;
      return XKB_ECUDA;
    }
    ptr[dev] = static_cast<unsigned char*>(p);
    ctx_of[dev] = current_ctx_id();  // the lookup made the primary context current
  }
  *out = ptr[dev];
  return XKB_OK;
}
}  // namespace oz

int noalloc_prepare() {
  unsigned char* p = nullptr;
  return oz::noalloc_base(&p);
}
}  // namespace xkb

extern "C" int xkb_cuda_ozaki_gemm_noalloc(const xkb_gemm_args* a, int nmod, void* stream) {
  if (!a || a->dtype != XKB_D) return XKB_EINVAL;
  if (a->M < 0 || a->N < 0 || a->K < 0) return XKB_EINVAL;
  if (a->M > kNoAllocMaxDim || a->N > kNoAllocMaxDim || a->K > kNoAllocMaxDim) return XKB_ERANGE;
  if (a->M == 0 || a->N == 0) return XKB_OK;
  if (a->K > 0 && a->alpha[0] != 0.0 && (a->opA < XKB_OP_N || a->opA > XKB_OP_C ||
                                         a->opB < XKB_OP_N || a->opB > XKB_OP_C))
    return XKB_EINVAL;
  // nmod == 0: the data rule's count, at most 16 (there is no plain fallback
  // here: the plain kernel may need scratch for unaligned operands)
  ModPlan pl;
  if (!plan_moduli(nmod, a->K > 0 ? a->K : 1, &pl)) return XKB_ERANGE;
  const Consts* c = pl.chi;
  nmod = pl.hi;
  unsigned char* base = nullptr;
  int err = noalloc_base(&base);
  if (err) return err;
  cudaStream_t st = resolve_stream(stream);
  if (a->K == 0 || a->alpha[0] == 0.0) {  // beta C only
    const size_t total = (size_t)a->M * (size_t)a->N;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 1024);
    const long long tv = evlog_kern_begin(st, "k_oz_beta");
    k_oz_beta<<<blocks, 256, 0, st>>>(a->M, a->N, a->beta[0], static_cast<double*>(a->C), a->ldc,
                                      a->uplo, a->diag);
    evlog_kern_end(tv, st);
    count_launch();
    return cudaPeekAtLastError() == cudaSuccess ? XKB_OK : XKB_ECUDA;
  }
  const int M = a->M, N = a->N, K = a->K;
  const long Kpad = (long)rup(K, BKB), Mpad = (long)rup(M, BM), Npad = (long)rup(N, BN);
  const bool akc = a->opA != XKB_OP_N, bkc = a->opB == XKB_OP_N;
  const bool same = (a->A == a->B) && (a->lda == a->ldb) && (akc == bkc) && M == N;
  const long Arows = same ? std::max(Mpad, Npad) : Mpad;
  // carve the fixed array (all offsets 256-byte aligned)
  int8_t* Ap = reinterpret_cast<int8_t*>(base);
  int8_t* Bp = reinterpret_cast<int8_t*>(base + kNoAllocA);
  uint8_t* R = base + kNoAllocA + kNoAllocB;
  int* mu = reinterpret_cast<int*>(base + kNoAllocA + kNoAllocB + kNoAllocR);
  int* nu = mu + kNoAllocRows;
  unsigned char* tail = base + kNoAllocA + kNoAllocB + kNoAllocR + kNoAllocShift;
  double4* part = reinterpret_cast<double4*>(tail);
  CallWords* w = reinterpret_cast<CallWords*>(tail + kNoAllocPart);
  const OzSel* sel = &w->sel;
  const double* Ad = static_cast<const double*>(a->A);
  const double* Bd = static_cast<const double*>(a->B);
  const int slot = trace_begin("ozaki_noalloc", a->dtype, M, N, K, pl.fixed ? nmod : 0, st);
  View va{Ad, a->lda, akc, 1, 0, 1.0}, vb{Bd, a->ldb, bkc, 1, 0, 1.0};
  if (cudaMemsetAsync(w, 0, sizeof(CallWords), st) != cudaSuccess) err = XKB_ECUDA;
  if (!err) err = launch_norm(va, M, K, 0, part, mu, &w->rmax[0], st);
  if (!err) err = launch_norm(vb, N, K, 0, part + kNoAllocRows, nu, &w->rmax[1], st);
  if (!err) err = launch_pick(w, pl, false, st);
  if (!err) err = launch_res(va, M, K, mu, sel, c, Ap, Arows, Kpad, 0, st);
  if (!err && !same) err = launch_res(vb, N, K, nu, sel, c, Bp, Npad, Kpad, 0, st);
  if (!err && Kpad > (long)rup(K, 64)) {
    const size_t kz = rup(K, 64);
    if (cudaMemset2DAsync(Ap + kz, Kpad, 0, Kpad - kz, (size_t)nmod * Arows, st) != cudaSuccess ||
        (!same &&
         cudaMemset2DAsync(Bp + kz, Kpad, 0, Kpad - kz, (size_t)nmod * Npad, st) != cudaSuccess))
      err = XKB_ECUDA;
  }
  trace_mark(slot, 1, st);
  if (!err)
    err = same ? launch_gemm(Ap, Arows, Ap, Arows, Mpad, Npad, Kpad, c, sel, R, a->uplo, a->diag,
                             st)
               : launch_gemm(Ap, Mpad, Bp, Npad, Mpad, Npad, Kpad, c, sel, R, a->uplo, a->diag,
                             st);
  trace_mark(slot, 2, st);
  if (!err) {
    CrtP cp;
    std::memset(&cp, 0, sizeof(cp));
    cp.M = M;
    cp.N = N;
    cp.R = R;
    cp.Mpad = Mpad;
    cp.Npad = Npad;
    cp.mu = mu;
    cp.nu = nu;
    cp.sel = sel;
    cp.C = static_cast<double*>(a->C);
    cp.ldc = a->ldc;
    cp.ar = a->alpha[0];
    cp.br = a->beta[0];
    cp.uplo = a->uplo;
    cp.diag = a->diag;
    const dim3 cg((unsigned)(((M + 3) / 4 + 255) / 256), (unsigned)N);
    err = launch_crt(cg, st, cp, pl.clo, pl.chi, nullptr);
  }
  trace_mark(slot, 3, st);
  return err;
}
