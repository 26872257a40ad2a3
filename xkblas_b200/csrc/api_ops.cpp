// api_ops.cpp -- the level-3 entry points of xkblas.h (s/d/c/z):
// argument checking with the reference's -i codes, quick returns, tile
// directory acquisition, and the device call that replaces the reference's
// tile-task insertion loops.
//
// Reference drivers (argument checks / quick returns / tile loops):
//   gemm  blas/zgemm.c:118-370      gemmt blas/zgemmt.c:114-390
//   trsm  blas/ztrsm.c:102-499      trmm  blas/ztrmm.c:101-460
//   symm  blas/zsymm.c:107-400      hemm  blas/zhemm.c:106-390
//   syrk  blas/zsyrk.c:97-319       herk  blas/zherk.c:97-320
//   syr2k blas/zsyr2k.c:107-330     her2k blas/zher2k.c:107-383
// Instead of one task per NB x NB tile, each call becomes one (or, for
// trsm, a short sequence of) whole-matrix kernel launch on the compute
// stream; the tile directory supplies the operands and records what the
// call wrote.  Divergences from the reference, all deliberate:
//   * errors are returned, never abort();
//   * gemmt writes only the uplo triangle (the reference's GPU body writes
//     the whole diagonal tile, blas/ztask_gemmt.c:213);
//   * float / complex-float operands are computed in FP64 and rounded once.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <complex>
#include <cstring>

#include "runtime.hpp"

using namespace xkbrt;

namespace {

template <class T>
struct HT;
template <>
struct HT<float> {
  static constexpr int dt = XKB_S;
  static constexpr bool cplx = false;
};
template <>
struct HT<double> {
  static constexpr int dt = XKB_D;
  static constexpr bool cplx = false;
};
template <>
struct HT<Complex32_t> {
  static constexpr int dt = XKB_C;
  static constexpr bool cplx = true;
};
template <>
struct HT<Complex64_t> {
  static constexpr int dt = XKB_Z;
  static constexpr bool cplx = true;
};

// Call name for the trace (reference names: precision letter + operation,
// e.g. "dgemm", blas/zgemm.c:262), 7 characters at most.
struct OpName {
  char s[8];
  OpName(int dt, const char* op) {
    s[0] = "sdcz"[dt == XKB_S ? 0 : dt == XKB_D ? 1 : dt == XKB_C ? 2 : 3];
    std::strncpy(s + 1, op, 6);
    s[7] = 0;
  }
};
using U64 = uint64_t;

template <class T>
void sc(const T& v, double out[2]) {
  if constexpr (HT<T>::cplx) {
    out[0] = (double)v.real();
    out[1] = (double)v.imag();
  } else {
    out[0] = (double)v;
    out[1] = 0.0;
  }
}
template <class T>
bool is_zero(const T& v) {
  return v == T(0);
}
template <class T>
bool is_one(const T& v) {
  return v == T(1);
}

int opcode(int t) { return t == CblasNoTrans ? XKB_OP_N : (t == CblasTrans ? XKB_OP_T : XKB_OP_C); }
int maskcode(int uplo) { return uplo == CblasLower ? XKB_LOWER : XKB_UPPER; }

// Host error mapping: argument errors are -i; runtime failures are positive
// errno values so they never collide with an argument index.
int rt_error(int xkb) {
  switch (xkb) {
    case XKB_OK: return 0;
    case XKB_ENODEV: return ENODEV;
    case XKB_ENOMEM: return ENOMEM;
    case XKB_ETIMEDOUT: return ETIMEDOUT;
    case XKB_ERANGE: return ERANGE;
    default: return EIO;
  }
}

struct Guard {
  std::lock_guard<std::recursive_mutex> g;
  Guard() : g(rt().mu) { rt().call_epoch++; }  // operands of this call are not evicted by it
};

bool use_ozaki(int dt, long m, long n, long k) {
  Runtime& R = rt();
  if (thread_math() != XKBLAS_TENSOR_OP_MATH) return false;
  if (dt != XKB_D && dt != XKB_Z) return false;
  return std::min(m, std::min(n, k)) >= ozaki_min_dim() && xkb_ozaki_default_moduli(k) > 0;
}

// One contraction on device operands: plain DMMA or Ozaki.
int run_gemm(xkb_gemm_args& a) {
  Runtime& R = rt();
  if (int e = flush_pending()) return e;  // queued calls first, in call order
  if (use_ozaki(a.dtype, a.M, a.N, a.K)) {
    // XKBLAS_OZAKI_SLICES fixes the count; otherwise it is chosen on the
    // device from the operands (xkb_cuda_ozaki_gemm with nmod = 0)
    int e = xkb_cuda_ozaki_gemm(&a, R.ozaki_moduli, R.s_comp);
    if (e != XKB_ERANGE) return e;
  }
  return xkb_cuda_gemm(&a, R.s_comp);
}

template <class T>
xkb_gemm_args base_args(int opA, int opB, int M, int N, int K, const T* alpha, const T* beta) {
  xkb_gemm_args a{};
  a.dtype = HT<T>::dt;
  a.opA = opA;
  a.opB = opB;
  a.M = M;
  a.N = N;
  a.K = K;
  sc(*alpha, a.alpha);
  sc(*beta, a.beta);
  a.uplo = XKB_FULL;
  a.herm_diag = 0;
  a.diag = 0;
  return a;
}

// ---------------------------------------------------------------------------
template <class T>
int gemm_async(int transA, int transB, int M, int N, int K, const T* alpha, const T* A, int LDA,
               const T* B, int LDB, const T* beta, T* C, int LDC) {
  if (transA < CblasNoTrans || transA > CblasConjTrans) return -1;
  if (transB < CblasNoTrans || transB > CblasConjTrans) return -2;
  const int Am = transA == CblasNoTrans ? M : K, An = transA == CblasNoTrans ? K : M;
  const int Bm = transB == CblasNoTrans ? K : N, Bn = transB == CblasNoTrans ? N : K;
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (LDA < std::max(1, Am)) return -8;
  if (LDB < std::max(1, Bm)) return -10;
  if (LDC < std::max(1, M)) return -13;
  if (M == 0 || N == 0 || ((is_zero(*alpha) || K == 0) && is_one(*beta))) return 0;
  const OpName op_name(HT<T>::dt, "gemm");
  xkb::EvCall ev_call(op_name.s,
                      {U64(M), U64(N), U64(K),
                       U64(xkb::evlog_on() ? auto_tilesize(KERN_GEMM, M, N, K) : 0), U64(transA),
                       U64(transB), 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  add_flops(op_name.s, (HT<T>::cplx ? 8.0 : 2.0) * M * (double)N * K);
  const size_t NB = auto_tilesize(KERN_GEMM, M, N, K), es = sizeof(T);
  int err;
  const bool need_ab = !is_zero(*alpha) && K > 0;
  // Large real Ozaki contractions with op(B) = B and beta = 0 run block by
  // block: op(A) crosses the host link in row blocks and B in column panels,
  // interleaved so that the landed fractions of both grow together; every
  // landed block is multiplied with all of the other operand landed before
  // it, and coherence copies each finished rectangle of C back.  The
  // arithmetic (and the copy-back) starts after the first row block instead
  // of after all of op(A).  Tuning key ozaki_row_blocks (default 1; 0: the
  // column-panel form below), rows per block ozaki_block_rows (1024).
  if (need_ab && HT<T>::dt == XKB_D && transB == CblasNoTrans && N >= 4096 && M >= 4096 &&
      is_zero(*beta) && use_ozaki(XKB_D, M, N, K) &&
      xkb_tune_get("ozaki_row_blocks", 1.0) != 0.0) {
    if ((err = flush_pending())) return rt_error(err);
    Desc* dA = get_desc(A, Am, An, LDA, es, NB, &err);
    if (!dA) return rt_error(err);
    Desc* dB = get_desc(B, Bm, Bn, LDB, es, NB, &err);
    if (!dB) return rt_error(err);
    Desc* dC = get_desc(C, M, N, LDC, es, NB, &err);
    if (!dC) return rt_error(err);
    const long h = std::max<long>(256, (long)xkb_tune_get("ozaki_block_rows", 1024.0)) / 256 * 256;
    const long pc = std::max<long>(256, (long)xkb_tune_get("ozaki_panel_cols", 1024.0));
    const long np = std::min<long>(32, std::max<long>(2, N / pc));
    const long w = ((N + np - 1) / np + 255) / 256 * 256;
    std::vector<long> rb{0}, cb{0};
    while (rb.back() < M) rb.push_back(std::min<long>(M, rb.back() + h));
    while (cb.back() < N) cb.push_back(std::min<long>(N, cb.back() + w));
    const long nr = (long)rb.size() - 1, nc = (long)cb.size() - 1;
    // landing order: the next row block while the landed fraction of op(A)
    // does not exceed that of B
    std::vector<int> seq;
    for (long i = 0, j = 0; i < nr || j < nc;) {
      if (i < nr && (j >= nc || i * nc <= j * nr)) seq.push_back((int)(-1 - i++));
      else seq.push_back((int)j++);
    }
    std::vector<EventRef> fin(seq.size());
    std::vector<cudaEvent_t> ev_a, ev_b, done(seq.size());
    for (size_t k = 0; k < fin.size(); ++k) {
      if (!(fin[k] = new_event_ref())) return rt_error(XKB_ECUDA);
      done[k] = fin[k]->e;
    }
    if ((err = make_valid_blocks(dA, transA != CblasNoTrans, (size_t)K, rb, dB, cb, seq, ev_a,
                                 ev_b)))
      return rt_error(err);
    xkb_gemm_args a = base_args<T>(opcode(transA), opcode(transB), M, N, K, alpha, beta);
    a.A = dev_ptr(dA, 0, 0);
    a.lda = (long)dA->dld;
    a.B = dev_ptr(dB, 0, 0);
    a.ldb = (long)dB->dld;
    a.C = dev_ptr(dC, 0, 0);
    a.ldc = (long)dC->dld;
    const int nm = R.ozaki_moduli ? R.ozaki_moduli : xkb_ozaki_default_moduli(K);
    err = xkb_cuda_ozaki_gemm_blocks(&a, nm, R.s_comp, (int)nr, rb.data(), (int)nc, cb.data(),
                                     seq.data(), reinterpret_cast<void* const*>(ev_a.data()),
                                     reinterpret_cast<void* const*>(ev_b.data()),
                                     reinterpret_cast<void* const*>(done.data()));
    if (err) return rt_error(err);
    mark_full_overwrite(dC, 0, M, 0, N);
    // the rectangle each landing completed (as xkb_cuda_ozaki_gemm_blocks)
    long ra = 0, cn = 0;
    for (size_t k = 0; k < seq.size(); ++k) {
      long r0, r1, c0, c1;
      if (seq[k] < 0) {
        const long i = -1 - seq[k];
        r0 = rb[i], r1 = rb[i + 1], c0 = 0, c1 = cb[cn];
        ++ra;
      } else {
        r0 = 0, r1 = rb[ra], c0 = cb[seq[k]], c1 = cb[seq[k] + 1];
        ++cn;
      }
      if (r1 > r0 && c1 > c0)
        dC->ready.push_back({(size_t)r0, (size_t)r1, (size_t)c0, (size_t)c1, fin[k]});
    }
    return 0;
  }
  // Large real Ozaki contractions with op(B) = B run panel by panel: B (and
  // C) cross the host link in column panels, each panel is multiplied as soon
  // as its operands landed, and coherence copies each finished panel back.
  if (need_ab && HT<T>::dt == XKB_D && transB == CblasNoTrans && N >= 4096 &&
      use_ozaki(XKB_D, M, N, K)) {
    if ((err = flush_pending())) return rt_error(err);
    Desc* dA = get_desc(A, Am, An, LDA, es, NB, &err);
    if (!dA) return rt_error(err);
    if ((err = make_valid(dA, 0, Am, 0, An))) return rt_error(err);  // compute waits for A
    Desc* dB = get_desc(B, Bm, Bn, LDB, es, NB, &err);
    if (!dB) return rt_error(err);
    Desc* dC = get_desc(C, M, N, LDC, es, NB, &err);
    if (!dC) return rt_error(err);
    const long pc = std::max<long>(256, (long)xkb_tune_get("ozaki_panel_cols", 1024.0));
    const long np = std::min<long>(32, std::max<long>(2, N / pc));
    const long w = ((N + np - 1) / np + 255) / 256 * 256;  // multiple of the INT8 tile width
    std::vector<long> bounds{0};
    while (bounds.back() < N) bounds.push_back(std::min<long>(N, bounds.back() + w));
    std::vector<std::pair<Desc*, size_t>> in{{dB, (size_t)K}};
    if (!is_zero(*beta)) in.emplace_back(dC, (size_t)M);
    // completion events stay with C until its coherence point: not taken
    // from the recycled pool
    std::vector<EventRef> fin(bounds.size() - 1);
    std::vector<cudaEvent_t> ev, done(fin.size());
    for (size_t p = 0; p < fin.size(); ++p) {
      if (!(fin[p] = new_event_ref())) return rt_error(XKB_ECUDA);
      done[p] = fin[p]->e;
    }
    if ((err = make_valid_panels(in, bounds, ev))) return rt_error(err);
    xkb_gemm_args a = base_args<T>(opcode(transA), opcode(transB), M, N, K, alpha, beta);
    a.A = dev_ptr(dA, 0, 0);
    a.lda = (long)dA->dld;
    a.B = dev_ptr(dB, 0, 0);
    a.ldb = (long)dB->dld;
    a.C = dev_ptr(dC, 0, 0);
    a.ldc = (long)dC->dld;
    const int nm = R.ozaki_moduli ? R.ozaki_moduli : xkb_ozaki_default_moduli(K);
    err = xkb_cuda_ozaki_gemm_panels(&a, nm, R.s_comp, (int)done.size(), bounds.data(),
                                     reinterpret_cast<void* const*>(ev.data()),
                                     reinterpret_cast<void* const*>(done.data()));
    if (err) return rt_error(err);

    mark_full_overwrite(dC, 0, M, 0, N);
    for (size_t p = 0; p < fin.size(); ++p)
      dC->ready.push_back({0, (size_t)M, (size_t)bounds[p], (size_t)bounds[p + 1], fin[p]});
    return 0;
  }
  Desc *dA = nullptr, *dB = nullptr;
  if (need_ab) {
    dA = get_desc(A, Am, An, LDA, es, NB, &err);
    if (!dA) return rt_error(err);
    if ((err = make_valid(dA, 0, Am, 0, An, false))) return rt_error(err);
    dB = get_desc(B, Bm, Bn, LDB, es, NB, &err);
    if (!dB) return rt_error(err);
    if ((err = make_valid(dB, 0, Bm, 0, Bn, false))) return rt_error(err);
  }
  Desc* dC = get_desc(C, M, N, LDC, es, NB, &err);
  if (!dC) return rt_error(err);
  if (!is_zero(*beta)) {
    if ((err = make_valid(dC, 0, M, 0, N, false))) return rt_error(err);
  }
  if ((err = comp_wait_h2d())) return rt_error(err);  // one wait for the three uploads
  xkb_gemm_args a = base_args<T>(opcode(transA), opcode(transB), M, N, K, alpha, beta);
  a.A = dA ? dev_ptr(dA, 0, 0) : nullptr;
  a.lda = dA ? (long)dA->dld : 1;
  a.B = dB ? dev_ptr(dB, 0, 0) : nullptr;
  a.ldb = dB ? (long)dB->dld : 1;
  a.C = dev_ptr(dC, 0, 0);
  a.ldc = (long)dC->dld;
  if (!need_ab) a.K = 0;
  if (R.batch_on && need_ab && (a.dtype == XKB_D || a.dtype == XKB_Z) &&
      !use_ozaki(a.dtype, M, N, K)) {
    // queued for the tile-task executor (launched at the next coherence point)
    xkb_batch_op o{};
    o.kind = XKB_BATCH_GEMM;
    o.dtype = a.dtype;
    o.opA = a.opA;
    o.opB = a.opB;
    o.M = M;
    o.N = N;
    o.K = K;
    o.A = a.A;
    o.lda = a.lda;
    o.B = a.B;
    o.ldb = a.ldb;
    o.C = a.C;
    o.ldc = a.ldc;
    o.alpha[0] = a.alpha[0];
    o.alpha[1] = a.alpha[1];
    o.beta[0] = a.beta[0];
    o.beta[1] = a.beta[1];
    // marked before queueing: a flush inside defer_op then leaves C's
    // completion event in place
    mark_full_overwrite(dC, 0, M, 0, N);
    if ((err = defer_op(o, dA, dB, is_zero(*beta) ? nullptr : dC, dC))) return rt_error(err);
    return 0;
  }
  if ((err = run_gemm(a))) return rt_error(err);
  mark_full_overwrite(dC, 0, M, 0, N);
  return 0;
}

template <class T>
int gemmt_async(int uplo, int transA, int transB, int N, int K, const T* alpha, const T* A,
                int LDA, const T* B, int LDB, const T* beta, T* C, int LDC) {
  // reference blas/zgemmt.c:114-190 (uplo 0 = full product, an XKBlas extension)
  // argument codes follow the reference (transA -1, transB -2, N -4, ...);
  // the reference does not check uplo, an invalid one is reported as -1 here.
  if (transA < CblasNoTrans || transA > CblasConjTrans) return -1;
  if (transB < CblasNoTrans || transB > CblasConjTrans) return -2;
  if (uplo != 0 && uplo != CblasUpper && uplo != CblasLower) return -1;
  const int Am = transA == CblasNoTrans ? N : K, An = transA == CblasNoTrans ? K : N;
  const int Bm = transB == CblasNoTrans ? K : N, Bn = transB == CblasNoTrans ? N : K;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (LDA < std::max(1, Am)) return -8;
  if (LDB < std::max(1, Bm)) return -10;
  if (LDC < std::max(1, N)) return -13;
  if (N == 0 || ((is_zero(*alpha) || K == 0) && is_one(*beta))) return 0;
  if (uplo == 0) return gemm_async<T>(transA, transB, N, N, K, alpha, A, LDA, B, LDB, beta, C, LDC);
  const OpName op_name(HT<T>::dt, "gemmt");
  xkb::EvCall ev_call(op_name.s,
                      {U64(N), U64(K), U64(xkb::evlog_on() ? auto_tilesize(KERN_GEMMT, N, N, K) : 0),
                       U64(transA), U64(transB), 0, 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  add_flops(op_name.s, (HT<T>::cplx ? 4.0 : 1.0) * N * (double)(N + 1) * K);
  const size_t NB = auto_tilesize(KERN_GEMMT, N, N, K), es = sizeof(T);
  int err;
  const bool need_ab = !is_zero(*alpha) && K > 0;
  Desc *dA = nullptr, *dB = nullptr;
  if (need_ab) {
    if (!(dA = get_desc(A, Am, An, LDA, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dA, 0, Am, 0, An))) return rt_error(err);
    if (!(dB = get_desc(B, Bm, Bn, LDB, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dB, 0, Bm, 0, Bn))) return rt_error(err);
  }
  Desc* dC = get_desc(C, N, N, LDC, es, NB, &err);
  if (!dC) return rt_error(err);
  if ((err = make_valid(dC, 0, N, 0, N))) return rt_error(err);  // other triangle kept
  xkb_gemm_args a = base_args<T>(opcode(transA), opcode(transB), N, N, need_ab ? K : 0, alpha, beta);
  a.A = dA ? dev_ptr(dA, 0, 0) : nullptr;
  a.lda = dA ? (long)dA->dld : 1;
  a.B = dB ? dev_ptr(dB, 0, 0) : nullptr;
  a.ldb = dB ? (long)dB->dld : 1;
  a.C = dev_ptr(dC, 0, 0);
  a.ldc = (long)dC->dld;
  a.uplo = maskcode(uplo);
  if ((err = run_gemm(a))) return rt_error(err);
  mark_written(dC, 0, N, 0, N, uplo);
  return 0;
}

// syrk / herk (herm = 1: alpha, beta real, A^H, real diagonal)
template <class T>
int rk_async(int herm, int uplo, int trans, int N, int K, const T& alpha, const T* A, int LDA,
             const T& beta, T* C, int LDC) {
  if (uplo != CblasUpper && uplo != CblasLower) return -1;
  // reference: syrk/syr2k accept N or T, herk/her2k N or C (all precisions)
  if (herm) {
    if (trans != CblasNoTrans && trans != CblasConjTrans) return -2;
  } else {
    if (trans != CblasNoTrans && trans != CblasTrans) return -2;
  }
  const int Am = trans == CblasNoTrans ? N : K, An = trans == CblasNoTrans ? K : N;
  if (N < 0) return -3;
  if (K < 0) return -4;
  if (LDA < std::max(1, Am)) return -7;
  if (LDC < std::max(1, N)) return -10;
  if (N == 0 || ((is_zero(alpha) || K == 0) && is_one(beta))) return 0;
  const OpName op_name(HT<T>::dt, herm ? "herk" : "syrk");
  xkb::EvCall ev_call(op_name.s, {U64(N), U64(K), U64(uplo), U64(trans), 0, 0, 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  add_flops(op_name.s, (HT<T>::cplx ? 4.0 : 1.0) * N * (double)(N + 1) * K);
  const size_t NB = auto_tilesize(herm ? KERN_HERK : KERN_SYRK, N, N, K), es = sizeof(T);
  int err;
  const bool need_a = !is_zero(alpha) && K > 0;
  Desc* dA = nullptr;
  if (need_a) {
    if (!(dA = get_desc(A, Am, An, LDA, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dA, 0, Am, 0, An))) return rt_error(err);
  }
  Desc* dC = get_desc(C, N, N, LDC, es, NB, &err);
  if (!dC) return rt_error(err);
  if ((err = make_valid(dC, 0, N, 0, N))) return rt_error(err);
  const int tr = herm ? XKB_OP_C : XKB_OP_T;
  const int opA = trans == CblasNoTrans ? XKB_OP_N : tr;
  const int opB = trans == CblasNoTrans ? tr : XKB_OP_N;
  xkb_gemm_args a = base_args<T>(opA, opB, N, N, need_a ? K : 0, &alpha, &beta);
  a.A = dA ? dev_ptr(dA, 0, 0) : nullptr;
  a.lda = dA ? (long)dA->dld : 1;
  a.B = a.A;
  a.ldb = a.lda;
  a.C = dev_ptr(dC, 0, 0);
  a.ldc = (long)dC->dld;
  a.uplo = maskcode(uplo);
  a.herm_diag = herm;
  if ((err = run_gemm(a))) return rt_error(err);
  mark_written(dC, 0, N, 0, N, uplo);
  return 0;
}

// syr2k / her2k: C = alpha op(A) op(B)^T + alpha' op(B) op(A)^T + beta C
template <class T>
int r2k_async(int herm, int uplo, int trans, int N, int K, const T& alpha, const T* A, int LDA,
              const T* B, int LDB, const T& beta, T* C, int LDC) {
  if (uplo != CblasUpper && uplo != CblasLower) return -1;
  // reference: syrk/syr2k accept N or T, herk/her2k N or C (all precisions)
  if (herm) {
    if (trans != CblasNoTrans && trans != CblasConjTrans) return -2;
  } else {
    if (trans != CblasNoTrans && trans != CblasTrans) return -2;
  }
  const int Am = trans == CblasNoTrans ? N : K, An = trans == CblasNoTrans ? K : N;
  if (N < 0) return -3;
  if (K < 0) return -4;
  if (LDA < std::max(1, Am)) return -7;
  if (LDB < std::max(1, Am)) return -9;
  if (LDC < std::max(1, N)) return -12;
  if (N == 0 || ((is_zero(alpha) || K == 0) && is_one(beta))) return 0;
  const OpName op_name(HT<T>::dt, herm ? "her2k" : "syr2k");
  xkb::EvCall ev_call(op_name.s, {U64(N), U64(K), U64(uplo), U64(trans), 0, 0, 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  add_flops(op_name.s, (HT<T>::cplx ? 8.0 : 2.0) * N * (double)N * K);
  const size_t NB = auto_tilesize(herm ? KERN_HER2K : KERN_SYR2K, N, N, K), es = sizeof(T);
  int err;
  const bool need_ab = !is_zero(alpha) && K > 0;
  Desc *dA = nullptr, *dB = nullptr;
  if (need_ab) {
    if (!(dA = get_desc(A, Am, An, LDA, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dA, 0, Am, 0, An))) return rt_error(err);
    if (!(dB = get_desc(B, Am, An, LDB, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dB, 0, Am, 0, An))) return rt_error(err);
  }
  Desc* dC = get_desc(C, N, N, LDC, es, NB, &err);
  if (!dC) return rt_error(err);
  if ((err = make_valid(dC, 0, N, 0, N))) return rt_error(err);
  const int tr = herm ? XKB_OP_C : XKB_OP_T;
  const int opA = trans == CblasNoTrans ? XKB_OP_N : tr;
  const int opB = trans == CblasNoTrans ? tr : XKB_OP_N;
  T alpha2 = alpha;
  if constexpr (HT<T>::cplx)
    if (herm) alpha2 = std::conj(alpha);
  const T one = T(1);
  xkb_gemm_args a = base_args<T>(opA, opB, N, N, need_ab ? K : 0, &alpha, &beta);
  a.A = dA ? dev_ptr(dA, 0, 0) : nullptr;
  a.lda = dA ? (long)dA->dld : 1;
  a.B = dB ? dev_ptr(dB, 0, 0) : nullptr;
  a.ldb = dB ? (long)dB->dld : 1;
  a.C = dev_ptr(dC, 0, 0);
  a.ldc = (long)dC->dld;
  a.uplo = maskcode(uplo);
  a.herm_diag = herm;
  if ((err = run_gemm(a))) return rt_error(err);
  if (need_ab) {
    xkb_gemm_args b = a;
    std::swap(b.A, b.B);
    std::swap(b.lda, b.ldb);
    sc(alpha2, b.alpha);
    sc(one, b.beta);
    if ((err = run_gemm(b))) return rt_error(err);
  }
  mark_written(dC, 0, N, 0, N, uplo);
  return 0;
}

template <class T>
int sm_async(int herm, int side, int uplo, int M, int N, const T* alpha, const T* A, int LDA,
             const T* B, int LDB, const T* beta, T* C, int LDC) {
  if (side != CblasLeft && side != CblasRight) return -1;
  if (uplo != CblasUpper && uplo != CblasLower) return -2;
  const int Am = side == CblasLeft ? M : N;
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (LDA < std::max(1, Am)) return -7;
  if (LDB < std::max(1, M)) return -9;
  if (LDC < std::max(1, M)) return -12;
  if (M == 0 || N == 0 || (is_zero(*alpha) && is_one(*beta))) return 0;
  const OpName op_name(HT<T>::dt, herm ? "hemm" : "symm");
  xkb::EvCall ev_call(op_name.s, {U64(M), U64(N), U64(side), U64(uplo), 0, 0, 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  add_flops(op_name.s, (HT<T>::cplx ? 8.0 : 2.0) * (double)M * N * Am);
  const size_t NB = auto_tilesize(herm ? KERN_HEMM : KERN_SYMM, M, N, 0), es = sizeof(T);
  int err;
  Desc* dA = get_desc(A, Am, Am, LDA, es, NB, &err);
  if (!dA) return rt_error(err);
  if ((err = make_valid(dA, 0, Am, 0, Am))) return rt_error(err);
  Desc* dB = get_desc(B, M, N, LDB, es, NB, &err);
  if (!dB) return rt_error(err);
  if ((err = make_valid(dB, 0, M, 0, N))) return rt_error(err);
  Desc* dC = get_desc(C, M, N, LDC, es, NB, &err);
  if (!dC) return rt_error(err);
  if (!is_zero(*beta))
    if ((err = make_valid(dC, 0, M, 0, N))) return rt_error(err);
  double al[2], be[2];
  sc(*alpha, al);
  sc(*beta, be);
  if ((err = flush_pending())) return rt_error(err);
  const bool tc = thread_math() == XKBLAS_TENSOR_OP_MATH && (HT<T>::dt == XKB_D || HT<T>::dt == XKB_Z);
  if ((err = xkb_cuda_symm(HT<T>::dt, herm, side == CblasLeft ? 0 : 1,
                           uplo == CblasLower ? XKB_LOWER : XKB_UPPER, M, N, al,
                           dev_ptr(dA, 0, 0), (long)dA->dld, dev_ptr(dB, 0, 0), (long)dB->dld,
                           be, dev_ptr(dC, 0, 0), (long)dC->dld,
                           tc ? (int)std::max<long>(ozaki_min_dim(), 1) : 0, R.s_comp)))
    return rt_error(err);
  mark_full_overwrite(dC, 0, M, 0, N);
  return 0;
}

template <class T>
int tr_async(int is_trsm, int side, int uplo, int transA, int diag, int M, int N, const T* alpha,
             const T* A, int LDA, T* B, int LDB) {
  // reference blas/ztrsm.c:117-169, blas/ztrmm.c:109-170 (N = rows of B, NRHS = cols)
  const int NA = side == CblasLeft ? M : N;
  if (side != CblasLeft && side != CblasRight) return -1;
  if (uplo != CblasUpper && uplo != CblasLower) return -2;
  if (transA < CblasNoTrans || transA > CblasConjTrans) return -3;
  if (diag != CblasUnit && diag != CblasNonUnit) return -4;
  if (M < 0) return -5;
  if (N < 0) return -6;
  if (LDA < std::max(1, NA)) return -8;
  if (LDB < std::max(1, M)) return -10;
  if (std::min(M, N) == 0) return 0;
  const OpName op_name(HT<T>::dt, is_trsm ? "trsm" : "trmm");
  xkb::EvCall ev_call(op_name.s,
                      {U64(M), U64(N), U64(side), U64(uplo), U64(transA), U64(diag), 0});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  {
    const double f = side == CblasLeft ? (double)N * M * (M + 1) : (double)M * N * (N + 1);
    add_flops(op_name.s, (HT<T>::cplx ? 4.0 : 1.0) * f);
  }
  const size_t NB = auto_tilesize(is_trsm ? KERN_TRSM : KERN_TRMM, M, N, NA), es = sizeof(T);
  int err;
  Desc* dB = get_desc(B, M, N, LDB, es, NB, &err);
  if (!dB) return rt_error(err);
  const bool zero = is_zero(*alpha);
  Desc* dA = nullptr;
  if (!zero) {
    if (!(dA = get_desc(A, NA, NA, LDA, es, NB, &err))) return rt_error(err);
    if ((err = make_valid(dA, 0, NA, 0, NA, false))) return rt_error(err);
    if ((err = make_valid(dB, 0, M, 0, N, false))) return rt_error(err);
    if ((err = comp_wait_h2d())) return rt_error(err);
  }
  double al[2];
  sc(*alpha, al);
  const int sd = side == CblasLeft ? 0 : 1;
  const int ul = uplo == CblasLower ? XKB_LOWER : XKB_UPPER;
  const int dg = diag == CblasUnit ? 1 : 0;
  const bool tc = (thread_math() == XKBLAS_TENSOR_OP_MATH) && (HT<T>::dt == XKB_D || HT<T>::dt == XKB_Z);
  if (!zero && is_trsm && sd == 0 && R.batch_on && !tc &&
      (HT<T>::dt == XKB_D || HT<T>::dt == XKB_Z)) {
    // left solve queued for the tile-task executor
    xkb_batch_op o{};
    o.kind = XKB_BATCH_TRSM;
    o.dtype = HT<T>::dt;
    o.side = 0;
    o.uplo = ul;
    o.trans = opcode(transA);
    o.diag = dg;
    o.M = M;
    o.N = N;
    o.A = dev_ptr(dA, 0, 0);
    o.lda = (long)dA->dld;
    o.C = dev_ptr(dB, 0, 0);
    o.ldc = (long)dB->dld;
    o.alpha[0] = al[0];
    o.alpha[1] = al[1];
    // marked before queueing: a flush inside defer_op then leaves B's
    // completion event in place
    mark_full_overwrite(dB, 0, M, 0, N);
    if ((err = defer_op(o, dA, dB, nullptr, dB))) return rt_error(err);
    return 0;
  }
  if ((err = flush_pending())) return rt_error(err);
  if (zero) {
    const double z[2] = {0, 0};
    err = xkb_cuda_scale(HT<T>::dt, M, N, z, dev_ptr(dB, 0, 0), (long)dB->dld, XKB_FULL, 0, 0,
                         R.s_comp);
  } else if (is_trsm) {
    const int oz = tc ? (int)std::max<long>(ozaki_min_dim(), 1) : 0;
    err = xkb_cuda_trsm(HT<T>::dt, sd, ul, opcode(transA), dg, M, N, al, dev_ptr(dA, 0, 0),
                        (long)dA->dld, dev_ptr(dB, 0, 0), (long)dB->dld, oz, R.s_comp);
  } else {
    err = xkb_cuda_trmm(HT<T>::dt, sd, ul, opcode(transA), dg, M, N, al, dev_ptr(dA, 0, 0),
                        (long)dA->dld, dev_ptr(dB, 0, 0), (long)dB->dld,
                        tc ? (int)std::max<long>(ozaki_min_dim(), 1) : 0, R.s_comp);
  }
  if (err) return rt_error(err);
  mark_full_overwrite(dB, 0, M, 0, N);
  return 0;
}

// Cholesky factorization (reference blas/zpotrf.c:46-220; argument codes
// :55-67).  Runs after the queued calls, on the stored triangle only.
template <class T>
int potrf_async(int uplo, int N, T* A, int LDA) {
  if (uplo != CblasUpper && uplo != CblasLower) return -2;
  if (N < 0) return -5;
  if (LDA < std::max(1, N)) return -8;
  if (N == 0) return 0;
  const OpName op_name(HT<T>::dt, "potrf");
  xkb::EvCall ev_call(op_name.s, {U64(N), U64(uplo)});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  {
    const double n = N;
    add_flops(op_name.s, (HT<T>::cplx ? 4.0 : 1.0) * (n * n * n / 3.0 + n * n / 2.0 + n / 6.0));
  }
  int err;
  if ((err = flush_pending())) return rt_error(err);
  const size_t NB = auto_tilesize(KERN_GEMM, N, N, N), es = sizeof(T);
  Desc* dA = get_desc(A, N, N, LDA, es, NB, &err);
  if (!dA) return rt_error(err);
  if ((err = make_valid(dA, 0, N, 0, N))) return rt_error(err);
  if (!R.d_potrf_info) {
    if (cudaMalloc(&R.d_potrf_info, sizeof(int)) != cudaSuccess) {
      R.d_potrf_info = nullptr;
      return rt_error(XKB_ENOMEM);
    }
  }
  cudaMemsetAsync(R.d_potrf_info, 0, sizeof(int), R.s_comp);
  const bool tc = thread_math() == XKBLAS_TENSOR_OP_MATH && (HT<T>::dt == XKB_D || HT<T>::dt == XKB_Z);
  err = xkb_cuda_potrf(HT<T>::dt, uplo == CblasLower ? XKB_LOWER : XKB_UPPER, N,
                       dev_ptr(dA, 0, 0), (long)dA->dld, R.d_potrf_info,
                       tc ? (int)std::max<long>(ozaki_min_dim(), 1) : 0, R.s_comp);
  if (err) return rt_error(err);
  mark_written(dA, 0, N, 0, N, uplo);
  return 0;
}

// LU without pivoting of a square matrix (reference blas/zgetrf_nopiv.c:
// 48-101; the tile driver is built there but not declared in its headers).
template <class T>
int getrf_async(int M, int N, T* A, int LDA) {
  if (M < 0) return -1;
  if (N < 0 || N != M) return -2;
  if (LDA < std::max(1, M)) return -4;
  if (N == 0) return 0;
  const OpName op_name(HT<T>::dt, "getrf");
  xkb::EvCall ev_call(op_name.s, {U64(M), U64(N)});
  Guard g;
  if (int e = ensure_init()) return rt_error(e);
  Runtime& R = rt();
  count_call(op_name.s);
  {
    const double n = N;
    add_flops(op_name.s, (HT<T>::cplx ? 4.0 : 1.0) * (2.0 * n * n * n / 3.0 - n * n / 2.0 - n / 6.0));
  }
  int err;
  if ((err = flush_pending())) return rt_error(err);
  const size_t NB = auto_tilesize(KERN_GEMM, N, N, N), es = sizeof(T);
  Desc* dA = get_desc(A, N, N, LDA, es, NB, &err);
  if (!dA) return rt_error(err);
  if ((err = make_valid(dA, 0, N, 0, N))) return rt_error(err);
  if (!R.d_potrf_info) {
    if (cudaMalloc(&R.d_potrf_info, sizeof(int)) != cudaSuccess) {
      R.d_potrf_info = nullptr;
      return rt_error(XKB_ENOMEM);
    }
  }
  cudaMemsetAsync(R.d_potrf_info, 0, sizeof(int), R.s_comp);
  const bool tc = thread_math() == XKBLAS_TENSOR_OP_MATH && (HT<T>::dt == XKB_D || HT<T>::dt == XKB_Z);
  err = xkb_cuda_getrf_nopiv(HT<T>::dt, N, dev_ptr(dA, 0, 0), (long)dA->dld, R.d_potrf_info,
                             tc ? (int)std::max<long>(ozaki_min_dim(), 1) : 0, R.s_comp);
  if (err) return rt_error(err);
  mark_full_overwrite(dA, 0, N, 0, N);
  return 0;
}

}  // namespace

extern "C" int xkblas_sgetrf_nopiv_async(int M, int N, float* A, int LDA) {
  return getrf_async<float>(M, N, A, LDA);
}
extern "C" int xkblas_dgetrf_nopiv_async(int M, int N, double* A, int LDA) {
  return getrf_async<double>(M, N, A, LDA);
}
extern "C" int xkblas_cgetrf_nopiv_async(int M, int N, Complex32_t* A, int LDA) {
  return getrf_async<Complex32_t>(M, N, A, LDA);
}
extern "C" int xkblas_zgetrf_nopiv_async(int M, int N, Complex64_t* A, int LDA) {
  return getrf_async<Complex64_t>(M, N, A, LDA);
}

extern "C" int xkblas_spotrf_async(int uplo, int N, float* A, int LDA) {
  return potrf_async<float>(uplo, N, A, LDA);
}
extern "C" int xkblas_dpotrf_async(int uplo, int N, double* A, int LDA) {
  return potrf_async<double>(uplo, N, A, LDA);
}
extern "C" int xkblas_cpotrf_async(int uplo, int N, Complex32_t* A, int LDA) {
  return potrf_async<Complex32_t>(uplo, N, A, LDA);
}
extern "C" int xkblas_zpotrf_async(int uplo, int N, Complex64_t* A, int LDA) {
  return potrf_async<Complex64_t>(uplo, N, A, LDA);
}
// the factorization calls share one device info word
extern "C" int xkblas_getrf_info(void) { return xkblas_potrf_info(); }

extern "C" int xkblas_potrf_info(void) {
  Runtime& R = rt();
  std::lock_guard<std::recursive_mutex> g(R.mu);
  if (!R.ready || !R.d_potrf_info) return 0;
  int v = 0;
  cudaStreamSynchronize(R.s_comp);
  if (cudaMemcpy(&v, R.d_potrf_info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  return v;
}

// ============================================================================
// exported symbols
// ============================================================================
#define XKB_DEFINE_OPS(p, T, R)                                                                \
  extern "C" int xkblas_##p##gemm_async(int tA, int tB, int M, int N, int K, const T* al,      \
                                        const T* A, int lda, const T* B, int ldb, const T* be, \
                                        T* C, int ldc) {                                       \
    return gemm_async<T>(tA, tB, M, N, K, al, A, lda, B, ldb, be, C, ldc);                     \
  }                                                                                            \
  extern "C" int xkblas_##p##gemmt_async(int ul, int tA, int tB, int N, int K, const T* al,    \
                                         const T* A, int lda, const T* B, int ldb,             \
                                         const T* be, T* C, int ldc) {                         \
    return gemmt_async<T>(ul, tA, tB, N, K, al, A, lda, B, ldb, be, C, ldc);                   \
  }                                                                                            \
  extern "C" int xkblas_##p##trsm_async(int sd, int ul, int tA, int dg, int M, int N,          \
                                        const T* al, const T* A, int lda, T* B, int ldb) {     \
    return tr_async<T>(1, sd, ul, tA, dg, M, N, al, A, lda, B, ldb);                           \
  }                                                                                            \
  extern "C" int xkblas_##p##trmm_async(int sd, int ul, int tA, int dg, int M, int N,          \
                                        const T* al, const T* A, int lda, T* B, int ldb) {     \
    return tr_async<T>(0, sd, ul, tA, dg, M, N, al, A, lda, B, ldb);                           \
  }                                                                                            \
  extern "C" int xkblas_##p##symm_async(int sd, int ul, int M, int N, const T* al, const T* A, \
                                        int lda, const T* B, int ldb, const T* be, T* C,       \
                                        int ldc) {                                             \
    return sm_async<T>(0, sd, ul, M, N, al, A, lda, B, ldb, be, C, ldc);                       \
  }                                                                                            \
  extern "C" int xkblas_##p##syrk_async(int ul, int tr, int N, int K, const T* al, const T* A, \
                                        int lda, const T* be, T* C, int ldc) {                 \
    return rk_async<T>(0, ul, tr, N, K, *al, A, lda, *be, C, ldc);                             \
  }                                                                                            \
  extern "C" int xkblas_##p##syr2k_async(int ul, int tr, int N, int K, const T* al,            \
                                         const T* A, int lda, const T* B, int ldb,             \
                                         const T* be, T* C, int ldc) {                         \
    return r2k_async<T>(0, ul, tr, N, K, *al, A, lda, B, ldb, *be, C, ldc);                    \
  }

#define XKB_DEFINE_HE_OPS(p, T, R)                                                             \
  extern "C" int xkblas_##p##hemm_async(int sd, int ul, int M, int N, const T* al, const T* A, \
                                        int lda, const T* B, int ldb, const T* be, T* C,       \
                                        int ldc) {                                             \
    return sm_async<T>(1, sd, ul, M, N, al, A, lda, B, ldb, be, C, ldc);                       \
  }                                                                                            \
  extern "C" int xkblas_##p##herk_async(int ul, int tr, int N, int K, const R* al, const T* A, \
                                        int lda, const R* be, T* C, int ldc) {                 \
    return rk_async<T>(1, ul, tr, N, K, T(*al), A, lda, T(*be), C, ldc);                       \
  }                                                                                            \
  extern "C" int xkblas_##p##her2k_async(int ul, int tr, int N, int K, const T* al,            \
                                         const T* A, int lda, const T* B, int ldb,             \
                                         const R* be, T* C, int ldc) {                         \
    return r2k_async<T>(1, ul, tr, N, K, *al, A, lda, B, ldb, T(*be), C, ldc);                 \
  }

XKB_DEFINE_OPS(s, float, float)
XKB_DEFINE_OPS(d, double, double)
XKB_DEFINE_OPS(c, Complex32_t, float)
XKB_DEFINE_OPS(z, Complex64_t, double)
XKB_DEFINE_HE_OPS(c, Complex32_t, float)
XKB_DEFINE_HE_OPS(z, Complex64_t, double)
