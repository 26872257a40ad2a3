"""Per-thread API semantics (reference: one context per pthread,
blas/xkblas.c:224-243): the math mode set by one thread does not change
another thread's arithmetic, each thread has its own context handle, and
threads issuing calls and xkblas_sync concurrently on their own matrices get
correct results.  Requires a B200."""
import threading

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_ = 111


def _gemm_case(xk, seed, n=256):
    A, B, C0 = O.plrnt(n, n, seed), O.plrnt(n, n, seed + 1), O.plrnt(n, n, seed + 2)
    C = C0.copy(order="F")
    xk.gemm(N_, N_, 1.5, A, B, -0.5, C)
    R = O.gemm(N_, N_, 1.5, A, B, -0.5, C0.copy(order="F"))
    return checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, n)


def test_math_mode_is_per_thread(xk):
    lib = xk.lib()
    main_mode = lib.xkblas_get_modemath()
    a_set, b_done = threading.Event(), threading.Event()
    out, errs = {}, []

    def thread_a():
        try:
            xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
            out["ctx_a"] = lib.xkblas_context_get()
            a_set.set()
            assert b_done.wait(120)
            c0 = xk.ozaki_counts()[0]
            out["ratio_a"] = _gemm_case(xk, 10)
            out["oz_a"] = xk.ozaki_counts()[0] - c0
            out["mode_a"] = lib.xkblas_get_modemath()
        except Exception as e:  # reported by the main thread
            errs.append(e)
            a_set.set()

    def thread_b():
        try:
            assert a_set.wait(120)
            out["ctx_b"] = lib.xkblas_context_get()
            c0 = xk.ozaki_counts()[0]
            out["ratio_b"] = _gemm_case(xk, 20)
            out["oz_b"] = xk.ozaki_counts()[0] - c0
            out["mode_b"] = lib.xkblas_get_modemath()
        except Exception as e:
            errs.append(e)
        finally:
            b_done.set()

    ta, tb = threading.Thread(target=thread_a), threading.Thread(target=thread_b)
    ta.start()
    tb.start()
    ta.join(300)
    tb.join(300)
    xk.invalidate_caches()
    assert not errs, errs
    assert out["mode_a"] == xk.XKBLAS_TENSOR_OP_MATH and out["oz_a"] >= 1
    assert out["mode_b"] == xk.XKBLAS_DEFAULT_MATH and out["oz_b"] == 0
    assert out["ratio_a"] <= 3.0 and out["ratio_b"] <= 3.0
    assert out["ctx_a"] != out["ctx_b"] and out["ctx_a"] and out["ctx_b"]
    assert lib.xkblas_get_modemath() == main_mode  # the main thread is untouched


def test_concurrent_threads_sync_their_own_work(xk):
    """Four threads, each issuing DGEMM / DTRSM chains on its own matrices
    and calling xkblas_sync, interleaved; every result meets the reference
    bounds."""
    errs, ratios = [], []
    lock = threading.Lock()

    def worker(k):
        try:
            for it in range(4):
                r1 = _gemm_case(xk, 100 + 10 * k + it, n=192 + 16 * k)
                M = 160 + 8 * k
                A = np.asfortranarray(np.tril(O.plrnt(M, M, 300 + k)) + M * np.eye(M))
                B0 = O.plrnt(M, 96, 400 + k)
                B = B0.copy(order="F")
                xk.trsm(141, 122, N_, 131, 2.0, A, B)
                R = O.trsm(O.LEFT, O.LOWER, O.NOTRANS, O.NONUNIT, 2.0, A, B0.copy(order="F"),
                           nb=64)
                r2 = checks.trsm_ratio(B, R, A, M, 96)
                with lock:
                    ratios.append((r1, r2))
        except Exception as e:
            errs.append(e)

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(600)
    xk.invalidate_caches()
    assert not errs, errs
    assert len(ratios) == 16
    assert all(r1 <= 3.0 and r2 <= 10 for r1, r2 in ratios), ratios
