"""Per-thread API semantics (reference: one context per pthread,
blas/xkblas.c:224-243): the math mode set by one thread does not change
another thread's arithmetic, each thread has its own context handle, and
threads issuing calls and xkblas_sync concurrently on their own matrices get
correct results.

The worker threads make library calls only.  Inputs are made, and kept
alive until the end, by the main thread (the library caches device copies
by host address, so a freed array's address must not come back as another
matrix), and every oracle check runs in the main thread afterwards.
Requires a B200."""
import threading

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_ = 111


def _gemm_inputs(seed, n=256):
    A, B, C0 = O.plrnt(n, n, seed), O.plrnt(n, n, seed + 1), O.plrnt(n, n, seed + 2)
    return A, B, C0, C0.copy(order="F")


def _gemm_ratio(A, B, C0, C):
    R = O.gemm(N_, N_, 1.5, A, B, -0.5, C0.copy(order="F"))
    return checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, A.shape[1])


def _run_threads(fns):
    errs = []

    def wrap(f):
        def run():
            try:
                f()
            except Exception as e:  # reported by the main thread
                errs.append(e)
        return run

    ts = [threading.Thread(target=wrap(f)) for f in fns]
    for t in ts:
        t.start()
    for t in ts:
        t.join(600)
    assert not any(t.is_alive() for t in ts)
    return errs


def test_math_mode_is_per_thread(xk):
    lib = xk.lib()
    main_mode = lib.xkblas_get_modemath()
    a_set, b_done = threading.Event(), threading.Event()
    ia, ib = _gemm_inputs(10), _gemm_inputs(20)
    out = {}

    def thread_a():
        xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
        out["ctx_a"] = lib.xkblas_context_get()
        a_set.set()
        assert b_done.wait(120)
        c0 = xk.ozaki_counts()[0]
        xk.gemm(N_, N_, 1.5, ia[0], ia[1], -0.5, ia[3])
        out["oz_a"] = xk.ozaki_counts()[0] - c0
        out["mode_a"] = lib.xkblas_get_modemath()

    def thread_b():
        try:
            assert a_set.wait(120)
            out["ctx_b"] = lib.xkblas_context_get()
            c0 = xk.ozaki_counts()[0]
            xk.gemm(N_, N_, 1.5, ib[0], ib[1], -0.5, ib[3])
            out["oz_b"] = xk.ozaki_counts()[0] - c0
            out["mode_b"] = lib.xkblas_get_modemath()
        finally:
            b_done.set()

    errs = _run_threads([thread_a, thread_b])
    xk.invalidate_caches()
    assert not errs, errs
    assert out["mode_a"] == xk.XKBLAS_TENSOR_OP_MATH and out["oz_a"] >= 1
    assert out["mode_b"] == xk.XKBLAS_DEFAULT_MATH and out["oz_b"] == 0
    assert _gemm_ratio(*ia) <= 3.0 and _gemm_ratio(*ib) <= 3.0
    assert out["ctx_a"] != out["ctx_b"] and out["ctx_a"] and out["ctx_b"]
    assert lib.xkblas_get_modemath() == main_mode  # the main thread is untouched


def test_concurrent_threads_sync_their_own_work(xk):
    """Four threads, each issuing DGEMM and DTRSM calls on its own matrices,
    each call followed by its coherence request and xkblas_sync, interleaved
    with the other threads'; every result meets the reference bounds."""
    nthreads, iters = 4, 4
    work = []
    for k in range(nthreads):
        items = []
        for it in range(iters):
            g = _gemm_inputs(100 + 10 * k + it, n=192 + 16 * k)
            M = 160 + 8 * k
            A = np.asfortranarray(np.tril(O.plrnt(M, M, 300 + 10 * k + it)) + M * np.eye(M))
            B0 = O.plrnt(M, 96, 400 + 10 * k + it)
            items.append((g, A, B0, B0.copy(order="F")))
        work.append(items)

    def worker(items):
        def run():
            for g, A, B0, B in items:
                xk.gemm(N_, N_, 1.5, g[0], g[1], -0.5, g[3])
                xk.trsm(141, 122, N_, 131, 2.0, A, B)
        return run

    errs = _run_threads([worker(items) for items in work])
    xk.invalidate_caches()
    assert not errs, errs
    for items in work:
        for g, A, B0, B in items:
            assert _gemm_ratio(*g) <= 3.0
            R = O.trsm(O.LEFT, O.LOWER, O.NOTRANS, O.NONUNIT, 2.0, A, B0.copy(order="F"), nb=64)
            assert checks.trsm_ratio(B, R, A, A.shape[0], B.shape[1]) <= 10


def test_concurrent_device_abi_factorizations(xk):
    """Three threads, each on its own CUDA stream, call xkb_cuda_potrf (the
    blocked form: side streams ordered by events) and xkb_cuda_trsm (two
    groups of right-hand sides on side streams) at the same time, several
    times over; every result is right.  The side streams are shared by the
    threads, the events that order them are each thread's own."""
    import ctypes
    import torch
    lib = xk.lib()
    n, nrhs = 1100, 2304
    work = []
    for k in range(3):
        g = torch.Generator(device="cuda").manual_seed(500 + k)
        Bm = torch.rand(n, n, generator=g, device="cuda", dtype=torch.float64) - 0.5
        A0 = Bm @ Bm.t() / n + torch.eye(n, device="cuda", dtype=torch.float64)
        T = torch.tril(torch.rand(n, n, generator=g, device="cuda", dtype=torch.float64) - 0.5)
        T += n * torch.eye(n, device="cuda", dtype=torch.float64)
        Tcm = T.t().contiguous()  # column-major lower
        R0 = torch.rand(nrhs, n, generator=g, device="cuda", dtype=torch.float64) - 0.5
        work.append({"A0": A0, "A": A0.clone(), "Tcm": Tcm, "T": T, "R0": R0, "R": R0.clone(),
                     "info": torch.zeros(1, dtype=torch.int32, device="cuda"),
                     "st": torch.cuda.Stream()})
    torch.cuda.synchronize()
    al = (ctypes.c_double * 2)(1.0, 0.0)
    alp = ctypes.cast(al, ctypes.POINTER(ctypes.c_double))

    def worker(w):
        def run():
            sp = ctypes.c_void_p(w["st"].cuda_stream)
            with torch.cuda.stream(w["st"]):
                for _ in range(4):
                    w["A"].copy_(w["A0"])
                    w["R"].copy_(w["R0"])
                    assert lib.xkb_cuda_potrf(1, 1, n, ctypes.c_void_p(w["A"].data_ptr()), n,
                                              ctypes.c_void_p(w["info"].data_ptr()), 0, sp) == 0
                    assert lib.xkb_cuda_trsm(1, 0, 1, 0, 0, n, nrhs, alp, w["Tcm"].data_ptr(), n,
                                             w["R"].data_ptr(), n, 0, sp) == 0
            w["st"].synchronize()
        return run

    errs = _run_threads([worker(w) for w in work])
    assert not errs, errs
    torch.cuda.synchronize()
    assert lib.xkb_cuda_take_device_error() == 0
    for w in work:
        L = torch.triu(w["A"])  # column-major lower factor = row-major upper
        r = (L.t() @ L - w["A0"]).abs().max().item() / w["A0"].abs().max().item()
        assert r <= 16 * n * 2.0 ** -53, r
        assert int(w["info"].item()) == 0
        X = w["R"].t()  # column-major n x nrhs solution of T X = R0^T
        res = (w["T"] @ X - w["R0"].t()).abs().max().item()
        assert res <= 16 * n * 2.0 ** -53 * (n + 0.5) * max(1.0, X.abs().max().item()), res
