"""Failure detection without a GPU fault: every device wait of the library
is bounded; when one gives up, the kernel records an error word and ends,
xkblas_sync reports it with a code of its own, and the context stays usable
for the next call.  The wait is made to run out by a task dependency that
nothing ever resolves (xkb_cuda_sched_wait_test), with a 20 ms limit.
Requires a B200."""
import time

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

XKB_ETIMEDOUT = -5
XKB_DEV_FULL_WAIT = 1


def test_bounded_wait_expires_and_context_survives(xk):
    lib = xk.lib()
    xk.sync()  # nothing pending, no stale error word
    assert lib.xkb_cuda_take_device_error() == 0
    t0 = time.perf_counter()
    assert lib.xkb_cuda_sched_wait_test(20, None) == 0
    r = lib.xkblas_sync()
    dt = time.perf_counter() - t0
    assert r == XKB_ETIMEDOUT, r
    assert lib.xkblas_last_device_error() == XKB_DEV_FULL_WAIT
    assert lib.xkblas_last_device_error() == 0  # read and cleared
    assert dt < 5.0  # the 20 ms limit, not the default 4 s one
    # the next call works and is right
    M, N, K = 130, 70, 90
    A, B, C0 = O.plrnt(M, K, 1), O.plrnt(K, N, 2), O.plrnt(M, N, 3)
    C = C0.copy(order="F")
    xk.gemm(xk.CblasNoTrans, xk.CblasNoTrans, 1.5, A, B, -0.5, C)
    xk.invalidate_caches()
    R = O.gemm(O.NOTRANS, O.NOTRANS, 1.5, A, B, -0.5, C0.copy(order="F"))
    assert checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, K) <= 3.0
    assert lib.xkb_cuda_take_device_error() == 0


def test_wait_limit_is_a_launch_parameter(xk):
    """The executor's limit comes from the tuning key sched_wait_ms at
    launch; a batch under a short limit still completes normally."""
    import ctypes
    import torch
    lib = xk.lib()
    lib.xkb_tune_set(b"sched_wait_ms", 50.0)
    try:
        M, N = 300, 200
        L = np.asfortranarray(np.tril(O.plrnt(M, M, 4)) + M * np.eye(M))
        B0 = O.plrnt(M, N, 5)
        dL = torch.from_numpy(np.ascontiguousarray(L.T)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B0.T)).cuda()
        o = xk.BatchOp()
        o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, 1, 0, 0, M, N
        o.A, o.lda, o.C, o.ldc = dL.data_ptr(), M, dB.data_ptr(), M
        o.alpha[0] = 1.0
        torch.cuda.synchronize()
        assert lib.xkb_cuda_batch(ctypes.byref(o), 1, 0, None) == 0
        xk.sync()
        assert lib.xkb_cuda_take_device_error() == 0
        X_ = np.asfortranarray(dB.cpu().numpy().T)
        R = O.trsm(O.LEFT, O.LOWER, O.NOTRANS, O.NONUNIT, 1.0, L, B0.copy(order="F"), nb=64)
        assert checks.trsm_ratio(X_, R, L, M, N) <= 10
    finally:
        lib.xkb_tune_set(b"sched_wait_ms", 4000.0)


def test_wait_test_rejects_bad_limits(xk):
    lib = xk.lib()
    assert lib.xkb_cuda_sched_wait_test(0, None) == -1
    assert lib.xkb_cuda_sched_wait_test(20000, None) == -1
