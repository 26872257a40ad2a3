"""The row-block / column-panel Ozaki path of xkblas_dgemm_async (real,
op(B) = B, beta = 0, M and N >= 4096 under XKBLAS_TENSOR_OP_MATH): op(A)
crosses the host link in row blocks and B in column panels, interleaved, and
each finished rectangle of C is copied back on its own event.  Checked with
the reference's GEMM acceptance bound (tests/checks.py) against numpy's FP64
product (its own error is far inside the bound at these sizes), bit for bit
against the column-panel path (tuning key ozaki_row_blocks = 0), and with a
descriptor larger than the call, results read on the device by a later call
before coherence.  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_, T_ = 111, 112


@pytest.fixture
def tc(xk):
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    yield xk
    xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)
    xk.lib().xkb_tune_set(b"ozaki_row_blocks", 1.0)


def _dgemm(xk, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al = np.array([alpha])
    be = np.array([beta])
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    r = xk.lib().xkblas_dgemm_async(ta, tb, M, N, K, p(al), p(A), lda, p(B), ldb, p(be), p(C), ldc)
    assert r == 0
    return al, be


@pytest.mark.parametrize("ta", [N_, T_])
def test_blocks_ragged_and_equal_to_panels(tc, ta):
    M, N, K = 4400, 4500, 2049  # ragged last row block and column panel
    A = O.plrnt(M, K, 41) if ta == N_ else O.plrnt(K, M, 41)
    B = O.plrnt(K, N, 42)
    C = np.zeros((M, N), order="F")
    with tc.contraction_trace() as tr:
        tc.gemm(ta, N_, 1.25, A, B, 0.0, C)
    assert "ozaki_blocks" in tr.ops(), tr.ops()
    tc.invalidate_caches()
    R = 1.25 * ((A if ta == N_ else A.T) @ B)
    Z = np.zeros((M, N))
    assert checks.gemm_ratio(C, R, A, B, Z, 1.25, 0.0, K) <= 3.0
    tc.lib().xkb_tune_set(b"ozaki_row_blocks", 0.0)  # the column-panel form
    C2 = np.zeros((M, N), order="F")
    tc.gemm(ta, N_, 1.25, A, B, 0.0, C2)
    tc.invalidate_caches()
    assert np.array_equal(C, C2)
    assert tc.lib().xkb_cuda_take_device_error() == 0


def test_blocks_chain_before_coherence(tc):
    """C1 = A B (blocks), then C2 = C1 B2 reads C1 on the device before any
    coherence; both come back right."""
    M, N, K = 4096, 4096, 1024
    A = O.plrnt(M, K, 51)
    B = O.plrnt(K, N, 52)
    B2 = O.plrnt(N, N, 53)
    C1 = np.zeros((M, N), order="F")
    C2 = np.zeros((M, N), order="F")
    keep = [_dgemm(tc, N_, N_, M, N, K, 1.0, A, M, B, K, 0.0, C1, M)]
    keep.append(_dgemm(tc, N_, N_, M, N, N, 1.0, C1, M, B2, N, 0.0, C2, M))
    tc.coherent(C2)
    tc.coherent(C1)
    tc.sync()
    tc.invalidate_caches()
    Z = np.zeros((M, N))
    assert checks.gemm_ratio(C1, A @ B, A, B, Z, 1.0, 0.0, K) <= 3.0
    assert checks.gemm_ratio(C2, C1 @ B2, C1, B2, Z, 1.0, 0.0, N) <= 3.0


def test_blocks_on_larger_descriptor(tc):
    """A full write of the big C, then a blocked call on its leading
    sub-block (same host pointer and ld: the descriptor is reused), both
    before coherence: the sub-block comes back rectangle by rectangle, the
    rest of C (written by the first call) after all queued work."""
    M, N, K = 4608, 5120, 1024
    m, n = 4200, 4300
    A = O.plrnt(M, K, 61)
    A2 = O.plrnt(M, K, 62)
    B = O.plrnt(K, N, 63)
    C = np.zeros((M, N), order="F")
    keep = [_dgemm(tc, N_, N_, M, N, K, 1.0, A, M, B, K, 0.0, C, M)]
    keep.append(_dgemm(tc, N_, N_, m, n, K, 2.0, A2, M, B, K, 0.0, C, M))
    tc.coherent(C)
    tc.sync()
    tc.invalidate_caches()
    P = A @ B
    Z = np.zeros((M, N))
    assert checks.gemm_ratio(C[m:, :], P[m:, :], A[m:], B, Z[m:], 1.0, 0.0, K) <= 3.0
    assert checks.gemm_ratio(C[:, n:], P[:, n:], A, B[:, n:], Z[:, n:], 1.0, 0.0, K) <= 3.0
    P2 = 2.0 * (A2[:m] @ B[:, :n])
    assert checks.gemm_ratio(C[:m, :n], P2, A2[:m], B[:, :n], Z[:m, :n], 2.0, 0.0, K) <= 3.0
    assert tc.lib().xkb_cuda_take_device_error() == 0
