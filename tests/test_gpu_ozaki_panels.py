"""The column-panel Ozaki path of xkblas_dgemm_async (real, op(B) = B,
N >= 4096 under XKBLAS_TENSOR_OP_MATH): B and C cross the host link panel by
panel and each finished panel of C is copied back on its own event.  Checked
with the reference's GEMM acceptance bound (tests/checks.py), including
descriptors larger than the call and results read on the device by a later
call before coherence.  At these sizes (N >= 4096) the reference product is
numpy's FP64 matmul, whose own error is far inside the bound; the oracle
covers the same contraction at small sizes in test_gpu_ozaki.py.  Requires a
B200."""
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


def _dgemm(xk, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    """xkblas_dgemm_async on (possibly sub-block) numpy views: pointers taken
    from the views, leading dimensions given."""
    al = np.array([alpha])
    be = np.array([beta])
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    r = xk.lib().xkblas_dgemm_async(ta, tb, M, N, K, p(al), p(A), lda, p(B), ldb, p(be), p(C), ldc)
    assert r == 0
    return al, be


@pytest.mark.parametrize("ta,beta", [(N_, -0.5), (T_, 0.0), (N_, 0.0)])
def test_panels_ragged(tc, ta, beta):
    M, N, K = 2100, 4500, 2049  # N not a multiple of the 256-column panel granule
    A = O.plrnt(M, K, 11) if ta == N_ else O.plrnt(K, M, 11)
    B = O.plrnt(K, N, 12)
    C0 = O.plrnt(M, N, 13)
    C = C0.copy(order="F")
    s0 = tc.stats()["ozaki_calls"]
    tc.gemm(ta, N_, 1.25, A, B, beta, C)
    assert tc.stats()["ozaki_calls"] == s0 + 1
    tc.invalidate_caches()
    R = 1.25 * ((A if ta == N_ else A.T) @ B) + beta * C0
    assert checks.gemm_ratio(C, R, A, B, C0, 1.25, beta, K) <= 3.0
    assert tc.lib().xkb_cuda_take_device_error() == 0


def test_panels_chain_before_coherence(tc):
    """C1 = A B (panels), then C2 = C1 B2 reads C1 on the device before any
    coherence; both come back right."""
    M, N, K = 2048, 4096, 2048
    A = O.plrnt(M, K, 21)
    B = O.plrnt(K, N, 22)
    B2 = O.plrnt(N, N, 23)
    C1 = np.zeros((M, N), order="F")
    C2 = np.zeros((M, N), order="F")
    keep = [_dgemm(tc, N_, N_, M, N, K, 1.0, A, M, B, K, 0.0, C1, M)]
    keep.append(_dgemm(tc, N_, N_, M, N, N, 1.0, C1, M, B2, N, 0.0, C2, M))
    tc.coherent(C2)
    tc.coherent(C1)
    tc.sync()
    tc.invalidate_caches()
    R1 = A @ B
    assert checks.gemm_ratio(C1, R1, A, B, np.zeros((M, N)), 1.0, 0.0, K) <= 3.0
    # second product against the device's C1 as it came back
    R2 = C1 @ B2
    assert checks.gemm_ratio(C2, R2, C1, B2, np.zeros((M, N)), 1.0, 0.0, N) <= 3.0


def test_panels_on_larger_descriptor(tc):
    """A full-width write of the big C, then a panel call on its leading
    sub-block (same host pointer and ld: the descriptor is reused): the
    columns past the sub-block still come back, and untouched rows keep the
    first result."""
    M, N, K = 2304, 5120, 2048
    m, n = 2100, 4300
    A = O.plrnt(M, K, 31)
    B = O.plrnt(K, N, 32)
    C = np.zeros((M, N), order="F")
    keep = [_dgemm(tc, N_, N_, M, N, K, 1.0, A, M, B, K, 0.0, C, M)]
    # second call: C[:m, :n] = 2 A[:m] B[:, :n] - C[:m, :n]
    keep.append(_dgemm(tc, N_, N_, m, n, K, 2.0, A, M, B, K, -1.0, C, M))
    tc.coherent(C)
    tc.sync()
    tc.invalidate_caches()
    P = A @ B
    Z = np.zeros((M, N))
    assert checks.gemm_ratio(C[m:, :], P[m:, :], A[m:], B, Z[m:], 1.0, 0.0, K) <= 3.0
    assert checks.gemm_ratio(C[:, n:], P[:, n:], A, B[:, n:], Z[:, n:], 1.0, 0.0, K) <= 3.0
    # leading block: 2P - P = P, within the bound of a second product on top
    assert checks.gemm_ratio(C[:m, :n], P[:m, :n], A[:m], B[:, :n], P[:m, :n], 2.0, -1.0, K) <= 3.0
    assert tc.lib().xkb_cuda_take_device_error() == 0
