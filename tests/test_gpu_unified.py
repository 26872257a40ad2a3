"""Unified-memory mode (reference blas/xkblas.c:155-220, 1959): with
xkblas_force_set_unified, xkblas_malloc_unified returns CUDA managed memory;
matrices in managed memory are used in place by the kernels (no tile copies
in either direction) and coherence only orders the work.  Checked through
the public async API against numpy FP64 and the oracle.  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_ = 111
LEFT, LO, NONUNIT = 141, 122, 131


def _managed(xk, rows, cols):
    lib = xk.lib()
    p = ctypes.c_void_p()
    assert lib.xkblas_malloc_unified(ctypes.byref(p), ctypes.c_size_t(8 * rows * cols)) == 0
    buf = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), shape=(rows * cols,))
    return p, buf.reshape((rows, cols), order="F")


def test_unified_gemm_trsm_in_place(xk):
    lib = xk.lib()
    if lib.xkblas_force_set_unified() != 0:
        pytest.skip("device without managed memory")
    n = 700
    pa, A = _managed(xk, n, n)
    pb, B = _managed(xk, n, n)
    pc, C = _managed(xk, n, n)
    pl, L = _managed(xk, n, n)
    A[:] = O.plrnt(n, n, 3)
    B[:] = O.plrnt(n, n, 4)
    C0 = O.plrnt(n, n, 5)
    C[:] = C0
    L[:] = np.tril(O.plrnt(n, n, 6)) / n + np.eye(n)
    X0 = B.copy()
    xk.reset_stats()
    al = np.array([1.5]); be = np.array([-0.5]); one = np.array([1.0])
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    assert lib.xkblas_dgemm_async(N_, N_, n, n, n, p(al), pa, n, pb, n, p(be), pc, n) == 0
    assert lib.xkblas_dtrsm_async(LEFT, LO, N_, NONUNIT, n, n, p(one), pl, n, pb, n) == 0
    for ptr in (pc, pb):
        assert lib.xkblas_memory_coherent_async(0, 0, ctypes.c_size_t(n), ctypes.c_size_t(n), ptr,
                                                ctypes.c_size_t(n), ctypes.c_size_t(8)) == 0
    assert lib.xkblas_sync() == 0
    st = xk.stats()
    assert st["h2d_bytes"] == 0 and st["d2h_bytes"] == 0, st  # used in place
    R = 1.5 * (A @ X0) - 0.5 * C0
    assert checks.gemm_ratio(C, R, A, X0, C0, 1.5, -0.5, n) <= 3.0
    Xref = np.linalg.solve(L, X0)
    assert np.abs(B - Xref).max() <= 1e-12 * np.abs(Xref).max()
    xk.invalidate_caches()
    for ptr in (pa, pb, pc, pl):
        assert lib.xkblas_free_unified(ptr) == 0
