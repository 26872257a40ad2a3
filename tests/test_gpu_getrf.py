"""LU factorization without pivoting through the public API
(xkblas_?getrf_nopiv_async + memory_coherent_async + sync; reference tile
driver blas/zgetrf_nopiv.c:48-101): the factors match the oracle's
restatement of the tile algorithm on the same diagonally dominant matrix,
reproduce A (backward error bound), and the first zero pivot is reported.
Requires a B200."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

EPS = {np.float64: 2.0 ** -53, np.complex128: 2.0 ** -53,
       np.float32: 2.0 ** -24, np.complex64: 2.0 ** -24}


def _dd(n, dt, seed):
    cplx = np.issubdtype(dt, np.complexfloating)
    A = O.plrnt(n, n, seed, cplx) + n * np.eye(n)  # diagonally dominant
    return np.asfortranarray(A.astype(dt))


def _getrf(xk, A):
    p = {np.dtype(np.float32): "s", np.dtype(np.float64): "d",
         np.dtype(np.complex64): "c", np.dtype(np.complex128): "z"}[A.dtype]
    lib = xk.lib()
    n = A.shape[0]
    r = getattr(lib, "xkblas_%sgetrf_nopiv_async" % p)(n, n, xk._ptr(A), n)
    assert r == 0
    xk.coherent(A)
    xk.sync()
    info = lib.xkblas_getrf_info()
    xk.invalidate_caches()
    return info


@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32, np.complex64])
@pytest.mark.parametrize("n", [1, 7, 64, 65, 127, 128, 129, 200, 700])
def test_getrf_nopiv_factor(xk, dt, n):
    A0 = _dd(n, dt, 31)
    A = A0.copy(order="F")
    assert _getrf(xk, A) == 0
    up = np.complex128 if np.iscomplexobj(A0) else np.float64
    ref = np.asfortranarray(A0.astype(up))
    assert O.getrf_nopiv(ref, nb=64) == 0
    L = np.tril(A, -1).astype(up) + np.eye(n)
    U = np.triu(A).astype(up)
    scale = np.abs(A0).max() * n * EPS[dt]
    assert np.abs(L @ U - A0.astype(up)).max() <= 16 * scale
    assert np.abs(A.astype(up) - ref).max() <= 64 * n * EPS[dt] * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("mode", [1, 3])
def test_getrf_nopiv_tensor_op_mode(xk, mode, dt):
    """Tensor-op mode: couplings with all dimensions >= 2048 run in the Ozaki
    form, in the recursive form (tuning key getrf_blocked = 1) and in the
    hybrid (= 3: the top coupling in the Ozaki form, the halves blocked);
    same backward-error bound."""
    n = 4200
    A0 = _dd(n, dt, 37)
    A = A0.copy(order="F")
    lib = xk.lib()
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    lib.xkb_tune_set(b"getrf_blocked", float(mode))
    try:
        c0 = xk.ozaki_counts()[0]
        assert _getrf(xk, A) == 0
        assert xk.ozaki_counts()[0] > c0
    finally:
        xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)
        lib.xkb_tune_set(b"getrf_blocked", 3.0)
    L = np.tril(A, -1) + np.eye(n)
    U = np.triu(A)
    assert np.abs(L @ U - A0).max() <= 16 * np.abs(A0).max() * n * EPS[np.float64]


@pytest.mark.parametrize("col", [1, 5, 70, 200])
def test_getrf_nopiv_reports_zero_pivot(xk, col):
    n = 300
    A = np.asfortranarray(np.eye(n) * 2.0)
    A[col - 1, col - 1] = 0.0  # an exact zero pivot at column col
    assert _getrf(xk, A) == col


def test_getrf_nopiv_argument_codes(xk):
    lib = xk.lib()
    A = np.zeros((4, 4), order="F")
    assert lib.xkblas_dgetrf_nopiv_async(-1, 4, xk._ptr(A), 4) == -1
    assert lib.xkblas_dgetrf_nopiv_async(4, 3, xk._ptr(A), 4) == -2
    assert lib.xkblas_dgetrf_nopiv_async(4, 4, xk._ptr(A), 3) == -4
    assert lib.xkblas_dgetrf_nopiv_async(0, 0, xk._ptr(A), 1) == 0  # empty: nothing to do


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_getrf_nopiv_blocked_and_recursive_forms(xk, dt):
    """The blocked look-ahead form (tuning key getrf_blocked = 1, several
    block widths, widths shrinking along the factorization, a ragged last
    block), the recursive form (= 0) and the hybrid (= 3 with getrf_oz_leaf
    = 512: the recursion's top coupling, blocked halves) meet the same
    backward-error bound, and all report a zero pivot in a late block."""
    lib = xk.lib()
    n = 1100
    up = np.complex128 if np.issubdtype(dt, np.complexfloating) else np.float64
    try:
        for mode, nb, shrink in ((1, 64, 12), (1, 128, 12), (1, 320, 12), (1, 512, 2),
                                 (0, 256, 12), (3, 256, 12)):
            lib.xkb_tune_set(b"getrf_blocked", float(mode))
            lib.xkb_tune_set(b"getrf_oz_leaf", 512.0 if mode == 3 else 4096.0)
            lib.xkb_tune_set(b"getrf_nb", float(nb))
            lib.xkb_tune_set(b"getrf_shrink", float(shrink))
            A0 = _dd(n, dt, 50 + nb)
            A = A0.copy(order="F")
            assert _getrf(xk, A) == 0
            L = np.tril(A, -1).astype(up) + np.eye(n)
            U = np.triu(A).astype(up)
            scale = np.abs(A0).max() * n * EPS[dt]
            assert np.abs(L @ U - A0.astype(up)).max() <= 16 * scale, (mode, nb)
            Z = np.asfortranarray((np.eye(n) * 2.0).astype(dt))
            Z[776, 776] = 0.0
            assert _getrf(xk, Z) == 777, (mode, nb)
    finally:
        lib.xkb_tune_set(b"getrf_blocked", 3.0)
        lib.xkb_tune_set(b"getrf_nb", 512.0)
        lib.xkb_tune_set(b"getrf_shrink", 12.0)
        lib.xkb_tune_set(b"getrf_oz_leaf", 4096.0)
