"""Cholesky factorization through the public API (xkblas_?potrf_async +
memory_coherent_async on the stored triangle + sync; reference
blas/zpotrf.c): the factor reproduces A (backward error bound), matches
LAPACK's factor from numpy on the same matrix, leaves the other triangle of
the host matrix untouched, and reports the first non-positive pivot of a
matrix that is not positive definite.  Requires a B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UP, LO = 121, 122
EPS = {np.float64: 2.0 ** -53, np.complex128: 2.0 ** -53,
       np.float32: 2.0 ** -24, np.complex64: 2.0 ** -24}


def _spd(n, dt, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n))
    if np.issubdtype(dt, np.complexfloating):
        B = B + 1j * rng.standard_normal((n, n))
    A = B @ B.conj().T / n + np.eye(n)
    return np.asfortranarray(A.astype(dt))


def _potrf(xk, A, uplo):
    p = {np.dtype(np.float32): "s", np.dtype(np.float64): "d",
         np.dtype(np.complex64): "c", np.dtype(np.complex128): "z"}[A.dtype]
    lib = xk.lib()
    r = getattr(lib, "xkblas_%spotrf_async" % p)(uplo, A.shape[0], xk._ptr(A), A.shape[0])
    assert r == 0
    xk.coherent(A, uplo)
    xk.sync()
    info = lib.xkblas_potrf_info()
    xk.invalidate_caches()
    return info


@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32, np.complex64])
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n", [1, 7, 64, 65, 127, 128, 129, 200, 700])
def test_potrf_factor(xk, dt, uplo, n):
    A0 = _spd(n, dt, 10 + n)
    A = A0.copy(order="F")
    assert _potrf(xk, A, uplo) == 0
    up = np.complex128 if np.issubdtype(dt, np.complexfloating) else np.float64
    if uplo == LO:
        L = np.tril(A).astype(up)
        R = L @ L.conj().T
        other = np.triu(A, 1) == np.triu(A0, 1)
        ref = np.linalg.cholesky(A0.astype(up))
        got = L
    else:
        U = np.triu(A).astype(up)
        R = U.conj().T @ U
        other = np.tril(A, -1) == np.tril(A0, -1)
        ref = np.linalg.cholesky(A0.astype(up)).conj().T
        got = U
    assert other.all()  # the other triangle of the host matrix is untouched
    scale = np.abs(A0).max() * n * EPS[dt]
    assert np.abs(R - A0.astype(up)).max() <= 16 * scale
    assert np.abs(got - ref).max() <= 64 * n * EPS[dt] * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("dt,uplo", [(np.float64, LO), (np.complex128, UP)])
@pytest.mark.parametrize("mode", [0, 2, 3])
def test_potrf_tensor_op_mode(xk, dt, uplo, mode):
    """XKBLAS_TENSOR_OP_MATH: in the recursive form (tuning key
    potrf_blocked = 0) the top-level trailing update and the panel solve's
    coupling updates (all dimensions >= 2048 at n = 4200) run in the Ozaki
    INT8 form; the blocked form (= 2) and the hybrid (= 3: the recursion's
    top update in the Ozaki form, the two halves blocked) are also checked.
    Same backward-error bound as the plain factorization."""
    n = 4200
    A0 = _spd(n, dt, 11)
    A = A0.copy(order="F")
    lib = xk.lib()
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    lib.xkb_tune_set(b"potrf_blocked", float(mode))
    try:
        c0 = xk.ozaki_counts()[0]
        assert _potrf(xk, A, uplo) == 0
        if mode in (0, 3):  # the recursion (3: down to 4096 rows, blocked below)
            assert xk.ozaki_counts()[0] > c0  # Ozaki contractions ran
    finally:
        xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)
        lib.xkb_tune_set(b"potrf_blocked", 3.0)
    up = np.complex128 if np.iscomplexobj(A0) else np.float64
    if uplo == LO:
        L = np.tril(A)
        R = L @ L.conj().T
    else:
        U = np.triu(A)
        R = U.conj().T @ U
    scale = np.abs(A0).max() * n * EPS[dt]
    assert np.abs(R - A0.astype(up)).max() <= 16 * scale


def test_potrf_reports_first_bad_pivot(xk):
    n = 300
    A = _spd(n, np.float64, 3)
    A[150, 150] = -5.0  # leading 150x150 block stays positive definite
    assert _potrf(xk, A, LO) == 151


@pytest.mark.parametrize("dt,uplo,col", [(np.float64, UP, 6), (np.complex128, LO, 70),
                                          (np.complex128, UP, 1), (np.float64, LO, 129)])
def test_potrf_reports_bad_pivot_in_block(xk, dt, uplo, col):
    """A non-positive pivot inside a diagonal block (first column of a step,
    mid-step, past the first block) is reported 1-based."""
    n = 160
    A = _spd(n, dt, 5)
    A[col - 1, col - 1] = -5.0  # the leading (col-1) x (col-1) block stays positive definite
    assert _potrf(xk, A, uplo) == col


def test_potrf_argument_codes(xk):
    lib = xk.lib()
    A = np.zeros((4, 4), order="F")
    assert lib.xkblas_dpotrf_async(120, 4, xk._ptr(A), 4) == -2
    assert lib.xkblas_dpotrf_async(122, 0, xk._ptr(A), 1) == 0  # empty: nothing to do
    assert lib.xkblas_dpotrf_async(LO, -1, xk._ptr(A), 4) == -5
    assert lib.xkblas_dpotrf_async(LO, 4, xk._ptr(A), 3) == -8
    assert lib.xkblas_dpotrf_async(LO, 0, xk._ptr(A), 1) == 0


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("uplo", [LO, UP])
def test_potrf_blocked_and_recursive_forms(xk, dt, uplo):
    """The blocked look-ahead form (tuning key potrf_blocked = 1, several
    block widths, widths shrinking along the factorization, a ragged last
    block) and the recursive form (= 0) meet the same backward-error bound,
    and both report a bad pivot in a late block."""
    lib = xk.lib()
    n = 1100
    up = np.complex128 if np.issubdtype(dt, np.complexfloating) else np.float64
    try:
        for mode, nb, shrink in ((1, 64, 8), (1, 128, 8), (1, 320, 8), (1, 512, 2), (0, 256, 8)):
            lib.xkb_tune_set(b"potrf_blocked", float(mode))
            lib.xkb_tune_set(b"potrf_nb", float(nb))
            lib.xkb_tune_set(b"potrf_shrink", float(shrink))
            A0 = _spd(n, dt, 40 + nb)
            A = A0.copy(order="F")
            assert _potrf(xk, A, uplo) == 0
            F = np.tril(A).astype(up) if uplo == LO else np.triu(A).astype(up)
            R = F @ F.conj().T if uplo == LO else F.conj().T @ F
            scale = np.abs(A0).max() * n * EPS[dt]
            assert np.abs(R - A0.astype(up)).max() <= 16 * scale, (mode, nb)
            B = _spd(n, dt, 41 + nb)
            B[776, 776] = -5.0
            assert _potrf(xk, B, uplo) == 777, (mode, nb)
    finally:
        lib.xkb_tune_set(b"potrf_blocked", 3.0)
        lib.xkb_tune_set(b"potrf_nb", 512.0)
        lib.xkb_tune_set(b"potrf_shrink", 12.0)
