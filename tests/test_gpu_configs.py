"""GPU parity at the benchmark configurations' own shapes, through the public
API with host matrices (reference calling sequence, testing/ztesting_*.c),
plain FP64 and tensor-op (Ozaki) mode:

  * DGEMM NN 1024^3, alpha 1.5, beta -0.5, NB = 256;
  * DTRSM L/L/N/N 4096 x 4096, alpha 2, diagonal + 4096, NB = 512;
  * DSYRK and ZHERK L/N, N = K = 8192, alpha = beta = 1;
  * DGEMM NN 16384^3 with exponents in [-20, 20] per row of A / column of B.

Each result is judged against the reference's CPU path -- the system BLAS
through the same Fortran symbols xkblas_?xxx_native calls, restated by the
oracle -- with the reference test programs' bounds (tests/checks.py), and
its error against the double-double oracle is measured on sampled entries:
the tensor-op form must be no worse than the plain one.  Requires a B200;
the large shapes take a few seconds of host BLAS each."""
import os

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_, T_, C_ = 111, 112, 113
UP, LO = 121, 122
LEFT, NONUNIT = 141, 131
EPS = 2.0 ** -53


@pytest.fixture(scope="module")
def blas():
    O.blas_open(threads=os.cpu_count())
    return O


def _modes(xk):
    for mode in (xk.XKBLAS_DEFAULT_MATH, xk.XKBLAS_TENSOR_OP_MATH):
        xk.set_modemath(mode)
        try:
            yield "ozaki" if mode else "plain"
        finally:
            xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)


def _sample(n, k, seed):
    return np.sort(np.random.default_rng(seed).choice(n, min(n, k), replace=False))


def dd_gemm_err(C, ta, tb, alpha, A, B, beta, C0, rows, cols):
    """max over the sampled entries of |C - C_dd| / (|alpha||op(A)||op(B)| +
    |beta||C0|), C_dd the double-double result rounded once."""
    dd = O.gemm_dd(ta, tb, alpha, A, B, beta, C0, rows, cols)
    opA = A if ta == N_ else A.T
    opB = B if tb == N_ else B.T
    scale = abs(alpha) * (np.abs(opA[rows]) @ np.abs(opB[:, cols]))
    if C0 is not None:
        scale = scale + abs(beta) * np.abs(C0[np.ix_(rows, cols)])
    return float(np.max(np.abs(C[np.ix_(rows, cols)] - dd) / scale))


def test_config1_dgemm_1024_nb256(xk, blas):
    M = N = K = 1024
    A, B, C0 = O.plrnt(M, K, 1), O.plrnt(K, N, 2), O.plrnt(M, N, 3)
    R = O.native_gemm(N_, N_, 1.5, A, B, -0.5, C0.copy(order="F"))
    rows, cols = _sample(M, 64, 1), _sample(N, 64, 2)
    err = {}
    xk.set_param(256)
    try:
        for mode in _modes(xk):
            C = C0.copy(order="F")
            xk.gemm(N_, N_, 1.5, A, B, -0.5, C)
            xk.invalidate_caches()
            assert checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, K) <= 3.0, mode
            assert checks.plasma_ratio(C, R, A, B, 1.5, K) < 10, mode
            err[mode] = dd_gemm_err(C, N_, N_, 1.5, A, B, -0.5, C0, rows, cols)
    finally:
        xk.set_param(0)
    assert err["ozaki"] <= max(err["plain"], EPS), err


def test_config2_dtrsm_4096_nb512(xk, blas):
    M = N = 4096
    A = np.asfortranarray(np.tril(O.plrnt(M, M, 21)) + M * np.eye(M))
    B0 = O.plrnt(M, N, 22)
    R = O.native_trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B0.copy(order="F"))
    rows, cols = _sample(M, 48, 3), _sample(N, 48, 4)
    berr = {}
    xk.set_param(512)
    try:
        for mode in _modes(xk):
            B = B0.copy(order="F")
            xk.trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B)
            xk.invalidate_caches()
            # reference bound, testing/ztesting_trsm.c:246-252
            assert checks.trsm_ratio(B, R, A, M, N) <= 10, mode
            # componentwise backward error of the solve: the residual
            # A X - 2 B0 in double-double on sampled entries
            res = O.gemm_dd(N_, N_, 1.0, A, B, -2.0, B0, rows, cols)
            den = np.abs(A[rows]) @ np.abs(B[:, cols]) + 2.0 * np.abs(B0[np.ix_(rows, cols)])
            berr[mode] = float(np.max(np.abs(res) / den))
            assert berr[mode] < M * EPS, (mode, berr[mode])
    finally:
        xk.set_param(0)


@pytest.mark.parametrize("herm", [False, True])
def test_config3_dsyrk_zherk_8192(xk, blas, herm):
    N = K = 8192
    A = O.plrnt(N, K, 31, cplx=herm)
    C0 = O.plgsy(N, 32, cplx=herm)
    if herm:
        C0[np.diag_indices(N)] = C0[np.diag_indices(N)].real
    R = O.native_rk(LO, N_, 1.0, A, 1.0, C0.copy(order="F"), herm=herm)
    # sampled lower-triangle entries
    rows = _sample(N, 64, 5)
    cols = np.sort(np.unique(np.concatenate([rows[:32], _sample(N, 32, 6)])))
    err = {}
    for mode in _modes(xk):
        C = C0.copy(order="F")
        xk.syrk(LO, N_, 1.0, A, 1.0, C, herm=herm)
        xk.invalidate_caches()
        # reference bound, testing/ztesting_syrk.c:225-231 / ztesting_herk.c:239-245
        assert checks.rk_ratio(np.tril(C), np.tril(R), A, C0, N) <= 10, mode
        iu = np.triu_indices(N, 1)
        assert np.array_equal(C[iu], C0[iu]), mode  # upper triangle untouched
        if herm:
            assert np.all(np.diag(C).imag == 0), mode
        dd = O.gemm_dd(N_, C_ if herm else T_, 1.0, A, A, 1.0, C0, rows, cols)
        scale = np.abs(A[rows]) @ np.abs(A[cols]).T + np.abs(C0[np.ix_(rows, cols)])
        low = rows[:, None] >= cols[None, :]
        e = np.abs(C[np.ix_(rows, cols)] - dd) / scale
        err[mode] = float(e[low].max())
    assert err["ozaki"] <= max(err["plain"], EPS), err
    assert err["ozaki"] < 2.0 ** -50


def test_config4_dgemm_16384_exponent_spread(xk):
    """The headline workload at full size: Ozaki error vs the double-double
    oracle no worse than the plain DMMA kernel's, on sampled entries."""
    M = N = K = 16384
    A = O.expspread(M, K, 1, emax=20, by_col=False)
    B = O.expspread(K, N, 2, emax=20, by_col=True)
    rows, cols = _sample(M, 16, 7), _sample(N, 256, 8)
    err = {}
    for mode in _modes(xk):
        C = np.zeros((M, N), order="F")
        xk.gemm(N_, N_, 1.0, A, B, 0.0, C)
        xk.invalidate_caches()
        err[mode] = dd_gemm_err(C, N_, N_, 1.0, A, B, 0.0, None, rows, cols)
        del C
    assert err["ozaki"] <= err["plain"], err
    assert err["ozaki"] < 2.0 ** -52, err
