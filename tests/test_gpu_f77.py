"""The synchronous forms: the Fortran-77 drop-in BLAS (libxkblas_blas.so:
dgemm_, ztrsm_, zherk_ ... with character options and by-reference
arguments, reference blas/zlibxkblas_wrapper.c) and the C entry points
xkblas_?xxx_sync, checked against the CPU oracle under the reference's
acceptance bounds (tests/checks.py).  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
import xkblas_b200 as X
from tests import checks

pytestmark = pytest.mark.gpu

byref = ctypes.byref
c_int = ctypes.c_int


def _f77():
    X.lib()  # libxkblas.so first (the F77 library resolves against it)
    return ctypes.CDLL(X.F77_LIB_PATH)


def _scal(v, dt):
    return np.array([v], dtype=dt)


_KEEP = []


def _p(a):
    _KEEP.append(a)  # the array must outlive the call that receives its address
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32])
@pytest.mark.parametrize("ta,tb", [(b"N", b"N"), (b"T", b"N"), (b"n", b"c")])
def test_f77_gemm(xk, dt, ta, tb):
    cplx = np.issubdtype(dt, np.complexfloating)
    if not cplx and tb == b"c":
        tb = b"t"
    M, N, K = 157, 93, 211
    A = O.plrnt(M, K, 5, cplx) if ta in (b"N", b"n") else O.plrnt(K, M, 5, cplx)
    B = O.plrnt(K, N, 6, cplx) if tb in (b"N", b"n") else O.plrnt(N, K, 6, cplx)
    C0 = O.plrnt(M, N, 7, cplx)
    A, B, C0 = (np.asfortranarray(x.astype(dt)) for x in (A, B, C0))
    C = C0.copy(order="F")
    al, be = (1.5 - 0.5j, -0.25 + 0.5j) if cplx else (1.5, -0.25)
    name = {np.float64: "dgemm_", np.complex128: "zgemm_", np.float32: "sgemm_"}[dt]
    getattr(_f77(), name)(ta, tb, byref(c_int(M)), byref(c_int(N)), byref(c_int(K)),
                          _p(_scal(al, dt)), _p(A), byref(c_int(M if ta in (b"N", b"n") else K)),
                          _p(B), byref(c_int(K if tb in (b"N", b"n") else N)), _p(_scal(be, dt)),
                          _p(C), byref(c_int(M)))
    up = np.complex128 if cplx else np.float64
    code = {b"N": 111, b"n": 111, b"T": 112, b"t": 112, b"c": 113}
    ref = O.gemm(code[ta], code[tb], al, A.astype(up), B.astype(up), be, C0.astype(up, order="F"))
    r = checks.gemm_ratio(C, ref, A, B, C0, al, be, K)
    assert r <= 3, r


def test_f77_trsm_herk_and_sync_forms(xk):
    f = _f77()
    # ztrsm_ L / L / C / N
    M, N = 190, 77
    A = np.asfortranarray(O.plrnt(M, M, 21, True) / M + np.eye(M))
    B0 = O.plrnt(M, N, 22, True)
    B = B0.copy(order="F")
    al = _scal(2.0 - 1.0j, np.complex128)
    f.ztrsm_(b"L", b"L", b"C", b"N", byref(c_int(M)), byref(c_int(N)), _p(al), _p(A),
             byref(c_int(M)), _p(B), byref(c_int(M)))
    R = O.trsm(141, 122, 113, 131, al[0], A, B0.copy(order="F"), nb=64)
    assert checks.trsm_ratio(B, R, A, M, N) <= 10
    # zherk_ U / N, real alpha / beta
    n, k = 150, 201
    Ah = O.plrnt(n, k, 23, True)
    C0 = np.asfortranarray(O.plgsy(n, 24, cplx=True))
    C = C0.copy(order="F")
    f.zherk_(b"U", b"N", byref(c_int(n)), byref(c_int(k)), _p(_scal(0.5, np.float64)), _p(Ah),
             byref(c_int(n)), _p(_scal(2.0, np.float64)), _p(C), byref(c_int(n)))
    R = O.syrk(121, 111, 0.5, Ah, 2.0, C0.copy(order="F"), herm=True)
    r = checks.rk_ratio(np.triu(C), np.triu(R), Ah, C0, n)
    assert r <= 10, r
    # the C synchronous form: xkblas_dsyrk_sync (lower, transposed)
    Ad = O.plrnt(k, n, 25)
    Cd0 = np.asfortranarray(O.plgsy(n, 26))
    Cd = Cd0.copy(order="F")
    assert xk.lib().xkblas_dsyrk_sync(122, 112, n, k, _p(_scal(1.0, np.float64)), _p(Ad), k,
                                      _p(_scal(-1.0, np.float64)), _p(Cd), n) == 0
    R = O.syrk(122, 112, 1.0, Ad, -1.0, Cd0.copy(order="F"))
    assert checks.rk_ratio(np.tril(Cd), np.tril(R), Ad, Cd0, n) <= 10
    # each synchronous call ran through the async entry points (counted there)
    assert xk.stats()["calls"] >= 3


def test_f77_reports_bad_option_without_computing(xk, capfd):
    C = np.ones((4, 4), order="F")
    A = np.ones((4, 4), order="F")
    _f77().dgemm_(b"X", b"N", byref(c_int(4)), byref(c_int(4)), byref(c_int(4)),
                  _p(_scal(1.0, np.float64)), _p(A), byref(c_int(4)), _p(A), byref(c_int(4)),
                  _p(_scal(0.0, np.float64)), _p(C), byref(c_int(4)))
    err = capfd.readouterr().err
    assert "DGEMM parameter number 1" in err
    assert np.all(C == 1.0)
