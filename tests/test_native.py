"""The xkblas_?xxx_native entry points of libxkblas.so (the reference's CPU
tile bodies, blas/zgemm.c:383-414, blas/ztrsm.c:510-538, blas/zsyrk.c:330-357,
blas/zherk.c:333-360): direct calls of the system BLAS named by
XKBLAS_BLASLIB (blas/xkblas.c:2678-2696).  Checked against the golden
outputs of that BLAS (tests/golden/make_golden.py) on the same inputs: the
same library through the same Fortran symbols gives the same bits.
CPU only (no device is touched)."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
import xkblas_b200 as X

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "openblas_small.npz"))


@pytest.fixture(scope="module")
def native():
    path = O.find_openblas()
    if not path:
        pytest.skip("no system BLAS in this image")
    O.blas_open(path)  # preloads the BLAS's Fortran runtime libraries
    os.environ["XKBLAS_BLASLIB"] = path  # read by the library at its first native call
    return X.lib()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _sc(v, cplx):
    return np.array([v], dtype=np.complex128 if cplx else np.float64)


GEMM_KEYS = sorted(k[:-2] for k in GOLD.files if k.startswith("gemm_") and k.endswith("_R"))
TRSM_KEYS = sorted(k[:-2] for k in GOLD.files if k.startswith("trsm_") and k.endswith("_R"))
RK_KEYS = sorted(k[:-2] for k in GOLD.files if k.startswith("rk_") and k.endswith("_R"))


@pytest.mark.parametrize("key", GEMM_KEYS)
def test_native_gemm_matches_golden(native, key):
    _, p, ta, tb = key.split("_")
    ta, tb, cplx = int(ta), int(tb), p == "z"
    M, N, K, seed = 19, 13, 23, int(GOLD[key + "_seed"][0])
    A = O.plrnt(M, K, seed, cplx) if ta == O.NOTRANS else O.plrnt(K, M, seed, cplx)
    B = O.plrnt(K, N, seed + 1, cplx) if tb == O.NOTRANS else O.plrnt(N, K, seed + 1, cplx)
    C = O.plrnt(M, N, seed + 2, cplx)
    al, be = GOLD[key + "_ab"]
    if not cplx:
        al, be = al.real, be.real
    f = getattr(native, "xkblas_%sgemm_native" % p)
    assert f(ta, tb, M, N, K, _p(_sc(al, cplx)), _p(A), A.shape[0], _p(B), B.shape[0],
             _p(_sc(be, cplx)), _p(C), M) == 0
    np.testing.assert_array_equal(C, GOLD[key + "_R"])


@pytest.mark.parametrize("key", TRSM_KEYS)
def test_native_trsm_matches_golden(native, key):
    _, p, side, uplo, tr, dg = key.split("_")
    side, uplo, tr, dg, cplx = int(side), int(uplo), int(tr), int(dg), p == "z"
    seed = int(GOLD[key + "_seed"][0])
    M, N = 21, 17
    na = M if side == O.LEFT else N
    A = np.asfortranarray(O.plrnt(na, na, seed, cplx) / na + 2.0 * np.eye(na))
    B = O.plrnt(M, N, seed + 1, cplx)
    al = GOLD[key + "_ab"][0]
    if not cplx:
        al = al.real
    f = getattr(native, "xkblas_%strsm_native" % p)
    assert f(side, uplo, tr, dg, M, N, _p(_sc(al, cplx)), _p(A), na, _p(B), M) == 0
    np.testing.assert_array_equal(B, GOLD[key + "_R"])


@pytest.mark.parametrize("key", RK_KEYS)
def test_native_syrk_herk_matches_golden(native, key):
    _, p, uplo, tr = key.split("_")
    uplo, tr, cplx = int(uplo), int(tr), p == "z"
    seed = int(GOLD[key + "_seed"][0])
    N, K = 19, 15
    A = O.plrnt(N, K, seed, cplx) if tr == O.NOTRANS else O.plrnt(K, N, seed, cplx)
    C = O.plgsy(N, seed + 1, cplx=cplx)
    one = np.array([1.0])
    f = getattr(native, "xkblas_zherk_native" if cplx else "xkblas_dsyrk_native")
    assert f(uplo, tr, N, K, _p(one), _p(A), A.shape[0], _p(one), _p(C), N) == 0
    sel = np.tril if uplo == O.LOWER else np.triu
    np.testing.assert_array_equal(sel(C), sel(GOLD[key + "_R"]))


def test_native_missing_library_is_an_error_code():
    """A BLAS that cannot be loaded gives ENOSYS, not an abort (the
    reference aborts, blas/xkblas.c:2685-2690): checked in a fresh process
    so the library's one-time load sees the bad path."""
    import subprocess
    import sys
    code = ("import ctypes, errno, os, sys, numpy as np; sys.path.insert(0, %r);"
            "os.environ['XKBLAS_BLASLIB'] = '/nonexistent/libblas.so';"
            "import xkblas_b200 as X; a = np.ones(4); p = ctypes.c_void_p(a.ctypes.data);"
            "r = X.lib().xkblas_dgemm_native(111, 111, 2, 2, 2, p, p, 2, p, 2, p, p, 2);"
            "sys.exit(0 if r == errno.ENOSYS else 1)"
            % os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert subprocess.run([sys.executable, "-c", code], timeout=120).returncode == 0
