"""ctypes binding of the CPU oracle (libxkb_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, always as the reference results are
compared with.  The library under
test (xkblas_b200 / libxkblas.so) never imports or links this package.
"""
import ctypes
import glob
import os
import subprocess
import sysconfig
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxkb_oracle.so")

NOTRANS, TRANS, CONJTRANS = 111, 112, 113
UPPER, LOWER = 121, 122
NONUNIT, UNIT = 131, 132
LEFT, RIGHT = 141, 142

_lib = None


def build():
    """Compile libxkb_oracle.so from oracle/ (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.xko_blas_sym.restype = ctypes.c_void_p
        _lib.xko_blas_loaded.restype = ctypes.c_char_p
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


_KEEP = threading.local()


def _s(v, dt):
    # scalar passed by pointer: kept alive until 32 more are made in the same
    # thread (a list per thread: another thread never frees it mid-call)
    a = np.array([v], dtype=dt)
    keep = _KEEP.__dict__.setdefault("a", [])
    keep.append(a)
    if len(keep) > 64:
        del keep[:32]
    return a


def _pre(a):
    return "z" if np.iscomplexobj(a) else "d"


def _f(a):
    assert a.flags.f_contiguous
    assert a.dtype in (np.float64, np.complex128)


# ---- tiled drivers (in place, like the BLAS they restate) --------------------
def gemm(ta, tb, alpha, A, B, beta, C, nb=256):
    _f(A), _f(B), _f(C)
    M, N = C.shape
    K = A.shape[1] if ta == NOTRANS else A.shape[0]
    getattr(lib(), _pre(C) + "_xko_gemm")(ta, tb, M, N, K, _p(_s(alpha, C.dtype)), _p(A),
                                          A.shape[0], _p(B), B.shape[0], _p(_s(beta, C.dtype)),
                                          _p(C), C.shape[0], nb)
    return C


def gemmt(uplo, ta, tb, alpha, A, B, beta, C, nb=256):
    _f(A), _f(B), _f(C)
    N = C.shape[0]
    K = A.shape[1] if ta == NOTRANS else A.shape[0]
    getattr(lib(), _pre(C) + "_xko_gemmt")(uplo, ta, tb, N, K, _p(_s(alpha, C.dtype)), _p(A),
                                           A.shape[0], _p(B), B.shape[0],
                                           _p(_s(beta, C.dtype)), _p(C), C.shape[0], nb)
    return C


def trsm(side, uplo, trans, diag, alpha, A, B, nb=256):
    _f(A), _f(B)
    M, N = B.shape
    getattr(lib(), _pre(B) + "_xko_trsm")(side, uplo, trans, diag, M, N, _p(_s(alpha, B.dtype)),
                                          _p(A), A.shape[0], _p(B), B.shape[0], nb)
    return B


def getrf_nopiv(A, nb=256):
    """LU without pivoting in place (tile algorithm of blas/zgetrf_nopiv.c:
    48-101); returns the first zero pivot, 1-based (0 = none)."""
    _f(A)
    M, N = A.shape
    return int(getattr(lib(), _pre(A) + "_xko_getrf_nopiv")(M, N, _p(A), A.shape[0], nb))


def trmm(side, uplo, trans, diag, alpha, A, B, nb=256):
    _f(A), _f(B)
    M, N = B.shape
    getattr(lib(), _pre(B) + "_xko_trmm")(side, uplo, trans, diag, M, N, _p(_s(alpha, B.dtype)),
                                          _p(A), A.shape[0], _p(B), B.shape[0], nb)
    return B


def syrk(uplo, trans, alpha, A, beta, C, herm=False, nb=256):
    _f(A), _f(C)
    N = C.shape[0]
    K = A.shape[1] if trans == NOTRANS else A.shape[0]
    if herm:
        lib().z_xko_herk(uplo, trans, N, K, _p(_s(alpha, np.float64)), _p(A), A.shape[0],
                         _p(_s(beta, np.float64)), _p(C), C.shape[0], nb)
    else:
        getattr(lib(), _pre(C) + "_xko_syrk")(uplo, trans, N, K, _p(_s(alpha, C.dtype)), _p(A),
                                              A.shape[0], _p(_s(beta, C.dtype)), _p(C),
                                              C.shape[0], nb)
    return C


def syr2k(uplo, trans, alpha, A, B, beta, C, herm=False, nb=256):
    _f(A), _f(B), _f(C)
    N = C.shape[0]
    K = A.shape[1] if trans == NOTRANS else A.shape[0]
    if herm:
        lib().z_xko_her2k(uplo, trans, N, K, _p(_s(alpha, np.complex128)), _p(A), A.shape[0],
                          _p(B), B.shape[0], _p(_s(beta, np.float64)), _p(C), C.shape[0], nb)
    else:
        getattr(lib(), _pre(C) + "_xko_syr2k")(uplo, trans, N, K, _p(_s(alpha, C.dtype)), _p(A),
                                               A.shape[0], _p(B), B.shape[0],
                                               _p(_s(beta, C.dtype)), _p(C), C.shape[0], nb)
    return C


def symm(side, uplo, alpha, A, B, beta, C, herm=False, nb=256):
    _f(A), _f(B), _f(C)
    M, N = C.shape
    name = "z_xko_hemm" if herm else _pre(C) + "_xko_symm"
    getattr(lib(), name)(side, uplo, M, N, _p(_s(alpha, C.dtype)), _p(A), A.shape[0], _p(B),
                         B.shape[0], _p(_s(beta, C.dtype)), _p(C), C.shape[0], nb)
    return C


# ---- double-double reference on chosen entries ---------------------------------
def gemm_dd(ta, tb, alpha, A, B, beta, C, rows, cols):
    """alpha*op(A)op(B) + beta*C at (rows x cols), dot products in
    double-double, rounded once.  Returns an (len(rows), len(cols)) array."""
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    _f(A), _f(B)
    if C is not None:
        _f(C)
    K = A.shape[1] if ta == NOTRANS else A.shape[0]
    Cp = C if C is not None else None
    if np.iscomplexobj(A):
        out = np.zeros((len(rows), len(cols)), dtype=np.complex128, order="F")
        lib().xko_zgemm_dd(ta, tb, K, _p(_s(alpha, np.complex128)), _p(A), A.shape[0], _p(B),
                           B.shape[0], _p(_s(beta, np.complex128)),
                           _p(Cp) if Cp is not None else None, Cp.shape[0] if Cp is not None else 1,
                           _p(rows), len(rows), _p(cols), len(cols), _p(out))
    else:
        out = np.zeros((len(rows), len(cols)), dtype=np.float64, order="F")
        lib().xko_dgemm_dd(ta, tb, K, ctypes.c_double(alpha), _p(A), A.shape[0], _p(B),
                           B.shape[0], ctypes.c_double(beta),
                           _p(Cp) if Cp is not None else None, Cp.shape[0] if Cp is not None else 1,
                           _p(rows), len(rows), _p(cols), len(cols), _p(out))
    return out


# ---- generators --------------------------------------------------------------
def plrnt(M, N, seed, cplx=False, bigM=None, i0=0, j0=0):
    """Column-major M x N matrix, entries 0.5 - ran*2^-64 (double multiplier)."""
    bigM = M if bigM is None else bigM
    dt = np.complex128 if cplx else np.float64
    A = np.zeros((M, N), dtype=dt, order="F")
    if M and N:
        lib().xko_plrnt(int(cplx), ctypes.c_long(M), ctypes.c_long(N), _p(A), ctypes.c_long(M),
                        ctypes.c_long(bigM), ctypes.c_long(i0), ctypes.c_long(j0),
                        ctypes.c_uint64(seed))
    return A


def plgsy(N, seed, bump=0.0, cplx=False):
    """The reference's testing_zplgsy generator (float multiplier kept)."""
    dt = np.complex128 if cplx else np.float64
    A = np.zeros((N, N), dtype=dt, order="F")
    lib().xko_plgsy(int(cplx), ctypes.c_double(bump), ctypes.c_long(N), _p(A), ctypes.c_long(N),
                    ctypes.c_uint64(seed))
    return A


def expspread(M, N, seed, emax=20, by_col=False):
    A = np.zeros((M, N), dtype=np.float64, order="F")
    lib().xko_expspread(ctypes.c_long(M), ctypes.c_long(N), _p(A), ctypes.c_long(M), emax,
                        int(by_col), ctypes.c_uint64(seed))
    return A


# ---- system BLAS (the reference's CPU path) -------------------------------------
def find_openblas():
    """The OpenBLAS shipped in this image (LP64 Fortran symbols)."""
    env = os.environ.get("XKBLAS_BLASLIB")
    if env and os.path.exists(env):
        return env
    sp = sysconfig.get_paths()["purelib"]
    for pat in ("opencv_python_headless.libs/libopenblas*.so", "opencv_python.libs/libopenblas*.so"):
        hits = sorted(glob.glob(os.path.join(sp, pat)))
        if hits:
            return hits[0]
    return None


def blas_open(path=None, threads=None):
    path = path or find_openblas()
    if not path:
        raise RuntimeError("no system BLAS found")
    # wheel-bundled OpenBLAS has no RPATH to its Fortran runtime: preload the
    # runtime libraries that sit next to it
    d = os.path.dirname(path)
    for pat in ("libquadmath*.so*", "libgfortran*.so*"):
        for dep in sorted(glob.glob(os.path.join(d, pat))):
            ctypes.CDLL(dep, mode=ctypes.RTLD_GLOBAL)
    if lib().xko_blas_open(path.encode()) != 0:
        raise RuntimeError("dlopen failed: " + path)
    if threads:
        lib().xko_blas_set_threads(int(threads))
    return path


def native_gemm(ta, tb, alpha, A, B, beta, C):
    p = {np.dtype(np.float32): b"s", np.dtype(np.float64): b"d",
         np.dtype(np.complex64): b"c", np.dtype(np.complex128): b"z"}[C.dtype]
    M, N = C.shape
    K = A.shape[1] if ta == NOTRANS else A.shape[0]
    r = lib().xko_native_gemm(ctypes.c_char(p), ta, tb, M, N, K, _p(_s(alpha, C.dtype)), _p(A),
                              A.shape[0], _p(B), B.shape[0], _p(_s(beta, C.dtype)), _p(C),
                              C.shape[0])
    if r:
        raise RuntimeError("native gemm missing")
    return C


def native_trsm(side, uplo, ta, diag, alpha, A, B):
    p = b"z" if np.iscomplexobj(B) else b"d"
    M, N = B.shape
    r = lib().xko_native_trsm(ctypes.c_char(p), side, uplo, ta, diag, M, N, _p(_s(alpha, B.dtype)),
                              _p(A), A.shape[0], _p(B), B.shape[0])
    if r:
        raise RuntimeError("native trsm missing")
    return B


def native_rk(uplo, trans, alpha, A, beta, C, herm=False):
    p = b"z" if np.iscomplexobj(C) else b"d"
    N = C.shape[0]
    K = A.shape[1] if trans == NOTRANS else A.shape[0]
    sdt = np.float64 if herm else C.dtype
    r = lib().xko_native_rk(ctypes.c_char(p), b"herk_" if herm else b"syrk_", uplo, trans, N, K,
                            _p(_s(alpha, sdt)), _p(A), A.shape[0], _p(_s(beta, sdt)), _p(C),
                            C.shape[0])
    if r:
        raise RuntimeError("native rk missing")
    return C
