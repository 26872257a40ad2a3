"""Python mirror of the XKBlas C API over libxkblas.so (ctypes).

The product is the C-ABI library ``libxkblas.so`` built in-tree by
``xkblas_b200.build``; this module only loads it and offers numpy-friendly
wrappers with the reference's calling sequence (``xkblas_?xxx_async`` ->
``xkblas_memory_coherent_async`` -> ``xkblas_sync``, reference
testing/ztesting_gemm.c:157-163).  Importing fails loudly when the library
is missing: there is no Python or CPU fallback for the GPU path.
"""
import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxkblas.so")
# the Fortran-77 drop-in BLAS (dgemm_ ...), built on top of libxkblas.so
F77_LIB_PATH = os.path.join(HERE, "libxkblas_blas.so")

# CBLAS enum values of the reference header (blas/xkblas.h:114-118)
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113
CblasUpper, CblasLower = 121, 122
CblasNonUnit, CblasUnit = 131, 132
CblasLeft, CblasRight = 141, 142
XKBLAS_DEFAULT_MATH, XKBLAS_TENSOR_OP_MATH = 0, 1

_PREFIX = {np.dtype(np.float32): "s", np.dtype(np.float64): "d",
           np.dtype(np.complex64): "c", np.dtype(np.complex128): "z"}
_REAL = {"s": np.float32, "d": np.float64, "c": np.float32, "z": np.float64}

_lib = None


class GemmArgs(ctypes.Structure):
    """xkb_gemm_args of include/xkb_cuda.h."""
    _fields_ = [("dtype", ctypes.c_int), ("opA", ctypes.c_int), ("opB", ctypes.c_int),
                ("M", ctypes.c_int), ("N", ctypes.c_int), ("K", ctypes.c_int),
                ("A", ctypes.c_void_p), ("lda", ctypes.c_long),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_long),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_long),
                ("alpha", ctypes.c_double * 2), ("beta", ctypes.c_double * 2),
                ("uplo", ctypes.c_int), ("herm_diag", ctypes.c_int), ("diag", ctypes.c_long)]


class BatchOp(ctypes.Structure):
    """xkb_batch_op of include/xkb_cuda.h."""
    _fields_ = [("kind", ctypes.c_int), ("dtype", ctypes.c_int), ("opA", ctypes.c_int),
                ("opB", ctypes.c_int), ("side", ctypes.c_int), ("uplo", ctypes.c_int),
                ("trans", ctypes.c_int), ("diag", ctypes.c_int), ("M", ctypes.c_int),
                ("N", ctypes.c_int), ("K", ctypes.c_int),
                ("A", ctypes.c_void_p), ("lda", ctypes.c_long),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_long),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_long),
                ("alpha", ctypes.c_double * 2), ("beta", ctypes.c_double * 2)]


class TraceRec(ctypes.Structure):
    """xkb_trace_rec of include/xkb_cuda.h (per-call phase timings)."""
    _fields_ = [("op", ctypes.c_char * 16), ("dtype", ctypes.c_int), ("M", ctypes.c_int),
                ("N", ctypes.c_int), ("K", ctypes.c_int), ("nmod", ctypes.c_int),
                ("ms_total", ctypes.c_float), ("ms_convert", ctypes.c_float),
                ("ms_gemm", ctypes.c_float), ("ms_crt", ctypes.c_float)]


class XkblasError(RuntimeError):
    pass


class Stats(ctypes.Structure):
    _fields_ = [("calls", ctypes.c_uint64), ("kernels", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("tile_hits", ctypes.c_uint64), ("tile_misses", ctypes.c_uint64),
                ("ozaki_calls", ctypes.c_uint64), ("ozaki_moduli", ctypes.c_uint64),
                ("flops", ctypes.c_double), ("batches", ctypes.c_uint64),
                ("batched_calls", ctypes.c_uint64), ("evictions", ctypes.c_uint64)]


def lib():
    """The loaded libxkblas.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise XkblasError("libxkblas.so not built: run python -m xkblas_b200.build")
        _lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        _lib.xkblas_get_configuration.restype = ctypes.c_char_p
        _lib.xkblas_elapsedtime.restype = ctypes.c_double
        _lib.xkblas_elapsedns.restype = ctypes.c_uint64
        _lib.xkblas_malloc.restype = ctypes.c_void_p
        _lib.xkblas_malloc.argtypes = [ctypes.c_size_t]
        _lib.xkblas_free.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        _lib.xkblas_find.restype = ctypes.c_void_p
        _lib.xkblas_find.argtypes = [ctypes.c_void_p]
        _lib.xkblas_get_param.restype = ctypes.c_size_t
        _lib.xkblas_set_param.argtypes = [ctypes.c_size_t, ctypes.c_size_t]
        _lib.xkblas_auto_tilesize.restype = ctypes.c_size_t
        _lib.xkblas_auto_tilesize.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t,
                                              ctypes.c_size_t, ctypes.c_size_t]
        _lib.xkblas_context_get.restype = ctypes.c_void_p
        _lib.xkblas_memory_coherent_async.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p,
            ctypes.c_size_t, ctypes.c_size_t]
        _lib.xkblas_memory_invalidate.argtypes = [ctypes.c_void_p]
        _lib.xkb_cuda_kernel_count.restype = ctypes.c_uint64
        _lib.xkb_tune_get.restype = ctypes.c_double
        _lib.xkb_tune_get.argtypes = [ctypes.c_char_p, ctypes.c_double]
        _lib.xkb_tune_set.argtypes = [ctypes.c_char_p, ctypes.c_double]
        _lib.xkb_tune_load.argtypes = [ctypes.c_char_p]
        c_int, c_long, c_vp = ctypes.c_int, ctypes.c_long, ctypes.c_void_p
        dptr = ctypes.POINTER(ctypes.c_double)
        _lib.xkb_cuda_trsm.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, c_int, dptr,
                                       c_vp, c_long, c_vp, c_long, c_int, c_vp]
        _lib.xkb_cuda_trmm.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, c_int, dptr,
                                       c_vp, c_long, c_vp, c_long, c_int, c_vp]
        _lib.xkb_cuda_symm.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, dptr, c_vp,
                                       c_long, c_vp, c_long, dptr, c_vp, c_long, c_int, c_vp]
        _lib.xkb_cuda_scale.argtypes = [c_int, c_int, c_int, dptr, c_vp, c_long, c_int, c_int,
                                        c_long, c_vp]
        _lib.xkb_ozaki_default_moduli.argtypes = [c_long]
        _lib.xkb_cuda_potrf.argtypes = [c_int, c_int, c_int, c_vp, c_long, c_vp, c_int, c_vp]
        _lib.xkb_cuda_getrf_nopiv.argtypes = [c_int, c_int, c_vp, c_long, c_vp, c_int, c_vp]
        _lib.xkb_cuda_batch.argtypes = [ctypes.POINTER(BatchOp), c_int, c_int, c_vp]
        _lib.xkb_cuda_batch_latency.argtypes = [ctypes.POINTER(ctypes.c_double), c_int]
        _lib.xkblas_get_stats.argtypes = [ctypes.POINTER(Stats)]
        _lib.xkblas_trace_export.argtypes = [ctypes.c_char_p]
        _lib.xkblas_trace_dropped.restype = ctypes.c_uint64
        _lib.xkb_trace_take.argtypes = [ctypes.POINTER(TraceRec), c_int]
        _lib.xkb_ozaki_counts.argtypes = [ctypes.POINTER(ctypes.c_ulonglong),
                                          ctypes.POINTER(c_int), c_int]
    return _lib


def init():
    r = lib().xkblas_init()
    if r != 0:
        raise XkblasError("xkblas_init failed: %d" % r)


def finalize():
    return lib().xkblas_finalize()


def sync():
    r = lib().xkblas_sync()
    if r != 0:
        raise XkblasError("xkblas_sync failed: %d" % r)


def set_modemath(mode):
    lib().xkblas_set_modemath(int(mode))


def set_param(nb, p=8):
    lib().xkblas_set_param(nb, p)


def stats():
    s = Stats()
    lib().xkblas_get_stats(ctypes.byref(s))
    return {k: getattr(s, k) for k, _ in Stats._fields_}


def reset_stats():
    lib().xkblas_reset_stats()


def invalidate_caches():
    return lib().xkblas_memory_invalidate_caches()


def trace_record(on=True):
    """Switch event recording on or off; returns the previous state."""
    return bool(lib().xkblas_trace_record(1 if on else 0))


def trace_export(directory):
    """Write the recorded events as kern.csv, cpy.csv, call.csv, task.csv and
    parallel.csv into `directory` (the column layout of the reference's trace
    converter, bin/ukilli.cpp); raises on failure."""
    r = lib().xkblas_trace_export(os.fsencode(directory))
    if r != 0:
        raise XkblasError("xkblas_trace_export failed: %d" % r)


def kernel_count():
    return lib().xkb_cuda_kernel_count()


def ozaki_counts(reset=False):
    """Device counters of the Ozaki contractions: (calls, moduli summed,
    calls sent to the plain FP64 kernel, latest call's count)."""
    out = (ctypes.c_ulonglong * 3)()
    last = ctypes.c_int(-1)
    r = lib().xkb_ozaki_counts(out, ctypes.byref(last), 1 if reset else 0)
    if r != 0:
        raise XkblasError("xkb_ozaki_counts failed: %d" % r)
    return int(out[0]), int(out[1]), int(out[2]), int(last.value)


class contraction_trace:
    """Context manager collecting the per-call records (xkb_trace_rec) of the
    contractions launched inside it: `.records` after exit."""

    def __enter__(self):
        self.prev = lib().xkb_trace_enable(1)
        lib().xkb_trace_take(None, 0)
        self.records = []
        return self

    def __exit__(self, *exc):
        buf = (TraceRec * 256)()
        n = lib().xkb_trace_take(buf, 256)
        self.records = [buf[i] for i in range(n)]
        lib().xkb_trace_enable(self.prev)
        return False

    def ops(self):
        return [r.op.decode() for r in self.records]


# ---- numpy wrappers -----------------------------------------------------------
def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


_KEEP = threading.local()


def _scal(v, dt):
    # scalar passed by pointer: kept alive until the call returns (a list per
    # thread: another thread's trimming never frees it mid-call)
    a = np.array([v], dtype=dt)
    keep = _KEEP.__dict__.setdefault("a", [])
    keep.append(a)
    if len(keep) > 64:
        del keep[:32]
    return a


def _check_f(*arrs):
    for a in arrs:
        if a is not None and not a.flags.f_contiguous:
            raise ValueError("arrays must be Fortran (column-major) contiguous")


def coherent(C, uplo=0, memflag=0):
    r = lib().xkblas_memory_coherent_async(uplo, memflag, C.shape[0], C.shape[1], _ptr(C),
                                           C.shape[0], C.dtype.itemsize)
    if r != 0:
        raise XkblasError("coherent_async failed: %d" % r)


def _finish(C, r, name, uplo=0):
    if r != 0:
        raise XkblasError("%s returned %d" % (name, r))
    coherent(C, uplo)
    sync()


def gemm(transA, transB, alpha, A, B, beta, C, sync_result=True):
    """C <- alpha op(A) op(B) + beta C through xkblas_?gemm_async (in place)."""
    _check_f(A, B, C)
    p = _PREFIX[C.dtype]
    M, N = C.shape
    K = A.shape[1] if transA == CblasNoTrans else A.shape[0]
    f = getattr(lib(), "xkblas_%sgemm_async" % p)
    r = f(transA, transB, M, N, K, _ptr(_scal(alpha, C.dtype)), _ptr(A), A.shape[0], _ptr(B),
          B.shape[0], _ptr(_scal(beta, C.dtype)), _ptr(C), C.shape[0])
    if sync_result:
        _finish(C, r, "gemm")
    return r


def gemmt(uplo, transA, transB, alpha, A, B, beta, C):
    _check_f(A, B, C)
    p = _PREFIX[C.dtype]
    N = C.shape[0]
    K = A.shape[1] if transA == CblasNoTrans else A.shape[0]
    f = getattr(lib(), "xkblas_%sgemmt_async" % p)
    r = f(uplo, transA, transB, N, K, _ptr(_scal(alpha, C.dtype)), _ptr(A), A.shape[0], _ptr(B),
          B.shape[0], _ptr(_scal(beta, C.dtype)), _ptr(C), C.shape[0])
    _finish(C, r, "gemmt")
    return r


def trsm(side, uplo, trans, diag, alpha, A, B):
    _check_f(A, B)
    p = _PREFIX[B.dtype]
    M, N = B.shape
    f = getattr(lib(), "xkblas_%strsm_async" % p)
    r = f(side, uplo, trans, diag, M, N, _ptr(_scal(alpha, B.dtype)), _ptr(A), A.shape[0],
          _ptr(B), B.shape[0])
    _finish(B, r, "trsm")
    return r


def trmm(side, uplo, trans, diag, alpha, A, B):
    _check_f(A, B)
    p = _PREFIX[B.dtype]
    M, N = B.shape
    f = getattr(lib(), "xkblas_%strmm_async" % p)
    r = f(side, uplo, trans, diag, M, N, _ptr(_scal(alpha, B.dtype)), _ptr(A), A.shape[0],
          _ptr(B), B.shape[0])
    _finish(B, r, "trmm")
    return r


def symm(side, uplo, alpha, A, B, beta, C, herm=False):
    _check_f(A, B, C)
    p = _PREFIX[C.dtype]
    M, N = C.shape
    f = getattr(lib(), "xkblas_%s%smm_async" % (p, "he" if herm else "sy"))
    r = f(side, uplo, M, N, _ptr(_scal(alpha, C.dtype)), _ptr(A), A.shape[0], _ptr(B), B.shape[0],
          _ptr(_scal(beta, C.dtype)), _ptr(C), C.shape[0])
    _finish(C, r, "symm")
    return r


def syrk(uplo, trans, alpha, A, beta, C, herm=False):
    _check_f(A, C)
    p = _PREFIX[C.dtype]
    N = C.shape[0]
    K = A.shape[1] if trans == CblasNoTrans else A.shape[0]
    sdt = _REAL[p] if herm else C.dtype
    f = getattr(lib(), "xkblas_%s%srk_async" % (p, "he" if herm else "sy"))
    r = f(uplo, trans, N, K, _ptr(_scal(alpha, sdt)), _ptr(A), A.shape[0],
          _ptr(_scal(beta, sdt)), _ptr(C), C.shape[0])
    _finish(C, r, "syrk")
    return r


def syr2k(uplo, trans, alpha, A, B, beta, C, herm=False):
    _check_f(A, B, C)
    p = _PREFIX[C.dtype]
    N = C.shape[0]
    K = A.shape[1] if trans == CblasNoTrans else A.shape[0]
    bdt = _REAL[p] if herm else C.dtype
    f = getattr(lib(), "xkblas_%s%sr2k_async" % (p, "he" if herm else "sy"))
    r = f(uplo, trans, N, K, _ptr(_scal(alpha, C.dtype)), _ptr(A), A.shape[0], _ptr(B),
          B.shape[0], _ptr(_scal(beta, bdt)), _ptr(C), C.shape[0])
    _finish(C, r, "syr2k")
    return r


def pinned_empty(shape, dtype):
    """Column-major numpy array in pinned host memory (xkblas_malloc); the
    buffer stays alive as long as the returned array."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    p = lib().xkblas_malloc(max(n, 1))
    if not p:
        raise MemoryError("xkblas_malloc failed")
    buf = (ctypes.c_char * max(n, 1)).from_address(p)
    arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape, order="F")
    arr = arr.view(_Pinned)
    arr._xkb_ptr = p
    arr._xkb_n = n
    return arr


class _Pinned(np.ndarray):
    def __del__(self):
        # at interpreter exit module globals may already be gone: then the
        # process is ending and the pinned block goes with it
        try:
            p = getattr(self, "_xkb_ptr", None)
            if p and self.base is not None and not isinstance(self.base, _Pinned):
                lib().xkblas_free(ctypes.c_void_p(p), self._xkb_n)
        except Exception:
            pass
