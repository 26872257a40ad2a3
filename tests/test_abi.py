"""The C-ABI library loads on a machine without a GPU, exports every symbol
the public headers declare, and checks arguments with the reference's -i
codes before touching the device.  CPU only."""
import ctypes
import os
import re

import numpy as np
import pytest

import xkblas_b200 as X
from xkblas_b200 import GemmArgs  # xkb_gemm_args of include/xkb_cuda.h

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P = ctypes.c_void_p


def _header_functions(name):
    src = open(os.path.join(ROOT, "include", name)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    # plain declarations
    for m in re.finditer(r"\b(xkblas_\w+|xkb_\w+)\s*\(", src):
        names.add(m.group(1))
    # macro-generated level-3 entry points
    if "XKBLAS_DECL_OPS" in src:
        for p in "sdcz":
            for op in ("gemm", "gemmt", "trsm", "trmm", "symm", "syrk", "syr2k"):
                for kind in ("async", "native", "sync"):
                    names.add("xkblas_%s%s_%s" % (p, op, kind))
        for p in "cz":
            for op in ("hemm", "herk", "her2k"):
                for kind in ("async", "native", "sync"):
                    names.add("xkblas_%s%s_%s" % (p, op, kind))
    names = {n for n in names if not n.startswith("xkblas_blas2cblas")}
    names.discard("xkblas_DECL_OPS")
    return sorted(n for n in names if "##" not in n and not n.endswith("_t"))


@pytest.mark.parametrize("header", ["xkblas.h", "xkb_cuda.h"])
def test_exports_every_declared_symbol(header):
    lib = X.lib()
    missing = [n for n in _header_functions(header) if not hasattr(lib, n)]
    assert not missing, missing


def test_f77_library_exports_the_blas_names():
    """libxkblas_blas.so (the drop-in BLAS) exports every Fortran name that
    include/xkblas_f77.h declares, and libxkblas.so exports none of them (it
    must not replace a process's BLAS just by being loaded)."""
    src = open(os.path.join(ROOT, "include", "xkblas_f77.h")).read()
    names = []
    for p in "sdcz":
        for op in ("gemm", "gemmt", "trsm", "trmm", "symm", "syrk", "syr2k"):
            names.append("%s%s_" % (p, op))
    for p in "cz":
        for op in ("hemm", "herk", "her2k"):
            names.append("%s%s_" % (p, op))
    for op in ("gemm", "gemmt", "trsm", "trmm", "symm", "syrk", "syr2k", "hemm", "herk", "her2k"):
        assert "p##%s_(" % op in src  # declared by the header's macros
    f77 = ctypes.CDLL(X.F77_LIB_PATH)
    missing = [n for n in names if not hasattr(f77, n)]
    assert not missing, missing
    lib = X.lib()
    assert not [n for n in names if hasattr(lib, n)]


def test_configuration_and_tilesize():
    lib = X.lib()
    assert b"sm_100a" in lib.xkblas_get_configuration()
    ctx = lib.xkblas_context_get()
    # reference blas/xkblas.c:2494-2505 with one GPU: 16384 > 4096 -> 8192
    assert lib.xkblas_auto_tilesize(ctx, 1, 16384, 16384, 16384) == 8192
    assert lib.xkblas_auto_tilesize(ctx, 1, 1024, 1024, 1024) == 1024
    assert lib.xkblas_auto_tilesize(ctx, 1, 100, 100, 100) == 512
    lib.xkblas_set_param(256, 8)
    assert lib.xkblas_get_param() == 256
    assert lib.xkblas_auto_tilesize(ctx, 1, 16384, 16384, 16384) == 256
    lib.xkblas_set_param(0, 8)


def _s(v, dt=np.float64):
    return np.array([v], dtype=dt)


def test_gemm_argument_codes():
    f = X.lib().xkblas_dgemm_async
    a = _s(1.0)
    b = _s(0.5)
    A = np.zeros(64)
    pa, pb, pA = a.ctypes.data, b.ctypes.data, A.ctypes.data
    N, T = X.CblasNoTrans, X.CblasTrans
    assert f(110, N, 4, 4, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -1
    assert f(N, 114, 4, 4, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -2
    assert f(N, N, -1, 4, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -3
    assert f(N, N, 4, -1, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -4
    assert f(N, N, 4, 4, -1, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -5
    assert f(N, N, 4, 4, 4, P(pa), P(pA), 3, P(pA), 4, P(pb), P(pA), 4) == -8
    assert f(T, N, 4, 4, 5, P(pa), P(pA), 4, P(pA), 5, P(pb), P(pA), 4) == -8
    assert f(N, N, 4, 4, 5, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == -10
    assert f(N, N, 4, 4, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 3) == -13
    # quick returns (reference blas/zgemm.c:184-189) need no device
    one = _s(1.0)
    zero = _s(0.0)
    assert f(N, N, 0, 4, 4, P(pa), P(pA), 4, P(pA), 4, P(pb), P(pA), 4) == 0
    assert f(N, N, 4, 4, 4, P(zero.ctypes.data), P(pA), 4, P(pA), 4, P(one.ctypes.data),
             P(pA), 4) == 0
    assert f(N, N, 4, 4, 0, P(pa), P(pA), 4, P(pA), 4, P(one.ctypes.data), P(pA), 4) == 0


def test_other_argument_codes():
    lib = X.lib()
    a = _s(1.0)
    A = np.zeros(64)
    pa, pA = P(a.ctypes.data), P(A.ctypes.data)
    L, U, N, T, C = X.CblasLower, X.CblasUpper, X.CblasNoTrans, X.CblasTrans, X.CblasConjTrans
    Lf, R, NU = X.CblasLeft, X.CblasRight, X.CblasNonUnit
    # trsm / trmm (reference blas/ztrsm.c:124-163)
    for f in (lib.xkblas_dtrsm_async, lib.xkblas_dtrmm_async):
        assert f(0, L, N, NU, 4, 4, pa, pA, 4, pA, 4) == -1
        assert f(Lf, 0, N, NU, 4, 4, pa, pA, 4, pA, 4) == -2
        assert f(Lf, L, 0, NU, 4, 4, pa, pA, 4, pA, 4) == -3
        assert f(Lf, L, N, 0, 4, 4, pa, pA, 4, pA, 4) == -4
        assert f(Lf, L, N, NU, -1, 4, pa, pA, 4, pA, 4) == -5
        assert f(Lf, L, N, NU, 4, -1, pa, pA, 4, pA, 4) == -6
        assert f(Lf, L, N, NU, 4, 4, pa, pA, 3, pA, 4) == -8
        assert f(R, L, N, NU, 4, 5, pa, pA, 4, pA, 4) == -8
        assert f(Lf, L, N, NU, 4, 4, pa, pA, 4, pA, 3) == -10
        assert f(Lf, L, N, NU, 0, 4, pa, pA, 4, pA, 4) == 0
    # syrk (reference blas/zsyrk.c:104-132): ConjTrans rejected
    f = lib.xkblas_dsyrk_async
    assert f(0, N, 4, 4, pa, pA, 4, pa, pA, 4) == -1
    assert f(L, C, 4, 4, pa, pA, 4, pa, pA, 4) == -2
    assert f(L, N, -1, 4, pa, pA, 4, pa, pA, 4) == -3
    assert f(L, N, 4, -1, pa, pA, 4, pa, pA, 4) == -4
    assert f(L, N, 4, 4, pa, pA, 3, pa, pA, 4) == -7
    assert f(L, N, 4, 4, pa, pA, 4, pa, pA, 3) == -10
    # herk: Trans rejected
    z = _s(1.0 + 0j, np.complex128)
    f = lib.xkblas_zherk_async
    assert f(L, T, 4, 4, pa, pA, 4, pa, pA, 4) == -2
    # syr2k / symm
    assert lib.xkblas_dsyr2k_async(L, N, 4, 4, pa, pA, 4, pA, 3, pa, pA, 4) == -9
    assert lib.xkblas_dsyr2k_async(L, N, 4, 4, pa, pA, 4, pA, 4, pa, pA, 3) == -12
    assert lib.xkblas_dsymm_async(0, L, 4, 4, pa, pA, 4, pA, 4, pa, pA, 4) == -1
    assert lib.xkblas_dsymm_async(Lf, 0, 4, 4, pa, pA, 4, pA, 4, pa, pA, 4) == -2
    assert lib.xkblas_dsymm_async(R, L, 4, 5, pa, pA, 4, pA, 4, pa, pA, 4) == -7
    assert lib.xkblas_zhemm_async(Lf, L, 4, 4, P(z.ctypes.data), pA, 4, pA, 3, P(z.ctypes.data),
                                  pA, 4) == -9
    # gemmt (reference blas/zgemmt.c:123-160)
    assert lib.xkblas_dgemmt_async(L, 0, N, 4, 4, pa, pA, 4, pA, 4, pa, pA, 4) == -1
    assert lib.xkblas_dgemmt_async(L, N, 0, 4, 4, pa, pA, 4, pA, 4, pa, pA, 4) == -2
    assert lib.xkblas_dgemmt_async(L, N, N, -1, 4, pa, pA, 4, pA, 4, pa, pA, 4) == -4
    assert lib.xkblas_dgemmt_async(L, N, N, 4, 4, pa, pA, 4, pA, 4, pa, pA, 3) == -13


def test_no_device_reports_enodev_not_fallback():
    """Without a GPU a valid call fails with ENODEV: there is no CPU path."""
    import errno
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    a = _s(1.0)
    A = np.ones(16)
    C = np.zeros(16)
    pa, pA, pC = P(a.ctypes.data), P(A.ctypes.data), P(C.ctypes.data)
    r = X.lib().xkblas_dgemm_async(X.CblasNoTrans, X.CblasNoTrans, 4, 4, 4, pa, pA, 4, pA, 4,
                                   pa, pC, 4)
    assert r == errno.ENODEV
    assert np.all(C == 0)


def test_cuda_abi_rejects_bad_arguments_without_device():
    """The thin CUDA ABI checks its arguments before touching a device, so
    these codes are the same with or without a GPU."""
    lib = X.lib()
    EINVAL, ERANGE = -1, -6
    one = (ctypes.c_double * 2)(1.0, 0.0)
    dp = ctypes.cast(one, ctypes.POINTER(ctypes.c_double))
    # gemm: null record, negative size, unknown element type / op code
    assert lib.xkb_cuda_gemm(None, None) == EINVAL
    g = X.GemmArgs(1, 0, 0, -1, 4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_gemm(ctypes.byref(g), None) == EINVAL
    g = X.GemmArgs(7, 0, 0, 4, 4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_gemm(ctypes.byref(g), None) == EINVAL
    g = X.GemmArgs(1, 3, 0, 4, 4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_gemm(ctypes.byref(g), None) == EINVAL
    # Ozaki: real or complex double only; sizes checked
    g = X.GemmArgs(0, 0, 0, 4, 4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g), 0, None) == EINVAL
    g = X.GemmArgs(1, 0, 0, 4, -4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g), 0, None) == EINVAL
    # the scratch-free form: beyond its fixed array, or not real double
    g = X.GemmArgs(1, 0, 0, 4, 4, 513, 16, 4, 16, 513, 16, 4)
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == ERANGE
    g = X.GemmArgs(3, 0, 0, 4, 4, 4, 16, 4, 16, 4, 16, 4)
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == EINVAL
    # trsm / trmm / symm / scale
    assert lib.xkb_cuda_trsm(1, 0, 1, 0, 0, -1, 4, dp, 16, 4, 16, 4, 0, None) == EINVAL
    assert lib.xkb_cuda_trsm(1, 0, 1, 5, 0, 4, 4, dp, 16, 4, 16, 4, 0, None) == EINVAL
    assert lib.xkb_cuda_trsm(1, 0, 1, 0, 0, 4, 4, None, 16, 4, 16, 4, 0, None) == EINVAL
    assert lib.xkb_cuda_trmm(9, 0, 1, 0, 0, 4, 4, dp, 16, 4, 16, 4, 0, None) == EINVAL
    assert lib.xkb_cuda_symm(1, 0, 0, 1, 4, -2, dp, 16, 4, 16, 4, dp, 16, 4, 0, None) == EINVAL
    assert lib.xkb_cuda_scale(1, 4, 4, None, 16, 4, 0, 0, 0, None) == EINVAL
    # batch: null list or negative count; an empty list is a no-op
    assert lib.xkb_cuda_batch(None, 3, 0, None) == EINVAL
    ops = (X.BatchOp * 1)()
    assert lib.xkb_cuda_batch(ops, -1, 0, None) == EINVAL
    assert lib.xkb_cuda_batch(ops, 0, 0, None) == 0
    # zero-sized products are no-ops that never reach the device
    g = X.GemmArgs(1, 0, 0, 0, 4, 4, 16, 1, 16, 4, 16, 1)
    assert lib.xkb_cuda_gemm(ctypes.byref(g), None) == 0
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g), 0, None) == 0
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == 0



def test_tuning_table_load_and_lookup(tmp_path):
    """The autotuner's table: a file of "key value" lines is loaded, values
    are read back, and the moduli-count bands drive xkb_ozaki_default_moduli
    (host-only logic, no device needed)."""
    lib = X.lib()
    lib.xkb_tune_clear()
    k16384 = lib.xkb_ozaki_default_moduli(16384)
    assert k16384 == 16  # built-in rule: H - log2(K)/2 >= 53
    f = tmp_path / "tune.txt"
    f.write_text("# measured on a B200\n"
                 "ozaki_moduli_k<=4096 13\n"
                 "ozaki_moduli_k<=32768 15   # a comment\n"
                 "batch_schedule 1\n"
                 "not a number line\n")
    assert lib.xkb_tune_load(str(f).encode()) == 3
    assert lib.xkb_tune_get(b"batch_schedule", 0.0) == 1.0
    assert lib.xkb_tune_get(b"missing_key", 7.5) == 7.5
    assert lib.xkb_ozaki_default_moduli(1000) == 13
    assert lib.xkb_ozaki_default_moduli(4096) == 13
    assert lib.xkb_ozaki_default_moduli(16384) == 15
    assert lib.xkb_ozaki_default_moduli(65536) == 16  # no band covers it: the K rule
    lib.xkb_tune_clear()
    assert lib.xkb_ozaki_default_moduli(16384) == k16384
    assert lib.xkb_tune_load(b"/nonexistent/tune.txt") == -1
