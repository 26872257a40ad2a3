"""Trace export on the GPU: the CSV tables (the column layout of the
reference's trace converter, bin/ukilli.cpp:875-1115) describe the work the
library did -- the copies add up to the bytes it moved, kernels and copies
are ordered as the streams order them, each API call carries the reference's
call parameters (blas/zgemm.c:259-276, blas/ztrsm.c:220-236).  Requires a
B200."""
import csv
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

N_, LEFT, LO, NONUNIT = 111, 141, 122, 131
KERNELS = {"k_gemm_dmma", "k_repack", "k_scale", "k_sched", "k_sched(graph)", "k_trsm_block",
           "k_oz_norm+k_oz_shift", "k_oz_residues", "k_oz_gemm", "k_oz_gemm2", "k_oz_crt",
           "k_oz_crt_store", "k_tri_fill+k_copy2d", "k_sym_fill", "k_potrf_block",
           "k_getrf_block"}


def _rows(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


def _f(r, k):
    return float(r[k])


@pytest.fixture
def rec(xk, tmp_path):
    lib = xk.lib()
    scratch = tmp_path / "drain"
    scratch.mkdir()
    lib.xkblas_trace_record(0)
    assert lib.xkblas_trace_export(os.fsencode(str(scratch))) == 0  # events of earlier tests
    lib.xkblas_trace_record(1)
    yield lib
    lib.xkblas_trace_record(0)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _coherent(lib, a):
    m, n = a.shape
    assert lib.xkblas_memory_coherent_async(0, 0, m, n, _p(a), m, 8) == 0


def test_tables_describe_the_work(xk, rec, tmp_path):
    lib = rec
    n = 640
    A, B = O.plrnt(n, n, 1), O.plrnt(n, n, 2)
    C = np.asfortranarray(O.plrnt(n, n, 3))
    L = np.asfortranarray(np.tril(O.plrnt(n, n, 4)) + n * np.eye(n))
    X = np.asfortranarray(O.plrnt(n, n, 5))
    X0 = X.copy()
    al, be, one = np.array([1.5]), np.array([-0.5]), np.array([1.0])
    xk.reset_stats()
    assert lib.xkblas_dgemm_async(N_, N_, n, n, n, _p(al), _p(A), n, _p(B), n, _p(be), _p(C),
                                  n) == 0
    assert lib.xkblas_dtrsm_async(LEFT, LO, N_, NONUNIT, n, n, _p(one), _p(L), n, _p(X), n) == 0
    _coherent(lib, C)
    _coherent(lib, X)
    assert lib.xkblas_sync() == 0
    st = xk.stats()
    lib.xkblas_trace_record(0)
    assert lib.xkblas_trace_export(os.fsencode(str(tmp_path))) == 0
    assert lib.xkblas_trace_dropped() == 0
    assert np.abs(X - np.linalg.solve(L, X0)).max() < 1e-12

    kern = _rows(tmp_path / "kern.csv")
    cpy = _rows(tmp_path / "cpy.csv")
    calls = _rows(tmp_path / "call.csv")
    assert kern, "no kernel recorded"
    per_call = []
    for r in kern:
        call, _, kname = r["Name"].partition("/")
        assert call in ("dgemm", "dtrsm", "batch"), r["Name"]
        if re.fullmatch(r"(dgemm|zgemm|dtrsm|ztrsm)#\d+", kname):
            per_call.append(r)  # one call of an executor launch
        else:
            assert kname in KERNELS, r["Name"]
        assert r["Type"] == "CUDA" and r["Stream"] == "3"
        assert _f(r, "End") >= _f(r, "Start") >= _f(r, "Push") - 1e-3
        assert abs(_f(r, "Duration") - (_f(r, "End") - _f(r, "Start"))) < 1e-9
    # the two independent calls were queued and ran as one executor launch
    # (flushed by the first coherence call): one row per call inside it
    launches = [r for r in kern if r["Name"] in ("batch/k_sched", "batch/k_sched(graph)")]
    assert len(launches) == 1, [r["Name"] for r in kern]
    assert sorted(r["Name"] for r in per_call) == ["batch/dgemm#0", "batch/dtrsm#1"]
    k = launches[0]
    for r in per_call:
        assert r["Start"] == k["Start"]
        assert _f(r, "End") <= _f(k, "End") + 1e-4
    # the copies are exactly the bytes the directory moved
    h2d = [r for r in cpy if r["Dir"] == "1"]
    d2h = [r for r in cpy if r["Dir"] == "2"]
    assert sum(int(r["Size"]) for r in h2d) == st["h2d_bytes"]
    assert sum(int(r["Size"]) for r in d2h) == st["d2h_bytes"]
    assert all(r["Stream"] == "0" for r in h2d) and all(r["Stream"] == "1" for r in d2h)
    for r in cpy:
        assert _f(r, "End") >= _f(r, "Start")
    # stream order: results leave the device after the kernels that made them
    assert min(_f(r, "Start") for r in d2h) >= min(_f(r, "End") for r in kern) - 1e-4
    assert max(_f(r, "End") for r in d2h) >= max(_f(r, "End") for r in kern) - 1e-4
    # the calls, closed by the sync, with the reference's parameters
    assert [c["Name"] for c in calls] == ["dgemm", "dtrsm"]
    g, t = calls
    assert [int(g["Param%d" % i]) for i in (0, 1, 2, 4, 5)] == [n, n, n, N_, N_]
    assert [int(t["Param%d" % i]) for i in range(6)] == [n, n, LEFT, LO, N_, NONUNIT]
    assert (g["Level"], t["Level"]) == ("0", "1")
    for c in calls:
        assert _f(c, "End") >= _f(c, "Start")
        assert _f(c, "End") >= max(_f(r, "End") for r in cpy) - 1e-3  # sync waited for all
    tasks = _rows(tmp_path / "task.csv")
    assert [r["Name"] for r in tasks] == ["dgemm", "dtrsm"]
    par = _rows(tmp_path / "parallel.csv")
    assert {r["Type"] for r in par} == {"CPU", "CUDA"}


def test_tensor_op_kernels_named(xk, rec, tmp_path):
    lib = rec
    n = 512
    A, B = O.plrnt(n, n, 6), O.plrnt(n, n, 7)
    C = np.zeros((n, n), order="F")
    one, zero = np.array([1.0]), np.array([0.0])
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    try:
        assert lib.xkblas_dgemm_async(N_, N_, n, n, n, _p(one), _p(A), n, _p(B), n, _p(zero),
                                      _p(C), n) == 0
        _coherent(lib, C)
        assert lib.xkblas_sync() == 0
    finally:
        xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)
    lib.xkblas_trace_record(0)
    assert lib.xkblas_trace_export(os.fsencode(str(tmp_path))) == 0
    names = [r["Name"] for r in _rows(tmp_path / "kern.csv")]
    for k in ("dgemm/k_oz_residues", "dgemm/k_oz_gemm", "dgemm/k_oz_crt"):
        assert k in names, names
    assert np.abs(C - A @ B).max() <= 1e-12 * np.abs(A).sum(axis=1).max() * np.abs(B).max()


def test_trace_dir_env_writes_at_finalize(tmp_path):
    """XKBLAS_TRACE_DIR: recording from initialisation, tables written by the
    last xkblas_finalize (the reference's KAAPI_RECORD_TRACE workflow)."""
    out = tmp_path / "env"
    out.mkdir()
    code = (
        "import ctypes, numpy as np, xkblas_b200 as X\n"
        "L = X.lib(); X.init()\n"
        "n = 256; a = np.asfortranarray(np.random.default_rng(0).random((n, n)))\n"
        "c = np.zeros((n, n), order='F'); one = np.ones(1); z = np.zeros(1)\n"
        "p = lambda v: ctypes.c_void_p(v.ctypes.data)\n"
        "assert L.xkblas_dgemm_async(111, 111, n, n, n, p(one), p(a), n, p(a), n, p(z), p(c), n) == 0\n"
        "assert L.xkblas_memory_coherent_async(0, 0, n, n, p(c), n, 8) == 0\n"
        "assert L.xkblas_sync() == 0\n"
        "assert np.abs(c - a @ a).max() < 1e-10\n"
        "X.finalize()\n")
    env = dict(os.environ, XKBLAS_TRACE_DIR=str(out))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    kern = _rows(out / "kern.csv")
    cpy = _rows(out / "cpy.csv")
    calls = _rows(out / "call.csv")
    assert any(k["Name"].endswith("k_gemm_dmma") for k in kern), kern
    assert sum(int(c["Size"]) for c in cpy if c["Dir"] == "1") == 256 * 256 * 8
    assert sum(int(c["Size"]) for c in cpy if c["Dir"] == "2") == 256 * 256 * 8
    assert [c["Name"] for c in calls] == ["dgemm"]
