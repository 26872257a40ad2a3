"""XKBLAS_VERBOSE / XKBLAS_PRECISION (reference blas/xkblas.c:1472-1497,
1578-1604, 1635-1700): the configuration is printed at xkblas_init, the
per-operation counts and flops at the last xkblas_finalize; an unknown
precision is reported, not fatal.  Fresh processes.  Requires a B200."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = """
import sys
sys.path.insert(0, %r)
import numpy as np
import xkblas_b200 as X
X.init()
A = np.asfortranarray(np.random.default_rng(1).random((96, 80)))
B = np.asfortranarray(np.random.default_rng(2).random((80, 64)))
C = np.zeros((96, 64), order="F")
X.gemm(X.CblasNoTrans, X.CblasNoTrans, 1.0, A, B, 0.0, C)
X.gemm(X.CblasNoTrans, X.CblasNoTrans, 1.0, A, B, 1.0, C)
L = np.asfortranarray(np.tril(np.random.default_rng(3).random((96, 96))) + 96 * np.eye(96))
X.trsm(X.CblasLeft, X.CblasLower, X.CblasNoTrans, X.CblasNonUnit, 1.0, L, C)
X.invalidate_caches()
X.finalize()
""" % ROOT


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, "-c", PROG], env=env, capture_output=True, text=True,
                          timeout=300)


def test_verbose_reports_configuration_and_statistics():
    r = _run({"XKBLAS_VERBOSE": "2", "XKBLAS_PRECISION": "real*8"})
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert out.count("[XKBlas info]") == 2
    assert "precision: 8 bytes" in out
    assert "[XKBlas stats]" in out
    lines = {l.split("]")[0].strip("\t ["): l for l in out.splitlines() if "count=" in l}
    assert "count=           2" in lines["dgemm"], out
    assert "count=           1" in lines["dtrsm"], out
    assert "count=           3" in lines["sum -->"], out
    # flops of the two DGEMMs: 2 * (2 M N K)
    flops = float(lines["dgemm"].split("flops=")[1])
    assert abs(flops - 2 * 2.0 * 96 * 64 * 80) < 1.0
    assert "ozaki: contractions=" in out


def test_quiet_by_default_and_unknown_precision_reported():
    r = _run({"XKBLAS_VERBOSE": "", "XKBLAS_PRECISION": "quad"})
    assert r.returncode == 0, r.stderr
    assert "[XKBlas" not in r.stdout
    assert "XKBLAS_PRECISION must be" in r.stderr
