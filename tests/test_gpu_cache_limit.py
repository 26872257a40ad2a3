"""Device cache limit (reference: XKBLAS_CACHE_LIMIT, percent of device
memory, kaapi/kaapi_impl.c:311-316, kaapi_plugin_cuda.c:2306): beyond it the
least recently used matrices not used by the current call are evicted --
dirty tiles written back first, later uploads ordered after that copy -- and
results stay exact.  Run in a child process because the limit is read at
initialisation; XKBLAS_CACHE_LIMIT_MB (extension) gives a small absolute
limit so the case fits in a few hundred MB.  Requires a B200."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

CHILD = r"""
import ctypes, sys
import numpy as np
import xkblas_b200 as X
L = X.lib(); X.init()
n = 2048                                    # 32 MiB per matrix, limit 100 MiB
rng = np.random.default_rng(7)
A, B = (np.asfortranarray(rng.random((n, n)) - 0.5) for _ in range(2))
C, D, E, F = (np.zeros((n, n), order="F") for _ in range(4))
one, zero = np.ones(1), np.zeros(1)
p = lambda v: ctypes.c_void_p(v.ctypes.data)
def gemm(x, y, z):
    assert L.xkblas_dgemm_async(111, 111, n, n, n, p(one), p(x), n, p(y), n, p(zero), p(z), n) == 0
X.reset_stats()
gemm(A, B, C)    # A, B, C resident: 96 MiB
gemm(C, C, D)    # D does not fit: A (least recently used, clean) is evicted
gemm(D, B, E)    # E does not fit: C (dirty) is written back and evicted
gemm(C, A, F)    # C and A come back: C must hold the written-back product
for m in (C, D, E, F):
    assert L.xkblas_memory_coherent_async(0, 0, n, n, p(m), n, 8) == 0
assert L.xkblas_sync() == 0
st = X.stats()
Cr = A @ B; Dr = Cr @ Cr; Er = Dr @ B; Fr = Cr @ A
for got, ref in ((C, Cr), (D, Dr), (E, Er), (F, Fr)):
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, err
assert st["evictions"] >= 2, st
# A and C crossed the host link twice (B once; C, D, E, F are products)
assert st["h2d_bytes"] == 4 * n * n * 8, st
assert st["d2h_bytes"] == 4 * n * n * 8, st
print("ok", st["evictions"], st["h2d_bytes"], st["d2h_bytes"])
X.finalize()
"""


def test_lru_eviction_keeps_results_exact():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, XKBLAS_CACHE_LIMIT_MB="100", XKBLAS_BATCH="0")
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=root, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-3000:])
    assert r.stdout.startswith("ok"), r.stdout
