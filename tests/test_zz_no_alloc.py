"""xkb_cuda_ozaki_gemm_noalloc: the Ozaki contraction for callers that cannot
allocate device memory at call time (a program whose free GPU memory is
already held by its own caching allocator, or a loop in which an allocation
must never stall or fail).  Its scratch is a fixed array inside the library.

Checked through the C ABI against the pooled-scratch entry point
xkb_cuda_ozaki_gemm on the same device inputs, on two calls in a row.  Both
run the same kernels on the same integer residues (the INT32 tensor-core
sums are exact and the reconstruction is the same code), so their outputs
must agree bit for bit.  Collected last on purpose (file name), so that a run
stopping at the first failure has already run every other test.  Requires a
B200."""
import ctypes
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle as O
from xkblas_b200 import GemmArgs  # xkb_gemm_args of include/xkb_cuda.h

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
XKB_LOWER, XKB_UPPER = 1, 2


def _dev(X):
    import torch
    # column-major host matrix -> row-major device tensor of the transpose
    return torch.from_numpy(np.ascontiguousarray(X.T)).cuda()


def _run_both(xk, M, N, K, ta, tb, A, B, C0, alpha=1.5, beta=-0.5, uplo=0, same=False):
    """Two calls of each entry point on fresh copies of C0; returns
    {name: [C after call 1, C after call 2]}."""
    import torch
    lib = xk.lib()
    dA = _dev(A)
    dB = dA if same else _dev(B)
    outs = {}
    for name, fn in (("pooled", lib.xkb_cuda_ozaki_gemm),
                     ("noalloc", lib.xkb_cuda_ozaki_gemm_noalloc)):
        res = []
        for _ in range(2):  # two calls in a row: the fixed array is reused
            dC = _dev(C0)
            torch.cuda.synchronize()
            g = GemmArgs(1, ta, tb, M, N, K, dA.data_ptr(), A.shape[0], dB.data_ptr(),
                         B.shape[0], dC.data_ptr(), M)
            g.alpha[0] = alpha
            g.beta[0] = beta
            g.uplo = uplo
            assert fn(ctypes.byref(g), 0, None) == 0
            xk.sync()
            res.append(np.asfortranarray(dC.cpu().numpy().T))
        outs[name] = res
    assert lib.xkb_cuda_take_device_error() == 0
    return outs


def _assert_identical(outs):
    ref = outs["pooled"][0]
    for C in outs["noalloc"] + outs["pooled"][1:]:
        assert np.array_equal(C, ref)


@pytest.mark.parametrize("case", [(300, 200, 257, 0, 0), (512, 512, 512, 1, 0),
                                  (129, 511, 64, 0, 1)])
def test_noalloc_matches_pooled_entry_point(xk, case):
    M, N, K, ta, tb = case
    A = O.plrnt(M, K, 31) if ta == 0 else O.plrnt(K, M, 31)
    B = O.plrnt(K, N, 32) if tb == 0 else O.plrnt(N, K, 32)
    C0 = O.plrnt(M, N, 33)
    outs = _run_both(xk, M, N, K, ta, tb, A, B, C0)
    _assert_identical(outs)
    # and both are the contraction the oracle computes (GEMM bound of the
    # reference's test, testing/ztesting_gemm.c:289-303)
    from tests.checks import gemm_ratio
    R = O.gemm(O.NOTRANS + ta, O.NOTRANS + tb, 1.5, A, B, -0.5, C0.copy(order="F"), nb=128)
    assert gemm_ratio(outs["noalloc"][1], R, A, B, C0, 1.5, -0.5, K) <= 3.0


@pytest.mark.parametrize("ta,tb", [(0, 1), (1, 0)])
def test_noalloc_same_operand_branch(xk, ta, tb):
    """C = A A^T (or A^T A) with A passed as both operands: one residue
    buffer serves both sides."""
    N, K = 384, 300
    A = O.plrnt(N, K, 34) if ta == 0 else O.plrnt(K, N, 34)
    C0 = O.plrnt(N, N, 35)
    outs = _run_both(xk, N, N, K, ta, tb, A, A, C0, same=True)
    _assert_identical(outs)


@pytest.mark.parametrize("uplo", [XKB_LOWER, XKB_UPPER])
def test_noalloc_triangle_mask(xk, uplo):
    """SYRK-shaped call (A A^T, one triangle written); the other triangle of
    C keeps its input values."""
    N, K = 448, 200
    A = O.plrnt(N, K, 36)
    C0 = O.plrnt(N, N, 37)
    outs = _run_both(xk, N, N, K, 0, 1, A, A, C0, alpha=1.0, beta=1.0, uplo=uplo, same=True)
    _assert_identical(outs)
    C = outs["noalloc"][1]
    off = np.triu(np.ones((N, N), bool), 1) if uplo == XKB_LOWER else np.tril(np.ones((N, N), bool), -1)
    assert np.array_equal(C[off], C0[off])


def test_noalloc_beta_only(xk):
    """alpha = 0: C <- beta C, no contraction."""
    M, N, K = 200, 120, 64
    A, B, C0 = O.plrnt(M, K, 38), O.plrnt(K, N, 39), O.plrnt(M, N, 40)
    outs = _run_both(xk, M, N, K, 0, 0, A, B, C0, alpha=0.0, beta=-0.5)
    _assert_identical(outs)
    assert np.array_equal(outs["noalloc"][0], -0.5 * C0)


def test_noalloc_refuses_sizes_beyond_its_array(xk):
    lib = xk.lib()
    g = GemmArgs(1, 0, 0, 513, 8, 8, 16, 513, 16, 8, 16, 513)  # pointers never used
    g.alpha[0] = 1.0
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == -6  # XKB_ERANGE
    g = GemmArgs(3, 0, 0, 8, 8, 8, 16, 8, 16, 8, 16, 8)  # complex: not offered
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == -1  # XKB_EINVAL


_EXHAUSTED = textwrap.dedent("""
    import ctypes, json, sys
    import numpy as np
    import torch
    sys.path.insert(0, %(root)r)
    import oracle as O
    import xkblas_b200 as X
    from xkblas_b200 import GemmArgs

    X.init()  # places the fixed array and the kernels of the path
    lib = X.lib()
    M, N, K = 256, 192, 320
    A, B, C0 = O.plrnt(M, K, 41), O.plrnt(K, N, 42), O.plrnt(M, N, 43)
    dev = lambda X_: torch.from_numpy(np.ascontiguousarray(X_.T)).cuda()
    dA, dB = dev(A), dev(B)
    outs = [dev(C0), dev(C0), dev(C0)]
    torch.cuda.synchronize()

    def args(dC):
        g = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
        g.alpha[0], g.beta[0] = 1.5, -0.5
        return g

    # hand (nearly) all free device memory to torch's caching allocator
    hog, chunk = [], 1 << 32
    while chunk >= (2 << 20):
        try:
            hog.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
        except torch.OutOfMemoryError:
            chunk //= 2
    left = torch.cuda.mem_get_info()[0]
    rc = [lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(args(outs[i])), 0, None)
          for i in range(2)]
    torch.cuda.synchronize()
    del hog
    torch.cuda.empty_cache()
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(args(outs[2])), 0, None) == 0
    torch.cuda.synchronize()
    assert lib.xkb_cuda_take_device_error() == 0
    same = [bool(torch.equal(outs[i], outs[2])) for i in range(2)]
    print("RESULT " + json.dumps({"left": left, "rc": rc, "same": same}))
""")


def test_noalloc_after_device_memory_is_taken():
    """Fresh process: xkblas_init, then a caching allocator takes (nearly)
    every free byte of device memory; the scratch-free entry point still runs,
    twice, and matches the pooled entry point bit for bit."""
    env = dict(os.environ)
    env.pop("CUDA_MODULE_LOADING", None)  # the default (lazy) module loading
    r = subprocess.run([sys.executable, "-c", _EXHAUSTED % {"root": ROOT}], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT ")][-1]
    res = json.loads(line[len("RESULT "):])
    assert res["left"] < 64 << 20, "memory was not exhausted: %d bytes left" % res["left"]
    assert res["rc"] == [0, 0]
    assert res["same"] == [True, True]
