"""xkb_cuda_ozaki_gemm_noalloc: the Ozaki contraction for callers that cannot
allocate device memory at call time (its scratch is a fixed array inside the
library).  Checked through the C ABI against the pooled-scratch entry point
xkb_cuda_ozaki_gemm on the same device inputs, on two calls in a row.
Collected last on purpose (file name) so a run stopping at the first failure
has already run every other test.  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
from xkblas_b200 import GemmArgs  # xkb_gemm_args of include/xkb_cuda.h

pytestmark = pytest.mark.gpu


def _dev(X):
    import torch
    # column-major host matrix -> row-major device tensor of the transpose
    return torch.from_numpy(np.ascontiguousarray(X.T)).cuda()


@pytest.mark.parametrize("case", [(300, 200, 257, 0, 0), (512, 512, 512, 1, 0),
                                  (129, 511, 64, 0, 1)])
def test_noalloc_matches_pooled_entry_point(xk, case):
    import torch
    M, N, K, ta, tb = case
    lib = xk.lib()
    A = O.plrnt(M, K, 31) if ta == 0 else O.plrnt(K, M, 31)
    B = O.plrnt(K, N, 32) if tb == 0 else O.plrnt(N, K, 32)
    C0 = O.plrnt(M, N, 33)
    dA, dB = _dev(A), _dev(B)
    outs = {}
    for name, fn in (("pooled", lib.xkb_cuda_ozaki_gemm),
                     ("noalloc", lib.xkb_cuda_ozaki_gemm_noalloc)):
        res = []
        for _ in range(2):  # two calls in a row: the fixed array is reused
            dC = _dev(C0)
            torch.cuda.synchronize()
            g = GemmArgs(1, ta, tb, M, N, K, dA.data_ptr(), A.shape[0], dB.data_ptr(),
                         B.shape[0], dC.data_ptr(), M)
            g.alpha[0] = 1.5
            g.beta[0] = -0.5
            assert fn(ctypes.byref(g), 0, None) == 0
            xk.sync()
            res.append(np.asfortranarray(dC.cpu().numpy().T))
        outs[name] = res
    assert lib.xkb_cuda_take_device_error() == 0
    ref = outs["pooled"][0]
    scale = 1.5 * np.abs(A).max() * np.abs(B).max() * K + 0.5 * np.abs(C0).max()
    for C in outs["noalloc"] + outs["pooled"][1:]:
        # same tolerance as the other GEMM parity checks (a few eps of |A||B|K)
        assert np.abs(C - ref).max() <= 4 * 2.0 ** -53 * scale


def test_noalloc_refuses_sizes_beyond_its_array(xk):
    lib = xk.lib()
    g = GemmArgs(1, 0, 0, 513, 8, 8, 16, 513, 16, 8, 16, 513)  # pointers never used
    g.alpha[0] = 1.0
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == -6  # XKB_ERANGE
    g = GemmArgs(3, 0, 0, 8, 8, 8, 16, 8, 16, 8, 16, 8)  # complex: not offered
    assert lib.xkb_cuda_ozaki_gemm_noalloc(ctypes.byref(g), 0, None) == -1  # XKB_EINVAL
