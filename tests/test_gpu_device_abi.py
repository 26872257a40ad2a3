"""The device-pointer ABI (include/xkb_cuda.h) on operands the TMA kernels
cannot load directly: odd leading dimensions and bases 8 bytes off a
16-byte boundary, as cuBLAS-style callers pass them.  Each call is checked
against an FP64 PyTorch reference of the same operation on the same device
data.  Requires a B200."""
import ctypes

import numpy as np
import pytest
from xkblas_b200 import GemmArgs  # xkb_gemm_args of include/xkb_cuda.h

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


def _mat(torch, rows, cols, ld, off, dt, g):
    """A rows x cols column-major matrix with leading dimension ld inside a
    flat buffer, starting `off` elements in; returns (buffer, pointer, view)."""
    real = torch.float64 if dt in (1, 3) else torch.float32
    n = off + ld * cols
    buf = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) - 0.5
    if dt in (2, 3):
        buf = torch.complex(buf, torch.rand(n, generator=g, device="cuda", dtype=torch.float64) - 0.5)
    buf = buf.to(torch.complex64 if dt == 2 else (real if dt in (0, 1) else torch.complex128))
    view = buf[off:off + ld * cols].view(cols, ld)[:, :rows].t()  # rows x cols logical
    return buf, buf.data_ptr() + off * buf.element_size(), view


def _op(X, op):
    return X if op == 0 else (X.t() if op == 1 else X.t().conj())


@pytest.mark.parametrize("dt", [0, 1, 2, 3])
@pytest.mark.parametrize("ops", [(0, 0), (1, 0), (0, 1), (2, 2)])
def test_gemm_unaligned_operands(xk, dt, ops):
    import torch
    opA, opB = ops
    if dt in (0, 1) and 2 in ops:
        pytest.skip("conjugate transpose is complex only")
    g = torch.Generator(device="cuda").manual_seed(100 + dt)
    M, N, K = 131, 77, 203
    ar, ac = (M, K) if opA == 0 else (K, M)
    br, bc = (K, N) if opB == 0 else (N, K)
    bufA, pA, A = _mat(torch, ar, ac, ar + 1, 1, dt, g)   # odd ld, base one element off
    bufB, pB, B = _mat(torch, br, bc, br + 3, 3, dt, g)
    bufC, pC, C = _mat(torch, M, N, M + 1, 1, dt, g)
    C0 = C.clone()
    ga = GemmArgs(dt, opA, opB, M, N, K, pA, ar + 1, pB, br + 3, pC, M + 1)
    ga.alpha[0], ga.alpha[1] = 1.25, (0.5 if dt >= 2 else 0.0)
    ga.beta[0], ga.beta[1] = -0.75, (0.25 if dt >= 2 else 0.0)
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_gemm(ctypes.byref(ga), None) == 0
    xk.sync()
    al = complex(ga.alpha[0], ga.alpha[1])
    be = complex(ga.beta[0], ga.beta[1])
    hi = torch.complex128 if dt >= 2 else torch.float64
    ref = (al if dt >= 2 else al.real) * (_op(A.to(hi), opA) @ _op(B.to(hi), opB)) \
        + (be if dt >= 2 else be.real) * C0.to(hi)
    err = (C.to(hi) - ref).abs().max().item()
    scale = (A.abs().max() * B.abs().max()).item() * K * abs(al) + abs(be) * C0.abs().max().item()
    # single precision types: inputs and C are fp32, the product is formed in fp64
    tol = (4 * EPS if dt in (1, 3) else 2.0 ** -23) * scale
    assert err <= tol, (err, tol)
    assert xk.lib().xkb_cuda_take_device_error() == 0


@pytest.mark.parametrize("uplo,trans", [(1, 0), (2, 1)])
def test_trsm_unaligned(xk, uplo, trans):
    import torch
    g = torch.Generator(device="cuda").manual_seed(7 + uplo)
    M, N = 193, 71
    bufA, pA, A = _mat(torch, M, M, M + 1, 1, 1, g)
    A.mul_(1.0 / M)
    A.add_(torch.eye(M, device="cuda", dtype=torch.float64))
    bufB, pB, B = _mat(torch, M, N, M + 2, 1, 1, g)
    B0 = B.clone()
    al = (ctypes.c_double * 2)(2.0, 0.0)
    torch.cuda.synchronize()
    lib = xk.lib()
    assert lib.xkb_cuda_trsm(1, 0, uplo, trans, 0, M, N, ctypes.cast(al, ctypes.POINTER(ctypes.c_double)),
                             pA, M + 1, pB, M + 2, 0, None) == 0
    xk.sync()
    T = torch.tril(A) if uplo == 1 else torch.triu(A)
    res = (_op(T, trans) @ B - 2.0 * B0).abs().max().item()
    assert res <= 64 * EPS * M * (1 + B0.abs().max().item())
    assert lib.xkb_cuda_take_device_error() == 0


@pytest.mark.parametrize("dt", [1, 3])
@pytest.mark.parametrize("side,uplo,trans", [(0, 1, 0), (0, 2, 1), (1, 2, 0), (1, 1, 2)])
def test_trsm_many_rhs_halves(xk, dt, side, uplo, trans):
    """2113 right-hand sides (at least 2048: solved as two concurrent halves,
    1088 + 1025) on both sides, both triangles, transposed, complex, with
    unaligned leading dimensions: the residual of op(T) X = alpha B (left) /
    X op(T) = alpha B (right)."""
    import torch
    if dt == 1 and trans == 2:
        pytest.skip("conjugate transpose is complex only")
    g = torch.Generator(device="cuda").manual_seed(300 + 10 * side + uplo + dt)
    na, nrhs = 200, 2113
    M, N = (na, nrhs) if side == 0 else (nrhs, na)
    bufA, pA, A = _mat(torch, na, na, na + 1, 1, dt, g)
    A.mul_(1.0 / na)
    A.add_(torch.eye(na, device="cuda", dtype=A.dtype))
    bufB, pB, B = _mat(torch, M, N, M + 2, 1, dt, g)
    B0 = B.clone()
    al = (ctypes.c_double * 2)(2.0, 0.0)
    torch.cuda.synchronize()
    lib = xk.lib()
    assert lib.xkb_cuda_trsm(dt, side, uplo, trans, 0, M, N,
                             ctypes.cast(al, ctypes.POINTER(ctypes.c_double)), pA, na + 1, pB,
                             M + 2, 0, None) == 0
    xk.sync()
    T = _op(torch.tril(A) if uplo == 1 else torch.triu(A), trans)
    lhs = T @ B if side == 0 else B @ T
    res = (lhs - 2.0 * B0).abs().max().item()
    assert res <= 64 * EPS * na * (1 + B0.abs().max().item()), res
    assert lib.xkb_cuda_take_device_error() == 0


def test_ozaki_unaligned(xk):
    import torch
    g = torch.Generator(device="cuda").manual_seed(42)
    M, N, K = 150, 97, 301
    bufA, pA, A = _mat(torch, M, K, M + 1, 1, 1, g)
    bufB, pB, B = _mat(torch, K, N, K + 2, 1, 1, g)
    bufC, pC, C = _mat(torch, M, N, M + 3, 1, 1, g)
    C0 = C.clone()
    ga = GemmArgs(1, 0, 0, M, N, K, pA, M + 1, pB, K + 2, pC, M + 3)
    ga.alpha[0], ga.beta[0] = 1.5, -0.5
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, None) == 0
    xk.sync()
    ref = 1.5 * (A @ B) - 0.5 * C0
    scale = 1.5 * A.abs().max().item() * B.abs().max().item() * K + 0.5
    assert (C - ref).abs().max().item() <= 4 * EPS * scale
    assert xk.lib().xkb_cuda_take_device_error() == 0


def test_ozaki_panels_ragged(xk):
    """xkb_cuda_ozaki_gemm_panels with ragged column panels (widths 256, 44,
    700) and no events, on unaligned operands; bad boundaries are EINVAL."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(43)
    M, N, K = 300, 1000, 700
    bufA, pA, A = _mat(torch, M, K, M + 1, 1, 1, g)
    bufB, pB, B = _mat(torch, K, N, K + 2, 1, 1, g)
    bufC, pC, C = _mat(torch, M, N, M + 3, 1, 1, g)
    C0 = C.clone()
    ga = GemmArgs(1, 0, 0, M, N, K, pA, M + 1, pB, K + 2, pC, M + 3)
    ga.alpha[0], ga.beta[0] = 1.5, -0.5
    lib = xk.lib()
    bounds = (ctypes.c_long * 4)(0, 256, 300, N)
    torch.cuda.synchronize()
    assert lib.xkb_cuda_ozaki_gemm_panels(ctypes.byref(ga), 0, None, 3, bounds, None, None) == 0
    xk.sync()
    ref = 1.5 * (A @ B) - 0.5 * C0
    scale = 1.5 * A.abs().max().item() * B.abs().max().item() * K + 0.5
    assert (C - ref).abs().max().item() <= 4 * EPS * scale
    bad = (ctypes.c_long * 3)(0, 600, 500)
    assert lib.xkb_cuda_ozaki_gemm_panels(ctypes.byref(ga), 0, None, 2, bad, None, None) != 0
    assert lib.xkb_cuda_take_device_error() == 0


@pytest.mark.parametrize("opA", [0, 1])
def test_ozaki_blocks_match_panels(xk, opA):
    """xkb_cuda_ozaki_gemm_blocks (row blocks of op(A), column panels of
    op(B), several landing orders, no events, unaligned operands) gives
    bit for bit the column-panel form's result with the same moduli count;
    badly placed bounds and out-of-order landings are EINVAL."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(47)
    M, N, K = 700, 1100, 500
    ar, ac = (M, K) if opA == 0 else (K, M)
    bufA, pA, A = _mat(torch, ar, ac, ar + 1, 1, 1, g)
    bufB, pB, B = _mat(torch, K, N, K + 2, 1, 1, g)
    bufC, pC, C = _mat(torch, M, N, M + 3, 1, 1, g)
    C0 = C.clone()
    lib = xk.lib()
    L = ctypes.c_long
    rb = (L * 4)(0, 256, 512, M)
    cb = (L * 4)(0, 256, 768, N)

    def args():
        ga = GemmArgs(1, opA, 0, M, N, K, pA, ar + 1, pB, K + 2, pC, M + 3)
        ga.alpha[0], ga.beta[0] = 1.5, -0.5
        return ga

    ga = args()
    torch.cuda.synchronize()
    assert lib.xkb_cuda_ozaki_gemm_panels(ctypes.byref(ga), 15, None, 3, cb, None, None) == 0
    xk.sync()
    want = C.clone()
    opAm = A if opA == 0 else A.t()
    ref = 1.5 * (opAm @ B) - 0.5 * C0
    scale = 1.5 * A.abs().max().item() * B.abs().max().item() * K + 0.5
    assert (want - ref).abs().max().item() <= 4 * EPS * scale
    for order in ([-1, -2, -3, 0, 1, 2], [0, 1, 2, -1, -2, -3], [-1, 0, -2, 1, 2, -3]):
        C.copy_(C0)
        seq = (ctypes.c_int * 6)(*order)
        torch.cuda.synchronize()
        assert lib.xkb_cuda_ozaki_gemm_blocks(ctypes.byref(ga), 15, None, 3, rb, 3, cb, seq,
                                              None, None, None) == 0
        xk.sync()
        assert torch.equal(C, want), order
    ok = (ctypes.c_int * 6)(-1, -2, -3, 0, 1, 2)
    bad_rb = (L * 4)(0, 300, 512, M)  # interior bound not a multiple of 256
    assert lib.xkb_cuda_ozaki_gemm_blocks(ctypes.byref(ga), 15, None, 3, bad_rb, 3, cb, ok,
                                          None, None, None) != 0
    swapped = (ctypes.c_int * 6)(-2, -1, -3, 0, 1, 2)  # row blocks out of order
    assert lib.xkb_cuda_ozaki_gemm_blocks(ctypes.byref(ga), 15, None, 3, rb, 3, cb, swapped,
                                          None, None, None) != 0
    twice = (ctypes.c_int * 6)(-1, -2, -2, 0, 1, 2)  # a block missing, another repeated
    assert lib.xkb_cuda_ozaki_gemm_blocks(ctypes.byref(ga), 15, None, 3, rb, 3, cb, twice,
                                          None, None, None) != 0
    assert lib.xkb_cuda_take_device_error() == 0
