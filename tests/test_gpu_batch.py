"""The persistent tile-task executor (xkb_cuda_batch): mixed batches of
DGEMM / ZGEMM / left DTRSM / ZTRSM calls in one launch, each call checked
against an FP64 reference of the same operation (torch on the device is the
comparator here; the oracle covers the same operations elsewhere).
Requires a B200."""
import ctypes

import numpy as np
import pytest

import xkblas_b200 as X

pytestmark = pytest.mark.gpu

N_, T_, C_ = 0, 1, 2
LO, UP = 1, 2


def _op(M, opc):
    return M if opc == N_ else (M.transpose(0, 1) if opc == T_ else M.transpose(0, 1).conj())


@pytest.mark.parametrize("schedule", [0, 1])
def test_mixed_batch(xk, schedule):
    import torch
    rng = np.random.default_rng(7)
    gen = torch.Generator(device="cuda").manual_seed(11)
    ops, refs, keep, hold = [], [], [], []

    def rnd(r, c, cplx):
        if cplx:
            return torch.complex(torch.rand(c, r, generator=gen, device="cuda", dtype=torch.float64) - 0.5,
                                 torch.rand(c, r, generator=gen, device="cuda", dtype=torch.float64) - 0.5)
        return torch.rand(c, r, generator=gen, device="cuda", dtype=torch.float64) - 0.5

    # tensors are stored transposed: torch (cols, rows) row-major == (rows, cols) column-major
    for i in range(40):
        kind = rng.choice(["dgemm", "zgemm", "dtrsm", "ztrsm"], p=[0.5, 0.2, 0.2, 0.1])
        cplx = kind[0] == "z"
        M, N, K = (int(x) for x in rng.integers(1, 300, 3))
        o = X.BatchOp()
        o.dtype = 3 if cplx else 1
        if kind.endswith("gemm"):
            opA = int(rng.integers(0, 3 if cplx else 2))
            opB = int(rng.integers(0, 3 if cplx else 2))
            A = rnd(M, K, cplx) if opA == N_ else rnd(K, M, cplx)
            B = rnd(K, N, cplx) if opB == N_ else rnd(N, K, cplx)
            C = rnd(M, N, cplx)
            al = complex(1.5, -0.25) if cplx else 1.5
            be = complex(-0.5, 0.125) if cplx else -0.5
            Acm, Bcm, Ccm = A.t(), B.t(), C.t()
            ref = al * (_op(Acm, opA) @ _op(Bcm, opB)) + be * Ccm
            o.kind, o.opA, o.opB, o.M, o.N, o.K = 0, opA, opB, M, N, K
            o.A, o.lda = A.data_ptr(), A.shape[1]
            o.B, o.ldb = B.data_ptr(), B.shape[1]
            o.C, o.ldc = C.data_ptr(), M
            o.alpha[0], o.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
            o.beta[0], o.beta[1] = (be.real, be.imag) if cplx else (be, 0.0)
            out = C
            hold.append(B)  # every operand must outlive the batch (allocator reuse)
        else:
            uplo = int(rng.choice([LO, UP]))
            trans = int(rng.integers(0, 3 if cplx else 2))
            diag = int(rng.integers(0, 2))
            A = rnd(M, M, cplx) / M + torch.eye(M, device="cuda", dtype=A_dtype(cplx))
            Bm = rnd(M, N, cplx)
            Acm = A.t()
            tri = torch.tril(Acm) if uplo == LO else torch.triu(Acm)
            if diag:
                tri = tri - torch.diag(torch.diag(tri)) + torch.eye(M, device="cuda", dtype=tri.dtype)
            al = complex(2.0, 0.5) if cplx else 2.0
            ref = torch.linalg.solve(_op(tri, trans), al * Bm.t())
            o.kind, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 0, uplo, trans, diag, M, N
            o.A, o.lda = A.data_ptr(), M
            o.C, o.ldc = Bm.data_ptr(), M
            o.alpha[0], o.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
            out = Bm
        ops.append(o)
        refs.append(ref)
        keep.append((A, out))
    arr = (X.BatchOp * len(ops))(*ops)
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(arr, len(ops), schedule, None) == 0
    xk.sync()
    lat = (ctypes.c_double * len(ops))()
    assert xk.lib().xkb_cuda_batch_latency(lat, len(ops)) == 0
    assert xk.lib().xkb_cuda_take_device_error() == 0
    for i, (ref, (A, out)) in enumerate(zip(refs, keep)):
        got = out.t()
        err = (got - ref).abs().max().item()
        scale = max(ref.abs().max().item(), 1.0)
        assert err <= 1e-11 * scale, (i, ops[i].kind, err)
    assert all(v > 0 for v in lat)


def A_dtype(cplx):
    import torch
    return torch.complex128 if cplx else torch.float64


def test_batch_trsm_large_chain(xk):
    """One 1000 x 700 left-lower solve: a long dependency chain of 16 steps."""
    import torch
    M, N = 1000, 700
    g = torch.Generator(device="cuda").manual_seed(3)
    L = torch.tril(torch.rand(M, M, generator=g, device="cuda", dtype=torch.float64) - 0.5) \
        + M * torch.eye(M, device="cuda", dtype=torch.float64)
    A = L.t().contiguous()  # column-major storage of the lower triangular L
    B0 = torch.rand(N, M, generator=g, device="cuda", dtype=torch.float64) - 0.5
    B = B0.clone()
    o = X.BatchOp()
    o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, LO, N_, 0, M, N
    o.A, o.lda, o.C, o.ldc = A.data_ptr(), M, B.data_ptr(), M
    o.alpha[0] = 2.0
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(ctypes.byref(o), 1, 0, None) == 0
    xk.sync()
    assert xk.lib().xkb_cuda_take_device_error() == 0
    res = (L @ B.t() - 2.0 * B0.t()).abs().max().item()
    assert res < 1e-10


def test_batch_ztrsm_multiblock(xk):
    """Complex solves span several 64-row blocks: their trailing updates are
    split into 32-row tasks (the complex tile height)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    ops, keep = [], []
    for (M, N, uplo, trans) in ((253, 182, UP, T_), (130, 70, LO, C_), (200, 65, LO, N_)):
        L = torch.complex(torch.rand(M, M, generator=g, device="cuda", dtype=torch.float64),
                          torch.rand(M, M, generator=g, device="cuda", dtype=torch.float64)) / M
        L = L + torch.eye(M, device="cuda", dtype=torch.complex128)
        A = L.t().contiguous()  # column-major storage of L
        B0 = torch.complex(torch.rand(N, M, generator=g, device="cuda", dtype=torch.float64),
                           torch.rand(N, M, generator=g, device="cuda", dtype=torch.float64))
        B = B0.clone()
        o = X.BatchOp()
        o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 3, 0, uplo, trans, 0, M, N
        o.A, o.lda, o.C, o.ldc = A.data_ptr(), M, B.data_ptr(), M
        o.alpha[0], o.alpha[1] = 1.0, -1.0
        ops.append(o)
        tri = torch.tril(L) if uplo == LO else torch.triu(L)
        keep.append((A, B, B0, _op(tri, trans)))
    arr = (X.BatchOp * len(ops))(*ops)
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(arr, len(ops), 1, None) == 0
    xk.sync()
    assert xk.lib().xkb_cuda_take_device_error() == 0
    for A, B, B0, opT in keep:
        res = (opT @ B.t() - complex(1.0, -1.0) * B0.t()).abs().max().item()
        assert res < 1e-12


def test_repeated_batch_replays_a_graph(xk):
    """The same op list three times: the second submission is kept as a CUDA
    graph and the third replays it; inputs changed between submissions are
    read afresh (the graph holds the task list, not the data)."""
    import torch
    lib = xk.lib()
    assert lib.xkb_cuda_batch_release() == 0
    g = torch.Generator(device="cuda").manual_seed(9)
    ops, mats = [], []
    for (M, N, K) in ((200, 130, 77), (64, 300, 129), (513, 65, 40)):
        A = torch.rand(K, M, generator=g, device="cuda", dtype=torch.float64) - 0.5
        B = torch.rand(N, K, generator=g, device="cuda", dtype=torch.float64) - 0.5
        C = torch.zeros(N, M, device="cuda", dtype=torch.float64)
        o = X.BatchOp()
        o.kind, o.dtype, o.opA, o.opB, o.M, o.N, o.K = 0, 1, N_, N_, M, N, K
        o.A, o.lda, o.B, o.ldb, o.C, o.ldc = A.data_ptr(), M, B.data_ptr(), K, C.data_ptr(), M
        o.alpha[0] = 1.0
        ops.append(o)
        mats.append((A, B, C))
    M, N = 300, 150
    L = torch.tril(torch.rand(M, M, generator=g, device="cuda", dtype=torch.float64)) / M \
        + torch.eye(M, device="cuda", dtype=torch.float64)
    A = L.t().contiguous()
    Bt = torch.zeros(N, M, device="cuda", dtype=torch.float64)
    o = X.BatchOp()
    o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, LO, N_, 0, M, N
    o.A, o.lda, o.C, o.ldc = A.data_ptr(), M, Bt.data_ptr(), M
    o.alpha[0] = 1.0
    ops.append(o)
    arr = (X.BatchOp * len(ops))(*ops)
    for rep in range(3):
        for (Am, Bm, Cm) in mats:
            Bm.mul_(-1.0)  # new input values every submission
            Cm.zero_()
        B0 = torch.rand(N, M, generator=g, device="cuda", dtype=torch.float64)
        Bt.copy_(B0)
        torch.cuda.synchronize()
        assert lib.xkb_cuda_batch(arr, len(ops), 0, None) == 0
        torch.cuda.synchronize()
        assert lib.xkb_cuda_take_device_error() == 0
        for (Am, Bm, Cm) in mats:
            ref = Am.t() @ Bm.t()
            assert (Cm.t() - ref).abs().max().item() <= 1e-12 * max(ref.abs().max().item(), 1)
        res = (L @ Bt.t() - B0.t()).abs().max().item()
        assert res < 1e-12
        if rep >= 1:
            assert lib.xkb_cuda_batch_cached() >= 1
    lat = (ctypes.c_double * len(ops))()
    assert lib.xkb_cuda_batch_latency(lat, len(ops)) == 0
    assert all(v > 0 for v in lat)
    assert lib.xkb_cuda_batch_release() == 0
    assert lib.xkb_cuda_batch_cached() == 0
