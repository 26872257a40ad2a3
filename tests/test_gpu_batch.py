"""The persistent tile-task executor (xkb_cuda_batch): mixed batches of
DGEMM / ZGEMM / left DTRSM / ZTRSM calls in one launch, each call checked
against the CPU oracle (the reference's tile algorithms, blas/zgemm.c and
blas/ztrsm.c, restated in oracle/) on the same seeded inputs, with the
reference test programs' bounds (tests/checks.py).  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
import xkblas_b200 as X
from tests import checks

pytestmark = pytest.mark.gpu

# executor codes (include/xkb_cuda.h) and the oracle's CBLAS codes
N_, T_, C_ = 0, 1, 2
LO, UP = 1, 2
CBLAS_OP = {N_: O.NOTRANS, T_: O.TRANS, C_: O.CONJTRANS}
CBLAS_UPLO = {LO: O.LOWER, UP: O.UPPER}


def _dev(A):
    """Column-major host matrix -> device tensor holding the same layout (a
    row-major torch tensor of the transpose)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda()


def _host(T):
    return np.asfortranarray(T.cpu().numpy().T)


def _tri_matrix(M, seed, cplx):
    """A / M + I: the reference's well-conditioned triangular test matrix
    (testing/ztesting_trsm.c:130-134)."""
    return np.asfortranarray(O.plrnt(M, M, seed, cplx) / M + np.eye(M))


@pytest.mark.parametrize("schedule", [0, 1])
def test_mixed_batch(xk, schedule):
    import torch
    rng = np.random.default_rng(7)
    ops, cases = [], []
    seed = 1000
    for i in range(40):
        kind = rng.choice(["dgemm", "zgemm", "dtrsm", "ztrsm"], p=[0.5, 0.2, 0.2, 0.1])
        cplx = kind[0] == "z"
        M, N, K = (int(x) for x in rng.integers(1, 300, 3))
        o = X.BatchOp()
        o.dtype = 3 if cplx else 1
        if kind.endswith("gemm"):
            opA = int(rng.integers(0, 3 if cplx else 2))
            opB = int(rng.integers(0, 3 if cplx else 2))
            A = O.plrnt(M, K, seed, cplx) if opA == N_ else O.plrnt(K, M, seed, cplx)
            B = O.plrnt(K, N, seed + 1, cplx) if opB == N_ else O.plrnt(N, K, seed + 1, cplx)
            C0 = O.plrnt(M, N, seed + 2, cplx)
            seed += 3
            al = complex(1.5, -0.25) if cplx else 1.5
            be = complex(-0.5, 0.125) if cplx else -0.5
            dA, dB, dC = _dev(A), _dev(B), _dev(C0)
            o.kind, o.opA, o.opB, o.M, o.N, o.K = 0, opA, opB, M, N, K
            o.A, o.lda = dA.data_ptr(), A.shape[0]
            o.B, o.ldb = dB.data_ptr(), B.shape[0]
            o.C, o.ldc = dC.data_ptr(), M
            o.alpha[0], o.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
            o.beta[0], o.beta[1] = (be.real, be.imag) if cplx else (be, 0.0)
            cases.append(("gemm", (opA, opB, al, A, B, be, C0, K), (dA, dB, dC)))
        else:
            uplo = int(rng.choice([LO, UP]))
            trans = int(rng.integers(0, 3 if cplx else 2))
            diag = int(rng.integers(0, 2))
            A = _tri_matrix(M, seed, cplx)
            B0 = O.plrnt(M, N, seed + 1, cplx)
            seed += 2
            al = complex(2.0, 0.5) if cplx else 2.0
            dA, dB = _dev(A), _dev(B0)
            o.kind, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 0, uplo, trans, diag, M, N
            o.A, o.lda = dA.data_ptr(), M
            o.C, o.ldc = dB.data_ptr(), M
            o.alpha[0], o.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
            cases.append(("trsm", (uplo, trans, diag, al, A, B0), (dA, dB)))
        ops.append(o)
    arr = (X.BatchOp * len(ops))(*ops)
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(arr, len(ops), schedule, None) == 0
    xk.sync()
    lat = (ctypes.c_double * len(ops))()
    assert xk.lib().xkb_cuda_batch_latency(lat, len(ops)) == 0
    assert xk.lib().xkb_cuda_take_device_error() == 0
    for i, (kind, args, dev) in enumerate(cases):
        if kind == "gemm":
            opA, opB, al, A, B, be, C0, K = args
            R = O.gemm(CBLAS_OP[opA], CBLAS_OP[opB], al, A, B, be, C0.copy(order="F"), nb=64)
            r = checks.gemm_ratio(_host(dev[2]), R, A, B, C0, al, be, K)
            assert r <= 3.0, (i, kind, r)
        else:
            uplo, trans, diag, al, A, B0 = args
            R = O.trsm(O.LEFT, CBLAS_UPLO[uplo], CBLAS_OP[trans], O.UNIT if diag else O.NONUNIT,
                       al, A, B0.copy(order="F"), nb=64)
            r = checks.trsm_ratio(_host(dev[1]), R, A, *B0.shape)
            assert r <= 10, (i, kind, r)
    assert all(v > 0 for v in lat)


def test_batch_trsm_large_chain(xk):
    """One 1000 x 700 left-lower solve: a long dependency chain of 16 steps;
    A lower with U[-0.5, 0.5] entries and M added to the diagonal."""
    import torch
    M, N = 1000, 700
    A = np.asfortranarray(np.tril(O.plrnt(M, M, 3)) + M * np.eye(M))
    B0 = O.plrnt(M, N, 4)
    dA, dB = _dev(A), _dev(B0)
    o = X.BatchOp()
    o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, LO, N_, 0, M, N
    o.A, o.lda, o.C, o.ldc = dA.data_ptr(), M, dB.data_ptr(), M
    o.alpha[0] = 2.0
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(ctypes.byref(o), 1, 0, None) == 0
    xk.sync()
    assert xk.lib().xkb_cuda_take_device_error() == 0
    R = O.trsm(O.LEFT, O.LOWER, O.NOTRANS, O.NONUNIT, 2.0, A, B0.copy(order="F"), nb=64)
    assert checks.trsm_ratio(_host(dB), R, A, M, N) <= 10


def test_batch_ztrsm_multiblock(xk):
    """Complex solves span several 64-row blocks: their trailing updates are
    split into 32-row tasks (the complex tile height)."""
    import torch
    ops, keep = [], []
    seed = 50
    for (M, N, uplo, trans) in ((253, 182, UP, T_), (130, 70, LO, C_), (200, 65, LO, N_)):
        A = _tri_matrix(M, seed, True)
        B0 = O.plrnt(M, N, seed + 1, True)
        seed += 2
        dA, dB = _dev(A), _dev(B0)
        o = X.BatchOp()
        o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 3, 0, uplo, trans, 0, M, N
        o.A, o.lda, o.C, o.ldc = dA.data_ptr(), M, dB.data_ptr(), M
        o.alpha[0], o.alpha[1] = 1.0, -1.0
        ops.append(o)
        keep.append((uplo, trans, A, B0, dA, dB))
    arr = (X.BatchOp * len(ops))(*ops)
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_batch(arr, len(ops), 1, None) == 0
    xk.sync()
    assert xk.lib().xkb_cuda_take_device_error() == 0
    for uplo, trans, A, B0, dA, dB in keep:
        R = O.trsm(O.LEFT, CBLAS_UPLO[uplo], CBLAS_OP[trans], O.NONUNIT, 1.0 - 1.0j, A,
                   B0.copy(order="F"), nb=64)
        assert checks.trsm_ratio(_host(dB), R, A, *B0.shape) <= 10


def test_repeated_batch_replays_a_graph(xk):
    """The same op list three times: the second submission is kept as a CUDA
    graph and the third replays it; inputs changed between submissions are
    read afresh (the graph holds the task list, not the data)."""
    import torch
    lib = xk.lib()
    assert lib.xkb_cuda_batch_release() == 0
    ops, mats = [], []
    seed = 70
    for (M, N, K) in ((200, 130, 77), (64, 300, 129), (513, 65, 40)):
        A, B = O.plrnt(M, K, seed), O.plrnt(K, N, seed + 1)
        seed += 2
        dA, dB = _dev(A), _dev(B)
        dC = torch.zeros(N, M, device="cuda", dtype=torch.float64)
        o = X.BatchOp()
        o.kind, o.dtype, o.opA, o.opB, o.M, o.N, o.K = 0, 1, N_, N_, M, N, K
        o.A, o.lda, o.B, o.ldb, o.C, o.ldc = dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M
        o.alpha[0] = 1.0
        ops.append(o)
        mats.append((A, B, dA, dB, dC))
    M, N = 300, 150
    L = np.asfortranarray(np.tril(_tri_matrix(M, 90, False)))
    dL = _dev(L)
    dBt = torch.zeros(N, M, device="cuda", dtype=torch.float64)
    o = X.BatchOp()
    o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, LO, N_, 0, M, N
    o.A, o.lda, o.C, o.ldc = dL.data_ptr(), M, dBt.data_ptr(), M
    o.alpha[0] = 1.0
    ops.append(o)
    arr = (X.BatchOp * len(ops))(*ops)
    for rep in range(3):
        for (A, B, dA, dB, dC) in mats:
            dB.mul_(-1.0)  # new input values every submission
            dC.zero_()
        B0 = O.plrnt(M, N, 100 + rep)
        dBt.copy_(_dev(B0))
        torch.cuda.synchronize()
        assert lib.xkb_cuda_batch(arr, len(ops), 0, None) == 0
        torch.cuda.synchronize()
        assert lib.xkb_cuda_take_device_error() == 0
        for (A, B, dA, dB, dC) in mats:
            Bs = _host(dB)  # the sign-flipped input this submission read
            C0 = np.zeros((A.shape[0], B.shape[1]), order="F")
            R = O.gemm(O.NOTRANS, O.NOTRANS, 1.0, A, Bs, 0.0, C0.copy(order="F"), nb=64)
            assert checks.gemm_ratio(_host(dC), R, A, Bs, C0, 1.0, 0.0, A.shape[1]) <= 3.0
        R = O.trsm(O.LEFT, O.LOWER, O.NOTRANS, O.NONUNIT, 1.0, L, B0.copy(order="F"), nb=64)
        assert checks.trsm_ratio(_host(dBt), R, L, M, N) <= 10
        if rep >= 1:
            assert lib.xkb_cuda_batch_cached() >= 1
    lat = (ctypes.c_double * len(ops))()
    assert lib.xkb_cuda_batch_latency(lat, len(ops)) == 0
    assert all(v > 0 for v in lat)
    assert lib.xkb_cuda_batch_release() == 0
    assert lib.xkb_cuda_batch_cached() == 0
