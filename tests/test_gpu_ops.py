"""GPU parity: every level-3 entry point through the C ABI (host buffers,
reference calling sequence) against the CPU oracle on the same seeded
inputs, judged by the reference's own acceptance bounds (tests/checks.py)
and the task's PLASMA-style bound.  Requires a B200."""
import math

import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_, T_, C_ = 111, 112, 113
UP, LO = 121, 122
LEFT, RIGHT = 141, 142
NONUNIT, UNIT = 131, 132

UPCAST = {np.dtype(np.float32): np.float64, np.dtype(np.complex64): np.complex128,
          np.dtype(np.float64): np.float64, np.dtype(np.complex128): np.complex128}


def gen(M, N, seed, dt):
    cplx = np.issubdtype(dt, np.complexfloating)
    A = O.plrnt(M, N, seed, cplx)
    return np.asfortranarray(A.astype(dt))


def up(X):
    return np.asfortranarray(X.astype(UPCAST[np.dtype(X.dtype)]))


def scal(v, dt):
    return v if np.issubdtype(dt, np.complexfloating) else v.real if isinstance(v, complex) else v


GEMM_CASES = [
    # (M, N, K)
    (37, 29, 41), (130, 257, 65), (1, 1, 1), (64, 64, 64), (300, 200, 513),
]


@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32, np.complex64])
@pytest.mark.parametrize("mnk", GEMM_CASES)
def test_gemm_all_trans(xk, dt, mnk):
    M, N, K = mnk
    cplx = np.issubdtype(dt, np.complexfloating)
    ops = (N_, T_, C_) if cplx else (N_, T_)
    alpha = scal(1.5 - 0.25j, dt)
    beta = scal(-0.5 + 0.125j, dt)
    seed = 100
    for ta in ops:
        for tb in ops:
            A = gen(M, K, seed, dt) if ta == N_ else gen(K, M, seed, dt)
            B = gen(K, N, seed + 1, dt) if tb == N_ else gen(N, K, seed + 1, dt)
            C0 = gen(M, N, seed + 2, dt)
            seed += 3
            C = C0.copy(order="F")
            xk.gemm(ta, tb, alpha, A, B, beta, C)
            xk.invalidate_caches()
            R = O.gemm(ta, tb, alpha, up(A), up(B), beta, up(C0), nb=256)
            r = checks.gemm_ratio(C, R, A, B, C0, alpha, beta, K)
            assert r <= 3.0, (ta, tb, r)
            assert checks.plasma_ratio(C, R, A, B, alpha, K) < 10


def test_gemm_config1(xk):
    """DGEMM NN 1024^3, alpha=1.5, beta=-0.5, NB=256 (the reference's CPU-runnable case)."""
    M = N = K = 1024
    A, B, C0 = O.plrnt(M, K, 1), O.plrnt(K, N, 2), O.plrnt(M, N, 3)
    xk.set_param(256)
    try:
        C = C0.copy(order="F")
        xk.gemm(N_, N_, 1.5, A, B, -0.5, C)
        xk.invalidate_caches()
    finally:
        xk.set_param(0)
    R = O.gemm(N_, N_, 1.5, A, B, -0.5, C0.copy(order="F"), nb=256)
    assert checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, K) <= 3.0
    assert checks.plasma_ratio(C, R, A, B, 1.5, K) < 10
    # against the double-double oracle on a sample
    rows = np.arange(0, M, 61)
    cols = np.arange(0, N, 53)
    dd = O.gemm_dd(N_, N_, 1.5, A, B, -0.5, C0, rows, cols)
    err = np.abs(C[np.ix_(rows, cols)] - dd).max()
    scale = 1.5 * np.abs(A).sum(axis=1).max() * np.abs(B).sum(axis=0).max()
    assert err / (scale * 2.0 ** -53) < 4


def test_gemm_edge_cases(xk):
    M, N, K = 70, 45, 33
    A, B = O.plrnt(M, K, 7), O.plrnt(K, N, 8)
    # beta = 0: C is not read (NaN must not propagate)
    C = np.full((M, N), np.nan, order="F")
    xk.gemm(N_, N_, 2.0, A, B, 0.0, C)
    xk.invalidate_caches()
    np.testing.assert_allclose(C, 2.0 * A @ B, rtol=1e-13, atol=1e-13)
    # alpha = 0: C = beta*C, A and B not referenced (NaN inputs)
    An = np.full((M, K), np.nan, order="F")
    C0 = O.plrnt(M, N, 9)
    C = C0.copy(order="F")
    xk.gemm(N_, N_, 0.0, An, An.copy(order="F")[:K, :N].copy(order="F"), -3.0, C)
    xk.invalidate_caches()
    np.testing.assert_array_equal(C, -3.0 * C0)
    # K = 0: C = beta*C
    C = C0.copy(order="F")
    A0 = np.zeros((M, 1), order="F")
    B0 = np.zeros((1, N), order="F")
    r = xk.lib().xkblas_dgemm_async(N_, N_, M, N, 0, xk._ptr(xk._scal(1.0, np.float64)),
                                    xk._ptr(A0), M, xk._ptr(B0), 1,
                                    xk._ptr(xk._scal(0.5, np.float64)), xk._ptr(C), M)
    assert r == 0
    xk.coherent(C)
    xk.sync()
    xk.invalidate_caches()
    np.testing.assert_array_equal(C, 0.5 * C0)


def test_gemm_leading_dimensions_and_reuse(xk):
    """Sub-matrix views with ld > M, and the tile directory's reuse of A."""
    M, N, K = 100, 80, 60
    big = O.plrnt(160, 120, 11)
    A = np.asfortranarray(big[:M, :K])  # copy: contiguous with ld = M
    Bfull = O.plrnt(K + 7, N, 12)       # B is the first K rows: ld = K+7
    Cfull = O.plrnt(M + 3, N, 13)
    # call through raw pointers with explicit ld
    lib = xk.lib()
    C = Cfull.copy(order="F")
    alpha, beta = xk._scal(1.0, np.float64), xk._scal(1.0, np.float64)
    r = lib.xkblas_dgemm_async(N_, N_, M, N, K, xk._ptr(alpha), xk._ptr(A), M, xk._ptr(Bfull),
                               K + 7, xk._ptr(beta), xk._ptr(C), M + 3)
    assert r == 0
    lib.xkblas_memory_coherent_async(0, 0, M, N, xk._ptr(C), M + 3, 8)
    xk.sync()
    s0 = xk.stats()
    # second call with the same A: A's tiles are hits
    C2 = Cfull.copy(order="F")
    r = lib.xkblas_dgemm_async(N_, N_, M, N, K, xk._ptr(alpha), xk._ptr(A), M, xk._ptr(Bfull),
                               K + 7, xk._ptr(beta), xk._ptr(C2), M + 3)
    assert r == 0
    lib.xkblas_memory_coherent_async(0, 0, M, N, xk._ptr(C2), M + 3, 8)
    xk.sync()
    s1 = xk.stats()
    assert s1["tile_hits"] > s0["tile_hits"]
    xk.invalidate_caches()
    ref = A @ Bfull[:K] + Cfull[:M]
    np.testing.assert_allclose(C[:M], ref, rtol=1e-13, atol=1e-12)
    np.testing.assert_array_equal(C[M:], Cfull[M:])  # rows beyond M untouched
    np.testing.assert_allclose(C2[:M], ref, rtol=1e-13, atol=1e-12)


TRSM_DT = [np.float64, np.complex128, np.float32, np.complex64]


@pytest.mark.parametrize("dt", TRSM_DT)
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_trsm_all_cases(xk, dt, side, uplo):
    cplx = np.issubdtype(dt, np.complexfloating)
    M, N = 200, 150
    na = M if side == LEFT else N
    seed = 300
    for tr in ((N_, T_, C_) if cplx else (N_, T_)):
        for dg in (NONUNIT, UNIT):
            # reference testing/ztesting_trsm.c:130-134: A/max(M,N) + unit diagonal
            A = np.asfortranarray((O.plrnt(na, na, seed, cplx) / max(M, N)
                                   + np.eye(na)).astype(dt))
            B0 = gen(M, N, seed + 1, dt)
            seed += 2
            alpha = scal(2.0 + 0.5j, dt)
            B = B0.copy(order="F")
            xk.trsm(side, uplo, tr, dg, alpha, A, B)
            xk.invalidate_caches()
            R = O.trsm(side, uplo, tr, dg, alpha, up(A), up(B0), nb=64)
            r = checks.trsm_ratio(B, R, A, M, N)
            assert r <= 10, (tr, dg, r)


def test_trsm_config2_shape(xk):
    """DTRSM L/L/N/N with M added to the diagonal, alpha=2, NB=512 (4096 in the
    benchmark; 1024 here so the oracle finishes in seconds)."""
    M = N = 1024
    A = O.plrnt(M, M, 21)
    A = np.asfortranarray(np.tril(A) + M * np.eye(M))
    B0 = O.plrnt(M, N, 22)
    xk.set_param(512)
    try:
        B = B0.copy(order="F")
        xk.trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B)
        xk.invalidate_caches()
    finally:
        xk.set_param(0)
    R = O.trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B0.copy(order="F"), nb=512)
    assert checks.trsm_ratio(B, R, A, M, N) <= 10
    # residual: A X = 2 B0
    res = np.abs(A @ B - 2.0 * B0).max() / (np.abs(A).sum(1).max() * np.abs(B).max())
    assert res < 1e-14


@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32, np.complex64])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_syrk_herk(xk, dt, uplo):
    cplx = np.issubdtype(dt, np.complexfloating)
    N, K = 190, 130
    for herm in ((False, True) if cplx else (False,)):
        for tr in (N_, (C_ if herm else T_)):
            A = gen(N, K, 400, dt) if tr == N_ else gen(K, N, 400, dt)
            C0 = np.asfortranarray(O.plgsy(N, 401, cplx=cplx).astype(dt))
            C = C0.copy(order="F")
            xk.syrk(uplo, tr, 1.0, A, 1.0, C, herm=herm)
            xk.invalidate_caches()
            R = O.syrk(uplo, tr, 1.0, up(A), 1.0, up(C0), herm=herm)
            sel = np.tril if uplo == LO else np.triu
            other = np.triu if uplo == LO else np.tril
            assert checks.rk_ratio(sel(C), sel(R), A, C0, N) <= 10
            k = 1 if uplo == LO else -1  # strictly the other triangle
            np.testing.assert_array_equal(other(C, k), other(C0, k))  # untouched
            if herm:
                assert np.all(np.diag(C).imag == 0)


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_syr2k_her2k(xk, dt, uplo):
    cplx = np.issubdtype(dt, np.complexfloating)
    N, K = 150, 97
    for herm in ((False, True) if cplx else (False,)):
        for tr in (N_, (C_ if herm else T_)):
            A = gen(N, K, 500, dt) if tr == N_ else gen(K, N, 500, dt)
            B = gen(N, K, 501, dt) if tr == N_ else gen(K, N, 501, dt)
            C0 = np.asfortranarray(O.plgsy(N, 502, cplx=cplx).astype(dt))
            alpha = scal(0.75 + 0.5j, dt)
            beta = 0.5
            C = C0.copy(order="F")
            xk.syr2k(uplo, tr, alpha, A, B, beta, C, herm=herm)
            xk.invalidate_caches()
            R = O.syr2k(uplo, tr, alpha, up(A), up(B), beta, up(C0), herm=herm)
            sel = np.tril if uplo == LO else np.triu
            assert checks.rk_ratio(sel(C), sel(R), A, C0, N, checks.ninf(B)) <= 10


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_gemmt(xk, dt, uplo):
    N, K = 170, 90
    A, B, C0 = gen(N, K, 600, dt), gen(K, N, 601, dt), gen(N, N, 602, dt)
    C = C0.copy(order="F")
    xk.gemmt(uplo, N_, N_, 1.25, A, B, -1.0, C)
    xk.invalidate_caches()
    R = O.gemmt(uplo, N_, N_, 1.25, A, B, -1.0, C0.copy(order="F"))
    sel = np.tril if uplo == LO else np.triu
    assert checks.gemm_ratio(sel(C), sel(R), A, B, C0, 1.25, -1.0, K) <= 3
    other = np.triu if uplo == LO else np.tril
    k = 1 if uplo == LO else -1
    np.testing.assert_array_equal(other(C, k), other(C0, k))


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_symm_hemm(xk, dt, side, uplo):
    cplx = np.issubdtype(dt, np.complexfloating)
    M, N = 140, 110
    na = M if side == LEFT else N
    for herm in ((False, True) if cplx else (False,)):
        A = gen(na, na, 700, dt)
        B, C0 = gen(M, N, 701, dt), gen(M, N, 702, dt)
        alpha, beta = scal(1.5 + 0.5j, dt), scal(-0.5, dt)
        C = C0.copy(order="F")
        xk.symm(side, uplo, alpha, A, B, beta, C, herm=herm)
        xk.invalidate_caches()
        R = O.symm(side, uplo, alpha, up(A), up(B), beta, up(C0), herm=herm)
        den = (checks.ninf(A) + checks.ninf(B) + checks.ninf(C0)) * max(M, N) * 2.0 ** -53
        assert checks.ninf(C - R) / den <= 10


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
def test_trmm(xk, dt, side):
    cplx = np.issubdtype(dt, np.complexfloating)
    M, N = 120, 90
    na = M if side == LEFT else N
    for uplo in (UP, LO):
        for tr in ((N_, T_, C_) if cplx else (N_, T_)):
            for dg in (NONUNIT, UNIT):
                A = gen(na, na, 800, dt)
                B0 = gen(M, N, 801, dt)
                B = B0.copy(order="F")
                xk.trmm(side, uplo, tr, dg, 1.5, A, B)
                xk.invalidate_caches()
                R = O.trmm(side, uplo, tr, dg, 1.5, up(A), up(B0))
                assert checks.trsm_ratio(B, R, A, M, N) <= 10, (uplo, tr, dg)


def test_coherence_uplo_writeback(xk):
    """coherent_async(uplo) writes back only tiles touching that triangle."""
    N, K = 512, 64
    xk.set_param(128)
    try:
        A = O.plrnt(N, K, 900)
        C0 = O.plrnt(N, N, 901)
        C = C0.copy(order="F")
        lib = xk.lib()
        al = xk._scal(1.0, np.float64)
        r = lib.xkblas_dgemm_async(N_, T_, N, N, K, xk._ptr(al), xk._ptr(A), N, xk._ptr(A), N,
                                   xk._ptr(al), xk._ptr(C), N)
        assert r == 0
        lib.xkblas_memory_coherent_async(LO, 0, N, N, xk._ptr(C), N, 8)
        xk.sync()
        full = A @ A.T + C0
        # tiles strictly above the diagonal were not copied back
        for ti in range(4):
            for tj in range(4):
                blk = (slice(ti * 128, ti * 128 + 128), slice(tj * 128, tj * 128 + 128))
                if tj <= ti:
                    np.testing.assert_allclose(C[blk], full[blk], rtol=1e-13, atol=1e-12)
                else:
                    np.testing.assert_array_equal(C[blk], C0[blk])
        # the rest follows on a full coherence request
        lib.xkblas_memory_coherent_async(0, 0, N, N, xk._ptr(C), N, 8)
        xk.sync()
        np.testing.assert_allclose(C, full, rtol=1e-13, atol=1e-12)
        xk.invalidate_caches()
    finally:
        xk.set_param(0)


def test_coherence_memflag_drops_other_triangle(xk):
    """coherent_async(uplo, memflag = 1) writes back the uplo tiles and drops
    the device copies of the others (reference blas/xkblas.c:2016-2049): a
    later full coherence request copies nothing back for them, and the next
    call reads them from the host again."""
    N, K, nb = 512, 64, 128
    xk.set_param(nb)
    try:
        A = O.plrnt(N, K, 910)
        C0 = O.plrnt(N, N, 911)
        C = C0.copy(order="F")
        lib = xk.lib()
        one = xk._scal(1.0, np.float64)
        args = (N_, T_, N, N, K, xk._ptr(one), xk._ptr(A), N, xk._ptr(A), N, xk._ptr(one),
                xk._ptr(C), N)
        assert lib.xkblas_dgemm_async(*args) == 0
        assert lib.xkblas_memory_coherent_async(LO, 1, N, N, xk._ptr(C), N, 8) == 0
        xk.sync()
        G = A @ A.T
        # block-upper tiles (strictly above the diagonal tiles) were dropped
        tile_up = np.kron(np.triu(np.ones((N // nb, N // nb), bool), 1), np.ones((nb, nb), bool))
        np.testing.assert_allclose(C[~tile_up], (G + C0)[~tile_up], rtol=1e-13, atol=1e-12)
        np.testing.assert_array_equal(C[tile_up], C0[tile_up])
        # nothing of the dropped tiles comes back on a full request
        assert lib.xkblas_memory_coherent_async(0, 0, N, N, xk._ptr(C), N, 8) == 0
        xk.sync()
        np.testing.assert_array_equal(C[tile_up], C0[tile_up])
        # the next call reads the dropped tiles from the host again
        H = C.copy(order="F")
        assert lib.xkblas_dgemm_async(*args) == 0
        assert lib.xkblas_memory_coherent_async(0, 0, N, N, xk._ptr(C), N, 8) == 0
        xk.sync()
        np.testing.assert_allclose(C, G + H, rtol=1e-13, atol=1e-12)
        xk.invalidate_caches()
    finally:
        xk.set_param(0)


def test_async_chain_without_host_round_trip(xk):
    """C1 = A B; C2 = C1 B (C1 consumed on the device, never copied back in
    between); only C2 is made coherent."""
    n = 256
    A, B = O.plrnt(n, n, 31), O.plrnt(n, n, 32)
    C1 = np.zeros((n, n), order="F")
    C2 = np.zeros((n, n), order="F")
    lib = xk.lib()
    one, zero = xk._scal(1.0, np.float64), xk._scal(0.0, np.float64)
    assert lib.xkblas_dgemm_async(N_, N_, n, n, n, xk._ptr(one), xk._ptr(A), n, xk._ptr(B), n,
                                  xk._ptr(zero), xk._ptr(C1), n) == 0
    assert lib.xkblas_dgemm_async(N_, N_, n, n, n, xk._ptr(one), xk._ptr(C1), n, xk._ptr(B), n,
                                  xk._ptr(zero), xk._ptr(C2), n) == 0
    xk.coherent(C2)
    xk.sync()
    assert np.all(C1 == 0)  # never requested
    np.testing.assert_allclose(C2, (A @ B) @ B, rtol=1e-12, atol=1e-11)
    xk.invalidate_caches()


@pytest.mark.parametrize("mnk", [(1024, 1024, 128), (1024, 1024, 1024), (1536, 1024, 777),
                                 (640, 2048, 1000)])
def test_gemm_many_ctas_per_sm(xk, mnk):
    """Mid sizes run the 64x64 tile with several CTAs per SM: stage reuse
    under co-residency must stay exact (repeated to catch ordering races)."""
    M, N, K = mnk
    A, B = O.plrnt(M, K, 41), O.plrnt(K, N, 42)
    ref = 1.5 * (A @ B)
    for _ in range(3):
        C = np.zeros((M, N), order="F")
        xk.gemm(N_, N_, 1.5, A, B, 0.0, C)
        xk.invalidate_caches()
        err = np.abs(C - ref).max() / (1.5 * np.abs(A).max() * np.abs(B).max() * K)
        assert err < 1e-15, err


@pytest.mark.parametrize("case", [
    # (dtype, M, N, K, opA, opB, uplo): few output tiles, long K -> split-K
    (np.float64, 2048, 512, 2048, N_, N_, 0),
    (np.float64, 256, 256, 4096, T_, N_, 0),
    (np.float64, 300, 200, 2049, N_, T_, 0),
    (np.complex128, 320, 256, 3000, C_, N_, 0),
    (np.float64, 384, 384, 2048, N_, T_, LO),
    (np.complex128, 256, 256, 1500, N_, C_, UP),
])
def test_gemm_split_k(xk, case):
    """Too few 128 x 128 output tiles for the SMs: the k range of each tile
    is split across CTAs and the slices are summed in a fixed order.  Same
    bounds as every GEMM, the masked triangle only, and bit-identical
    results on repeated calls (deterministic reduction)."""
    import ctypes
    import torch
    from xkblas_b200 import GemmArgs
    dt, M, N, K, ta, tb, uplo = case
    cplx = dt == np.complex128
    A = gen(M, K, 50, dt) if ta == N_ else gen(K, M, 50, dt)
    B = gen(K, N, 51, dt) if tb == N_ else gen(N, K, 51, dt)
    C0 = gen(M, N, 52, dt)
    al, be = (1.5 - 0.25j, -0.5 + 0.125j) if cplx else (1.5, -0.5)
    dev = lambda X: torch.from_numpy(np.ascontiguousarray(X.T)).cuda()
    dA, dB = dev(A), dev(B)
    outs = []
    for _ in range(2):
        dC = dev(C0)
        g = GemmArgs(3 if cplx else 1, ta - N_, tb - N_, M, N, K, dA.data_ptr(), A.shape[0],
                     dB.data_ptr(), B.shape[0], dC.data_ptr(), M)
        g.alpha[0], g.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
        g.beta[0], g.beta[1] = (be.real, be.imag) if cplx else (be, 0.0)
        g.uplo = {0: 0, LO: 1, UP: 2}[uplo]
        torch.cuda.synchronize()
        k0 = xk.kernel_count()
        assert xk.lib().xkb_cuda_gemm(ctypes.byref(g), None) == 0
        assert xk.kernel_count() - k0 == 2  # the split product and its reduction
        xk.sync()
        outs.append(np.asfortranarray(dC.cpu().numpy().T))
    assert xk.lib().xkb_cuda_take_device_error() == 0
    assert np.array_equal(outs[0], outs[1])
    C = outs[0]
    R = O.gemm(ta, tb, al, A, B, be, C0.copy(order="F"), nb=256)
    if uplo:
        sel = np.tril if uplo == LO else np.triu
        other = np.triu if uplo == LO else np.tril
        k = 1 if uplo == LO else -1
        np.testing.assert_array_equal(other(C, k), other(C0, k))
        C, R = sel(C), sel(R)
    assert checks.gemm_ratio(C, R, A, B, C0, al, be, K) <= 3.0


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
def test_trsm_inverse_leaves(xk, dt, side):
    """More than one diagonal block (600 unknowns): with the tuning key
    trsm_inv_leaves = 1 (default) the blocks are inverted in one launch and
    applied as GEMMs; = 0 solves them by substitution.  Both meet the
    reference bound for every uplo / trans / diag case."""
    cplx = np.issubdtype(dt, np.complexfloating)
    lib = xk.lib()
    M, N = (600, 300) if side == LEFT else (300, 600)
    na = M if side == LEFT else N
    seed = 1300
    try:
        for flag in (1.0, 0.0):
            lib.xkb_tune_set(b"trsm_inv_leaves", flag)
            for uplo in (UP, LO):
                for tr in ((N_, T_, C_) if cplx else (N_, T_)):
                    for dg in (NONUNIT, UNIT):
                        A = np.asfortranarray((O.plrnt(na, na, seed, cplx) / na
                                               + np.eye(na)).astype(dt))
                        B0 = gen(M, N, seed + 1, dt)
                        seed += 2
                        alpha = scal(2.0 + 0.5j, dt)
                        B = B0.copy(order="F")
                        xk.trsm(side, uplo, tr, dg, alpha, A, B)
                        xk.invalidate_caches()
                        R = O.trsm(side, uplo, tr, dg, alpha, up(A), up(B0), nb=64)
                        r = checks.trsm_ratio(B, R, A, M, N)
                        assert r <= 10, (flag, uplo, tr, dg, r)
    finally:
        lib.xkb_tune_set(b"trsm_inv_leaves", 1.0)


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_trsm_pair_leaves(xk, dt):
    """Left, lower, op(A) = A with >= 2048 unknowns: with the tuning key
    trsm_pair_leaves = 1 (default) every node of two diagonal blocks but the
    first is applied through the inverse of its triangle (formed on a side
    stream; trsm_pair_split = 0, default, multiplies by the whole inverse,
    = 1 skips its zero block in two products), = 0 keeps leaf,
    coupling update, leaf.  Ragged split points (2148 unknowns), unit and
    non-unit diagonals: every form meets the reference bound."""
    cplx = np.issubdtype(dt, np.complexfloating)
    lib = xk.lib()
    M, N = 2148, 160
    seed = 1700
    try:
        for flag, split in ((1.0, 0.0), (1.0, 1.0), (0.0, 0.0)):
            lib.xkb_tune_set(b"trsm_pair_leaves", flag)
            lib.xkb_tune_set(b"trsm_pair_split", split)
            for dg in (NONUNIT, UNIT):
                A = np.asfortranarray((O.plrnt(M, M, seed, cplx) / M + np.eye(M)).astype(dt))
                B0 = gen(M, N, seed + 1, dt)
                seed += 2
                alpha = scal(2.0 + 0.5j, dt)
                B = B0.copy(order="F")
                xk.trsm(LEFT, LO, N_, dg, alpha, A, B)
                xk.invalidate_caches()
                R = O.trsm(LEFT, LO, N_, dg, alpha, up(A), up(B0), nb=64)
                r = checks.trsm_ratio(B, R, A, M, N)
                assert r <= 10, (flag, split, dg, r)
    finally:
        lib.xkb_tune_set(b"trsm_pair_leaves", 1.0)
        lib.xkb_tune_set(b"trsm_pair_split", 0.0)


@pytest.mark.parametrize("case", [
    # (dtype, M, N, K, opA, opB): few output tiles, long K
    (np.float64, 640, 1280, 2048, T_, N_),
    (np.float64, 300, 200, 2049, N_, T_),
    (np.complex128, 320, 256, 3000, C_, N_),
    (np.float64, 1000, 900, 3000, N_, N_),
])
def test_gemm_stream_k(xk, case):
    """Stream-K (tuning key gemm_sk_fill = 1: taken whenever split-K would
    be) and split-K (gemm_streamk = 0) on the same operands: both meet the
    reference bound, and stream-K's fixed order of the pieces makes repeated
    calls bit-identical."""
    import ctypes
    import torch
    from xkblas_b200 import GemmArgs
    dt, M, N, K, ta, tb = case
    cplx = dt == np.complex128
    A = gen(M, K, 70, dt) if ta == N_ else gen(K, M, 70, dt)
    B = gen(K, N, 71, dt) if tb == N_ else gen(N, K, 71, dt)
    C0 = gen(M, N, 72, dt)
    al, be = (0.5 + 1.25j, 0.75 - 0.5j) if cplx else (0.5, 0.75)
    dev = lambda X: torch.from_numpy(np.ascontiguousarray(X.T)).cuda()
    dA, dB = dev(A), dev(B)
    lib = xk.lib()
    R = O.gemm(ta, tb, al, A, B, be, C0.copy(order="F"), nb=256)
    outs = {}
    try:
        for mode, (sk, fill) in (("sk", (1.0, 1.0)), ("sk2", (1.0, 1.0)), ("split", (0.0, 0.8))):
            lib.xkb_tune_set(b"gemm_streamk", sk)
            lib.xkb_tune_set(b"gemm_sk_fill", fill)
            dC = dev(C0)
            g = GemmArgs(3 if cplx else 1, ta - N_, tb - N_, M, N, K, dA.data_ptr(), A.shape[0],
                         dB.data_ptr(), B.shape[0], dC.data_ptr(), M)
            g.alpha[0], g.alpha[1] = (al.real, al.imag) if cplx else (al, 0.0)
            g.beta[0], g.beta[1] = (be.real, be.imag) if cplx else (be, 0.0)
            torch.cuda.synchronize()
            k0 = xk.kernel_count()
            assert lib.xkb_cuda_gemm(ctypes.byref(g), None) == 0
            assert xk.kernel_count() - k0 == 2  # the pieces and their reduction
            xk.sync()
            outs[mode] = np.asfortranarray(dC.cpu().numpy().T)
    finally:
        lib.xkb_tune_set(b"gemm_streamk", 1.0)
        lib.xkb_tune_set(b"gemm_sk_fill", 0.8)
    assert lib.xkb_cuda_take_device_error() == 0
    assert np.array_equal(outs["sk"], outs["sk2"])
    for mode in ("sk", "split"):
        assert checks.gemm_ratio(outs[mode], R, A, B, C0, al, be, K) <= 3.0, mode
