"""GPU parity of the Ozaki-II INT8 tensor-core form (XKBLAS_TENSOR_OP_MATH):
same reference bounds as the plain path, and never worse than the plain FP64
DMMA result against the double-double oracle.  Requires a B200."""
import ctypes

import numpy as np
import pytest

import oracle as O
from tests import checks
from xkblas_b200 import GemmArgs  # xkb_gemm_args of include/xkb_cuda.h

pytestmark = pytest.mark.gpu

N_, T_, C_ = 111, 112, 113
UP, LO = 121, 122
LEFT = 141
NONUNIT = 131


@pytest.fixture
def tc(xk):
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    yield xk
    xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)


def _dd_err(C, A, B, alpha, ta=N_, tb=N_, nrow=24, ncol=24, seed=0):
    rng = np.random.default_rng(seed)
    M, N = C.shape
    rows = np.sort(rng.choice(M, min(M, nrow), replace=False))
    cols = np.sort(rng.choice(N, min(N, ncol), replace=False))
    dd = O.gemm_dd(ta, tb, alpha, A, B, 0.0, None, rows, cols)
    opA = A if ta == N_ else A.T
    opB = B if tb == N_ else B.T
    scale = np.abs(opA[rows]) @ np.abs(opB[:, cols]) * abs(alpha)
    return float(np.max(np.abs(C[np.ix_(rows, cols)] - dd) / scale))


@pytest.mark.parametrize("mnk", [(300, 200, 513), (129, 257, 1000), (1024, 1024, 1024)])
def test_ozaki_dgemm_bounds(tc, mnk):
    M, N, K = mnk
    s0 = tc.stats()["ozaki_calls"]
    for ta in (N_, T_):
        for tb in (N_, T_):
            A = O.plrnt(M, K, 5) if ta == N_ else O.plrnt(K, M, 5)
            B = O.plrnt(K, N, 6) if tb == N_ else O.plrnt(N, K, 6)
            C0 = O.plrnt(M, N, 7)
            C = C0.copy(order="F")
            tc.gemm(ta, tb, 1.5, A, B, -0.5, C)
            tc.invalidate_caches()
            R = O.gemm(ta, tb, 1.5, A, B, -0.5, C0.copy(order="F"))
            assert checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, K) <= 3.0
            assert checks.plasma_ratio(C, R, A, B, 1.5, K) < 10
    assert tc.stats()["ozaki_calls"] >= s0 + 4


def test_ozaki_no_worse_than_plain_exponent_spread(xk):
    """Config-4 distribution (per-row / per-column exponents in [-20, 20]) at
    a size the oracle handles: Ozaki error vs double-double <= plain error."""
    M = N = K = 768
    A = O.expspread(M, K, 101, emax=20, by_col=False)
    B = O.expspread(K, N, 102, emax=20, by_col=True)
    Cp = np.zeros((M, N), order="F")
    xk.gemm(N_, N_, 1.0, A, B, 0.0, Cp)
    xk.invalidate_caches()
    xk.set_modemath(xk.XKBLAS_TENSOR_OP_MATH)
    try:
        Co = np.zeros((M, N), order="F")
        xk.gemm(N_, N_, 1.0, A, B, 0.0, Co)
        xk.invalidate_caches()
    finally:
        xk.set_modemath(xk.XKBLAS_DEFAULT_MATH)
    ep = _dd_err(Cp, A, B, 1.0, nrow=48, ncol=48)
    eo = _dd_err(Co, A, B, 1.0, nrow=48, ncol=48)
    assert eo <= max(ep, 2.0 ** -52), (eo, ep)
    assert eo < 2.0 ** -50


def test_ozaki_zgemm_all_trans(tc):
    M, N, K = 150, 170, 333
    for ta in (N_, T_, C_):
        for tb in (N_, T_, C_):
            A = O.plrnt(M, K, 8, True) if ta == N_ else O.plrnt(K, M, 8, True)
            B = O.plrnt(K, N, 9, True) if tb == N_ else O.plrnt(N, K, 9, True)
            C0 = O.plrnt(M, N, 10, True)
            al, be = 1.5 - 0.25j, -0.5 + 0.125j
            C = C0.copy(order="F")
            tc.gemm(ta, tb, al, A, B, be, C)
            tc.invalidate_caches()
            R = O.gemm(ta, tb, al, A, B, be, C0.copy(order="F"))
            assert checks.gemm_ratio(C, R, A, B, C0, al, be, K) <= 3.0, (ta, tb)


@pytest.mark.parametrize("uplo", [UP, LO])
def test_ozaki_syrk_herk(tc, uplo):
    N, K = 300, 280
    A = O.plrnt(N, K, 11)
    C0 = O.plgsy(N, 12)
    C = C0.copy(order="F")
    tc.syrk(uplo, N_, 1.0, A, 1.0, C)
    tc.invalidate_caches()
    R = O.syrk(uplo, N_, 1.0, A, 1.0, C0.copy(order="F"))
    sel = np.tril if uplo == LO else np.triu
    assert checks.rk_ratio(sel(C), sel(R), A, C0, N) <= 10
    Az = O.plrnt(K, N, 13, True)
    Cz0 = O.plgsy(N, 14, cplx=True)
    Cz = Cz0.copy(order="F")
    tc.syrk(uplo, C_, 1.0, Az, 1.0, Cz, herm=True)
    tc.invalidate_caches()
    Rz = O.syrk(uplo, C_, 1.0, Az, 1.0, Cz0.copy(order="F"), herm=True)
    assert checks.rk_ratio(sel(Cz), sel(Rz), Az, Cz0, N) <= 10
    assert np.all(np.diag(Cz).imag == 0)


def test_ozaki_trsm_updates(tc):
    M = N = 640
    A = np.asfortranarray(np.tril(O.plrnt(M, M, 15)) + M * np.eye(M))
    B0 = O.plrnt(M, N, 16)
    B = B0.copy(order="F")
    s0 = tc.stats()["ozaki_calls"]
    tc.trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B)
    tc.invalidate_caches()
    R = O.trsm(LEFT, LO, N_, NONUNIT, 2.0, A, B0.copy(order="F"), nb=128)
    assert checks.trsm_ratio(B, R, A, M, N) <= 10


def test_ozaki_moduli_count_controls_accuracy(xk):
    """Through the thin C ABI on device memory: fewer moduli -> larger error;
    the default count reaches FP64 accuracy."""
    import torch
    M = N = K = 512
    A = O.plrnt(M, K, 21)
    B = O.plrnt(K, N, 22)
    dA = torch.from_numpy(A.T.copy()).cuda()  # row-major (K,M) = column-major A
    dB = torch.from_numpy(B.T.copy()).cuda()
    torch.cuda.synchronize()
    lib = xk.lib()
    errs = {}
    for nm in (8, 10, 12, 0):
        dC = torch.zeros(N, M, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
        g.alpha[0] = 1.0
        assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g), nm, None) == 0
        xk.sync()
        C = np.asfortranarray(dC.cpu().numpy().T)
        errs[nm] = _dd_err(C, A, B, 1.0, nrow=32, ncol=32)
    assert errs[8] > errs[12] > 0 or errs[12] < 1e-15
    assert errs[0] < 2.0 ** -50
    assert lib.xkb_cuda_take_device_error() == 0


def test_ozaki_nonfinite_rows_and_columns(xk):
    """A NaN or Inf in a row of op(A) / column of op(B) makes that row /
    column of the Ozaki product NaN (the shift sentinel); the other entries
    are unaffected and meet the GEMM bound."""
    import torch
    M, N, K = 96, 80, 300
    A = O.plrnt(M, K, 21)
    B = O.plrnt(K, N, 22)
    A[3, 17] = np.nan
    A[7, 0] = np.inf
    B[5, 11] = -np.inf
    dA = torch.from_numpy(A.T.copy()).cuda()  # column-major device copies
    dB = torch.from_numpy(B.T.copy()).cuda()
    dC = torch.zeros(N, M, dtype=torch.float64, device="cuda")
    ga = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
    ga.alpha[0] = 1.0
    torch.cuda.synchronize()
    assert xk.lib().xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, None) == 0
    xk.sync()
    C = dC.cpu().numpy().T
    bad_r, bad_c = [3, 7], [11]
    assert np.isnan(C[bad_r, :]).all() and np.isnan(C[:, bad_c]).all()
    keep_r = [i for i in range(M) if i not in bad_r]
    keep_c = [j for j in range(N) if j not in bad_c]
    Cg = C[np.ix_(keep_r, keep_c)]
    R = A[keep_r] @ B[:, keep_c]
    assert np.isfinite(Cg).all()
    assert checks.gemm_ratio(Cg, R, A[keep_r], B[:, keep_c], np.zeros_like(R), 1.0, 0.0, K) <= 3.0
    assert xk.lib().xkb_cuda_take_device_error() == 0


def test_ozaki_k_beyond_int32_limit(tc):
    """K > 131072 exceeds exact INT32 accumulation: the Ozaki entry point
    returns XKB_ERANGE and the public API falls back to the plain kernel."""
    import torch
    M, N, K = 8, 8, 131073
    lib = tc.lib()
    dA = torch.rand(K, M, dtype=torch.float64, device="cuda")
    dB = torch.rand(N, K, dtype=torch.float64, device="cuda")
    dC = torch.zeros(N, M, dtype=torch.float64, device="cuda")
    ga = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
    ga.alpha[0] = 1.0
    torch.cuda.synchronize()
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, None) == -6  # XKB_ERANGE
    # public API in tensor-op mode: min(M, N, K) is below the crossover, so
    # this shape runs plain; force the crossover down to exercise the fallback
    A = np.asfortranarray(np.random.default_rng(1).random((M, K)))
    B = np.asfortranarray(np.random.default_rng(2).random((K, N)))
    C = np.zeros((M, N), order="F")
    lib.xkb_tune_set(b"ozaki_min_dim", 1.0)
    try:
        tc.gemm(N_, N_, 1.0, A, B, 0.0, C)
    finally:
        lib.xkb_tune_set(b"ozaki_min_dim", 2048.0)
    tc.invalidate_caches()
    assert checks.gemm_ratio(C, A @ B, A, B, np.zeros((M, N)), 1.0, 0.0, K) <= 3.0


@pytest.mark.parametrize("mnk", [(300, 200, 513), (1024, 1024, 1024)])
def test_ozaki_cta_pair_kernel_matches(xk, mnk):
    """The CTA-pair INT8 GEMM (tuning key oz_2cta = 1) gives bit-identical
    results to the single-CTA kernel (same residue products, exact)."""
    import torch
    M, N, K = mnk
    lib = xk.lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    dA = torch.rand(K, M, generator=g, dtype=torch.float64, device="cuda") - 0.5
    dB = torch.rand(N, K, generator=g, dtype=torch.float64, device="cuda") - 0.5
    out = []
    for flag in (0.0, 1.0):
        dC = torch.zeros(N, M, dtype=torch.float64, device="cuda")
        ga = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
        ga.alpha[0] = 1.0
        lib.xkb_tune_set(b"oz_2cta", flag)
        try:
            torch.cuda.synchronize()
            assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, None) == 0
            xk.sync()
        finally:
            lib.xkb_tune_set(b"oz_2cta", 0.0)
        out.append(dC.clone())
    assert torch.equal(out[0], out[1])
    ref = dB @ dA  # row-major N x M view of the column-major C = A B
    assert (out[0] - ref).abs().max().item() <= 4 * 2.0 ** -53 * K * 0.25 * 2
    assert lib.xkb_cuda_take_device_error() == 0


# ---- the remaining level-3 operations in tensor-op mode ----------------------
# Each call must run at least one Ozaki contraction (seen in the per-call
# trace) and meet the reference test program's bound against the oracle.
RIGHT, UNIT = 142, 132


def _gen(M, N, seed, cplx):
    return O.plrnt(M, N, seed, cplx)


def _ran_ozaki(tr):
    return "ozaki_gemm" in tr.ops()


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_ozaki_gemmt(tc, cplx, uplo):
    N, K = 260, 190
    A, B, C0 = _gen(N, K, 600, cplx), _gen(K, N, 601, cplx), _gen(N, N, 602, cplx)
    C = C0.copy(order="F")
    with tc.contraction_trace() as tr:
        tc.gemmt(uplo, N_, N_, 1.25, A, B, -1.0, C)
    tc.invalidate_caches()
    assert _ran_ozaki(tr)
    R = O.gemmt(uplo, N_, N_, 1.25, A, B, -1.0, C0.copy(order="F"))
    sel = np.tril if uplo == LO else np.triu
    assert checks.gemm_ratio(sel(C), sel(R), A, B, C0, 1.25, -1.0, K) <= 3
    other = np.triu if uplo == LO else np.tril
    k = 1 if uplo == LO else -1
    np.testing.assert_array_equal(other(C, k), other(C0, k))


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_ozaki_syr2k_her2k(tc, cplx, uplo):
    N, K = 230, 170
    for herm in ((False, True) if cplx else (False,)):
        for tr_ in (N_, (C_ if herm else T_)):
            A = _gen(N, K, 500, cplx) if tr_ == N_ else _gen(K, N, 500, cplx)
            B = _gen(N, K, 501, cplx) if tr_ == N_ else _gen(K, N, 501, cplx)
            C0 = O.plgsy(N, 502, cplx=cplx)
            alpha = (0.75 + 0.5j) if cplx else 0.75
            C = C0.copy(order="F")
            with tc.contraction_trace() as tr:
                tc.syr2k(uplo, tr_, alpha, A, B, 0.5, C, herm=herm)
            tc.invalidate_caches()
            assert _ran_ozaki(tr)
            R = O.syr2k(uplo, tr_, alpha, A, B, 0.5, C0.copy(order="F"), herm=herm)
            sel = np.tril if uplo == LO else np.triu
            # reference bound, testing/ztesting_syr2k.c (the syrk form with ||B||)
            assert checks.rk_ratio(sel(C), sel(R), A, C0, N, checks.ninf(B)) <= 10
            if herm:
                assert np.all(np.diag(C).imag == 0)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [UP, LO])
def test_ozaki_symm_hemm(tc, cplx, side, uplo):
    M, N = 240, 200
    na = M if side == LEFT else N
    for herm in ((False, True) if cplx else (False,)):
        A = _gen(na, na, 700, cplx)
        B, C0 = _gen(M, N, 701, cplx), _gen(M, N, 702, cplx)
        alpha = (1.5 + 0.5j) if cplx else 1.5
        C = C0.copy(order="F")
        with tc.contraction_trace() as tr:
            tc.symm(side, uplo, alpha, A, B, -0.5, C, herm=herm)
        tc.invalidate_caches()
        assert _ran_ozaki(tr)
        R = O.symm(side, uplo, alpha, A, B, -0.5, C0.copy(order="F"), herm=herm)
        # reference bound, testing/ztesting_symm.c:240-246
        den = (checks.ninf(A) + checks.ninf(B) + checks.ninf(C0)) * max(M, N) * 2.0 ** -53
        assert checks.ninf(C - R) / den <= 10


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
def test_ozaki_trmm(tc, cplx, side):
    M, N = 220, 180
    na = M if side == LEFT else N
    for uplo in (UP, LO):
        for tr_ in ((N_, T_, C_) if cplx else (N_, T_)):
            for dg in (NONUNIT, UNIT):
                A = _gen(na, na, 800, cplx)
                B0 = _gen(M, N, 801, cplx)
                B = B0.copy(order="F")
                with tc.contraction_trace() as tr:
                    tc.trmm(side, uplo, tr_, dg, 1.5, A, B)
                tc.invalidate_caches()
                assert _ran_ozaki(tr)
                R = O.trmm(side, uplo, tr_, dg, 1.5, A, B0.copy(order="F"))
                # reference bound, testing/ztesting_trmm.c (as TRSM's)
                assert checks.trsm_ratio(B, R, A, M, N) <= 10, (uplo, tr_, dg)


# ---- the data rule for the moduli count (nmod = 0) ----------------------------
def _elem_spread(M, N, seed, emax):
    """u 2^e with u ~ U[-1, 1] and e ~ U{-emax..emax} drawn per ENTRY: the
    dynamic range lies inside every row and column."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.uniform(-1.0, 1.0, (M, N))
                             * np.ldexp(1.0, rng.integers(-emax, emax + 1, (M, N))))


def _run_cabi(xk, A, B, nmod, plain=False):
    """C = A B through the C ABI on device copies; returns (C, latest count)."""
    import torch
    M, K = A.shape
    N = B.shape[1]
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dC = torch.zeros(N, M, dtype=torch.float64, device="cuda")
    g = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, dC.data_ptr(), M)
    g.alpha[0] = 1.0
    torch.cuda.synchronize()
    lib = xk.lib()
    r = lib.xkb_cuda_gemm(ctypes.byref(g), None) if plain else \
        lib.xkb_cuda_ozaki_gemm(ctypes.byref(g), nmod, None)
    assert r == 0
    xk.sync()
    assert lib.xkb_cuda_take_device_error() == 0
    return np.asfortranarray(dC.cpu().numpy().T), xk.ozaki_counts()[3]


def test_data_rule_per_element_spread_takes_more_moduli(xk):
    """Exponents in [-20, 20] per entry: the count rises to 16 and the result
    is no less accurate than the plain FP64 kernel's against double-double,
    while a fixed 15 is measurably less accurate."""
    xk.lib().xkb_tune_clear()
    n = 768
    A, B = _elem_spread(n, n, 1, 20), _elem_spread(n, n, 2, 20)
    Cp, _ = _run_cabi(xk, A, B, 0, plain=True)
    Ca, nm = _run_cabi(xk, A, B, 0)
    C15, _ = _run_cabi(xk, A, B, 15)
    assert nm == 16
    ep = _dd_err(Cp, A, B, 1.0, nrow=64, ncol=64)
    ea = _dd_err(Ca, A, B, 1.0, nrow=64, ncol=64)
    e15 = _dd_err(C15, A, B, 1.0, nrow=64, ncol=64)
    assert ea <= ep, (ea, ep)
    assert ea < e15, (ea, e15)


def test_data_rule_keeps_15_moduli_on_row_column_spread(xk):
    """The benchmark's distribution (exponents per row of A / column of B):
    every row is of one magnitude, the count stays at 15."""
    xk.lib().xkb_tune_clear()
    n = 640
    A = O.expspread(n, n, 101, emax=20, by_col=False)
    B = O.expspread(n, n, 102, emax=20, by_col=True)
    Ca, nm = _run_cabi(xk, A, B, 0)
    Cp, _ = _run_cabi(xk, A, B, 0, plain=True)
    assert nm == 15
    assert _dd_err(Ca, A, B, 1.0, nrow=48, ncol=48) <= _dd_err(Cp, A, B, 1.0, nrow=48, ncol=48)


def test_data_rule_falls_back_to_plain_kernel(xk):
    """A spread no 16-moduli product can carry (exponents in [-200, 200] per
    entry): the call is computed by the plain FP64 kernel on the device --
    the result equals that kernel's bit for bit, and the counters say so."""
    n = 300
    A, B = _elem_spread(n, n, 3, 200), _elem_spread(n, n, 4, 200)
    c0 = xk.ozaki_counts()
    Ca, nm = _run_cabi(xk, A, B, 0)
    c1 = xk.ozaki_counts()
    Cp, _ = _run_cabi(xk, A, B, 0, plain=True)
    assert nm == 0
    assert c1[2] == c0[2] + 1 and c1[0] == c0[0] + 1
    np.testing.assert_array_equal(Ca, Cp)


def test_data_rule_through_public_api(tc):
    """Tensor-op mode through xkblas_dgemm_async: per-entry spread takes 16
    moduli and meets the reference GEMM bound."""
    tc.lib().xkb_tune_clear()
    M, N, K = 520, 300, 700
    A, B = _elem_spread(M, K, 5, 20), _elem_spread(K, N, 6, 20)
    C0 = O.plrnt(M, N, 7)
    C = C0.copy(order="F")
    tc.gemm(N_, N_, 1.5, A, B, -0.5, C)
    tc.invalidate_caches()
    assert tc.ozaki_counts()[3] == 16
    R = O.gemm(N_, N_, 1.5, A, B, -0.5, C0.copy(order="F"))
    assert checks.gemm_ratio(C, R, A, B, C0, 1.5, -0.5, K) <= 3.0
