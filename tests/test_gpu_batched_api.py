"""Deferred execution of the public async API: xkblas_{d,z}gemm_async and
left xkblas_{d,z}trsm_async calls are queued and run as one launch of the
tile-task executor at the next coherence point.  Checked through the C ABI
with host buffers (the reference calling sequence, testing/ztesting_gemm.c:
157-163) against the CPU oracle, under the reference's acceptance bounds
(tests/checks.py); the queue's ordering rules (read-after-write,
write-after-read, write-after-write on a queued buffer) are exercised with
dependent call chains.  Requires a B200."""
import numpy as np
import pytest

import oracle as O
from tests import checks

pytestmark = pytest.mark.gpu

N_, T_, C_ = 111, 112, 113
UP, LO = 121, 122
LEFT = 141
NONUNIT, UNIT = 131, 132


def _call_gemm(xk, ta, tb, alpha, A, B, beta, C):
    p = "z" if np.iscomplexobj(C) else "d"
    M, N = C.shape
    K = A.shape[1] if ta == N_ else A.shape[0]
    f = getattr(xk.lib(), "xkblas_%sgemm_async" % p)
    return f(ta, tb, M, N, K, xk._ptr(xk._scal(alpha, C.dtype)), xk._ptr(A), A.shape[0],
             xk._ptr(B), B.shape[0], xk._ptr(xk._scal(beta, C.dtype)), xk._ptr(C), C.shape[0])


def _call_trsm(xk, uplo, tr, dg, alpha, A, B):
    p = "z" if np.iscomplexobj(B) else "d"
    M, N = B.shape
    f = getattr(xk.lib(), "xkblas_%strsm_async" % p)
    return f(LEFT, uplo, tr, dg, M, N, xk._ptr(xk._scal(alpha, B.dtype)), xk._ptr(A), A.shape[0],
             xk._ptr(B), B.shape[0])


@pytest.fixture(params=[None, 1.0], ids=["one_batch", "flush_1MiB"])
def flush_mb(xk, request):
    """None: the default threshold (all calls in one batch); 1.0: the queue
    is launched whenever its operands reach 1 MiB (many batches, results made
    coherent against each batch's own completion event)."""
    if request.param is not None:
        xk.lib().xkb_tune_set(b"batch_flush_mb", request.param)
    yield request.param
    xk.lib().xkb_tune_set(b"batch_flush_mb", 2048.0)


def test_many_independent_calls_one_batch(xk, flush_mb):
    rng = np.random.default_rng(5)
    xk.reset_stats()
    calls = []
    seed = 1000
    for i in range(48):
        kind = rng.choice(["dgemm", "zgemm", "dtrsm", "ztrsm"], p=[0.5, 0.2, 0.2, 0.1])
        cplx = kind[0] == "z"
        seed += 3
        if kind.endswith("gemm"):
            M, N, K = (int(x) for x in rng.integers(1, 400, 3))
            ta = int(rng.choice([N_, T_, C_] if cplx else [N_, T_]))
            tb = int(rng.choice([N_, T_, C_] if cplx else [N_, T_]))
            A = O.plrnt(M, K, seed, cplx) if ta == N_ else O.plrnt(K, M, seed, cplx)
            B = O.plrnt(K, N, seed + 1, cplx) if tb == N_ else O.plrnt(N, K, seed + 1, cplx)
            C0 = O.plrnt(M, N, seed + 2, cplx)
            C = C0.copy(order="F")
            al, be = (1.5 - 0.5j, 0.25 + 1j) if cplx else (1.5, -0.75)
            assert _call_gemm(xk, ta, tb, al, A, B, be, C) == 0
            calls.append(("gemm", (ta, tb, al, A, B, be, C0, K), C))
        else:
            M, N = (int(x) for x in rng.integers(1, 400, 2))
            uplo = int(rng.choice([UP, LO]))
            tr = int(rng.choice([N_, T_, C_] if cplx else [N_, T_]))
            dg = int(rng.choice([NONUNIT, UNIT]))
            # reference testing/ztesting_trsm.c:130-134: A/max(M,N) + unit diagonal
            A = np.asfortranarray(O.plrnt(M, M, seed, cplx) / max(M, N) + np.eye(M))
            B0 = O.plrnt(M, N, seed + 1, cplx)
            B = B0.copy(order="F")
            al = (2.0 + 0.5j) if cplx else 2.0
            assert _call_trsm(xk, uplo, tr, dg, al, A, B) == 0
            calls.append(("trsm", (uplo, tr, dg, al, A, B0, M, N), B))
    for _, _, out in reversed(calls):
        xk.coherent(out)
    xk.sync()
    st = xk.stats()
    if flush_mb is None:
        assert st["batches"] == 1 and st["batched_calls"] == len(calls), st
    else:  # lone calls run outside the executor and are not counted
        assert st["batches"] > 1 and st["batched_calls"] <= len(calls), st
    for kind, args, out in calls:
        if kind == "gemm":
            ta, tb, al, A, B, be, C0, K = args
            ref = O.gemm(ta, tb, al, A, B, be, C0.copy(order="F"))
            r = checks.gemm_ratio(out, ref, A, B, C0, al, be, K)
            assert r <= 3, r
        else:
            uplo, tr, dg, al, A, B0, M, N = args
            ref = O.trsm(LEFT, uplo, tr, dg, al, A, B0.copy(order="F"), nb=64)
            r = checks.trsm_ratio(out, ref, A, M, N)
            assert r <= 10, r
    xk.invalidate_caches()


def test_dependent_calls_keep_program_order(xk):
    """Queue ordering: C1 = A B and D = Ap B are independent (one batch);
    A = Ap Ap writes A while the queued first call reads it (write-after-
    read: the queue runs first); C1 = C1 + A I reads the new A (read-after-
    write); X = D I joins that batch; the left solve X = L^-1 X reads X
    (read-after-write).  Only the final values are made coherent."""
    n = 200
    A0, B, Ap = O.plrnt(n, n, 61), O.plrnt(n, n, 62), O.plrnt(n, n, 63)
    L = np.asfortranarray(np.tril(O.plrnt(n, n, 64)) / n + np.eye(n))
    A = A0.copy(order="F")
    C1 = np.zeros((n, n), order="F")
    D = np.zeros((n, n), order="F")
    I = np.asfortranarray(np.eye(n))
    X = np.zeros((n, n), order="F")
    xk.reset_stats()
    assert _call_gemm(xk, N_, N_, 1.0, A, B, 0.0, C1) == 0      # C1 = A0 B
    assert _call_gemm(xk, N_, N_, 1.0, Ap, B, 0.0, D) == 0      # D = Ap B
    assert _call_gemm(xk, N_, N_, 1.0, Ap, Ap, 0.0, A) == 0     # A = Ap Ap
    assert _call_gemm(xk, N_, N_, 1.0, A, I, 1.0, C1) == 0      # C1 = C1 + A
    assert _call_gemm(xk, N_, N_, 1.0, D, I, 0.0, X) == 0       # X = D
    assert _call_trsm(xk, LO, N_, NONUNIT, 1.0, L, X) == 0      # X = L^-1 X
    for M_ in (C1, D, A, X):
        xk.coherent(M_)
    xk.sync()
    c1, d, a = A0 @ B, Ap @ B, Ap @ Ap
    want = {"C1": c1 + a, "D": d, "A": a, "X": np.linalg.solve(L, d)}
    for name, got in (("C1", C1), ("D", D), ("A", A), ("X", X)):
        assert np.abs(got - want[name]).max() <= 1e-12 * np.abs(want[name]).max(), name
    st = xk.stats()
    # calls 1-2 and 4-5 ran as two-call batches; 3 and 6 alone
    assert st["batches"] == 2 and st["batched_calls"] == 4, st
    xk.invalidate_caches()
