"""Acceptance bounds of the reference's test programs, restated.

GEMM   testing/ztesting_gemm.c:289-303:
       ||C - Cref||_inf / (sqrt(K+2)|alpha| ||A||_inf ||B||_inf
                           + sqrt(2)|beta| ||C0||_inf)  <= 3 eps
TRSM   testing/ztesting_trsm.c:246-252 (TRMM identical, ztesting_trmm.c):
       ||B - Bref||_inf / ((||A||_inf + ||Bref||_inf) max(M,N) eps) <= 10
SYRK/HERK testing/ztesting_syrk.c:225-231, ztesting_herk.c:239-245:
       ||C - Cref|| / ((||A|| + ||C0||) N eps) <= 10
SYMM   testing/ztesting_symm.c:240-246:
       ||C - Cref|| / ((||A|| + ||B|| + ||C0||) N eps) <= 10
and the PLASMA-style bound of the task statement
       ||C - Cref|| / (|alpha| ||A|| ||B|| k eps) < 10.
eps is the unit roundoff of the storage precision (LAPACK dlamch('e')).
"""
import numpy as np

EPS = {np.dtype(np.float32): 2.0 ** -24, np.dtype(np.float64): 2.0 ** -53,
       np.dtype(np.complex64): 2.0 ** -24, np.dtype(np.complex128): 2.0 ** -53}


def ninf(X):
    X = np.asarray(X)
    if X.size == 0:
        return 0.0
    return float(np.abs(X).sum(axis=1).max())


def gemm_ratio(C, Cref, A, B, C0, alpha, beta, K):
    eps = EPS[np.dtype(C.dtype)]
    den = np.sqrt(K + 2.0) * abs(alpha) * ninf(A) * ninf(B) + np.sqrt(2.0) * abs(beta) * ninf(C0)
    if den == 0:
        return float(ninf(C - Cref))
    return ninf(np.asarray(C, dtype=np.complex128) - Cref) / den / eps


def plasma_ratio(C, Cref, A, B, alpha, K):
    eps = EPS[np.dtype(C.dtype)]
    den = abs(alpha) * ninf(A) * ninf(B) * max(K, 1) * eps
    return ninf(np.asarray(C, dtype=np.complex128) - Cref) / den


def trsm_ratio(B, Bref, A, M, N):
    eps = EPS[np.dtype(B.dtype)]
    den = (ninf(A) + ninf(Bref)) * max(M, N) * eps
    return ninf(np.asarray(B, dtype=np.complex128) - Bref) / den


def rk_ratio(C, Cref, A, C0, N, Bn=0.0):
    eps = EPS[np.dtype(C.dtype)]
    den = (ninf(A) + Bn + ninf(C0)) * max(N, 1) * eps
    return ninf(np.asarray(C, dtype=np.complex128) - Cref) / den


def tri(X, uplo_lower):
    return np.tril(X) if uplo_lower else np.triu(X)
