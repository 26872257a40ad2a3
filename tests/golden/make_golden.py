"""Generate tests/golden/openblas_small.npz: golden outputs of the reference's
CPU path for small seeded inputs.

The reference's CPU tile bodies and its own test reference are the system
BLAS reached through dlsym of the Fortran symbols (blas/zgemm.c:383-414,
blas/xkblas.c:2678-2696; testing/ztesting_gemm.c:262 compares against
xkblas_zgemm_native).  This script calls that same library (OpenBLAS 0.3.15
as shipped in this image) on inputs from the oracle's seeded generators and
stores the outputs with the generator seeds of the inputs (tests rebuild the
inputs with the same generators, whose first values are stored too), so the
oracle restatement is pinned against the reference's own CPU path without
needing the BLAS at test time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "openblas_small.npz")


def main():
    O.blas_open(threads=1)
    rec = {}
    seed = 11
    # GEMM: all trans pairs, ragged sizes, alpha 1.5 / beta -0.5 as in the DGEMM 1024^3 workload
    for cplx in (False, True):
        ops = (O.NOTRANS, O.TRANS, O.CONJTRANS) if cplx else (O.NOTRANS, O.TRANS)
        for ta in ops:
            for tb in ops:
                M, N, K = 19, 13, 23
                Am, An = (M, K) if ta == O.NOTRANS else (K, M)
                Bm, Bn = (K, N) if tb == O.NOTRANS else (N, K)
                A = O.plrnt(Am, An, seed, cplx)
                B = O.plrnt(Bm, Bn, seed + 1, cplx)
                C = O.plrnt(M, N, seed + 2, cplx)
                seed += 3
                alpha, beta = (1.5 - 0.25j, -0.5 + 0.125j) if cplx else (1.5, -0.5)
                R = C.copy(order="F")
                O.native_gemm(ta, tb, alpha, A, B, beta, R)
                key = "gemm_%s_%d_%d" % ("z" if cplx else "d", ta, tb)
                rec[key + "_R"] = R
                rec[key + "_seed"] = np.array([seed - 3])
                rec[key + "_ab"] = np.array([alpha, beta], dtype=np.complex128)
    # TRSM: all 8 side/uplo/trans cases x diag, well conditioned A
    for cplx in (False, True):
        for side in (O.LEFT, O.RIGHT):
            for uplo in (O.UPPER, O.LOWER):
                for tr in ((O.NOTRANS, O.TRANS, O.CONJTRANS) if cplx else (O.NOTRANS, O.TRANS)):
                    for dg in (O.NONUNIT, O.UNIT):
                        M, N = 21, 17
                        na = M if side == O.LEFT else N
                        A = O.plrnt(na, na, seed, cplx) / na
                        A = np.asfortranarray(A + (2.0 * np.eye(na)))
                        B = O.plrnt(M, N, seed + 1, cplx)
                        seed += 2
                        alpha = (2.0 + 0.5j) if cplx else 2.0
                        R = B.copy(order="F")
                        O.native_trsm(side, uplo, tr, dg, alpha, A, R)
                        key = "trsm_%s_%d_%d_%d_%d" % ("z" if cplx else "d", side, uplo, tr, dg)
                        rec[key + "_R"] = R
                        rec[key + "_seed"] = np.array([seed - 2])
                        rec[key + "_ab"] = np.array([alpha], dtype=np.complex128)
    # SYRK (d) and HERK (z), the reference test generator for C
    for cplx in (False, True):
        for uplo in (O.UPPER, O.LOWER):
            for tr in (O.NOTRANS, O.CONJTRANS if cplx else O.TRANS):
                N, K = 19, 15
                A = O.plrnt(N, K, seed, cplx) if tr == O.NOTRANS else O.plrnt(K, N, seed, cplx)
                C = O.plgsy(N, seed + 1, cplx=cplx)
                seed += 2
                R = C.copy(order="F")
                O.native_rk(uplo, tr, 1.0, A, 1.0, R, herm=cplx)
                key = "rk_%s_%d_%d" % ("z" if cplx else "d", uplo, tr)
                rec[key + "_R"] = R
                rec[key + "_seed"] = np.array([seed - 2])
    rec["generator_plrnt_d"] = O.plrnt(7, 5, 1)
    rec["generator_plrnt_z"] = O.plrnt(7, 5, 1, cplx=True)
    rec["generator_plgsy_d"] = O.plgsy(6, 51)
    rec["blas"] = np.array([os.path.basename(O.find_openblas() or "")])
    np.savez_compressed(OUT, **rec)
    print("wrote", OUT, len(rec), "arrays")


if __name__ == "__main__":
    main()
