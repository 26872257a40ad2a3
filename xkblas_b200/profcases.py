"""Small, self-contained cases for profiling single kernels with ncu:

    python -m xkblas_b200.profcases dmma|update256|ozaki|ozaki2|ozaki8192|splitk|streamk|repack|trsm|potrf|potrf8192|getrf|getrf8192|batch|copy

dmma    DGEMM NN 4096^3 through xkb_cuda_gemm (k_gemm_dmma), two calls
update256  the Cholesky's first trailing update at 8192 with 256-wide
        blocks: C(7680 x 7680, lower) -= P P^T, K = 256, two calls
ozaki   the same through xkb_cuda_ozaki_gemm, 16 moduli (k_oz_* kernels)
ozaki2  the same with the CTA-pair INT8 kernel (tuning key oz_2cta = 1, k_oz_gemm2)
ozaki8192  DGEMM NN 8192^3, xkb_cuda_ozaki_gemm with the count chosen on the
        device (nmod = 0: 15 moduli on these inputs), two calls: the DRAM
        traffic of k_oz_gemm at a size whose residue planes exceed L2
splitk  DGEMM NN 512 x 512 x 4096 through xkb_cuda_gemm: 16 output tiles,
        split-K (k_gemm_dmma slices + k_gemm_splitk)
streamk DGEMM TN 640 x 1280 x 2048 through xkb_cuda_gemm: 50 output tiles,
        stream-K (k_gemm_dmma_sk pieces + k_gemm_sk_reduce), two calls
repack  the DGEMM with lda = ldb = 4097 (k_repack, then k_gemm_dmma)
trsm    DTRSM L/L/N/N 4096 x 4096, diagonally dominant (k_trsm_block, GEMMs)
potrf   DPOTRF lower 4096 (k_potrf_block, k_trsm_block, GEMMs)
potrf8192  DPOTRF lower 8192, two factorizations (the blocked look-ahead
        form at its default block width)
getrf   DGETRF without pivoting 4096, diagonally dominant (k_getrf_block,
        k_trsm_block, GEMMs)
getrf8192  the same at 8192
copy    beta scaling (k_scale, 8192^2) and the TRMM / SYMM materialisations
        (k_tri_fill, k_copy2d, k_sym_fill, 4096^2)
batch   150 mixed calls (70% DGEMM, 20% DTRSM, 10% ZGEMM; M, N, K
        log-uniform in [64, 2048]) as one xkb_cuda_batch launch (k_sched)

Each case holds a few GB at most and finishes in seconds.  Inputs are seeded
uniform [-0.5, 0.5] matrices on the device."""
import ctypes
import sys

import numpy as np


from xkblas_b200 import GemmArgs as _GemmArgs  # xkb_gemm_args


def main(case):
    import torch
    import xkblas_b200 as X
    lib = X.lib()
    X.init()
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    sp = ctypes.c_void_p(st.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(1)
    f64 = torch.float64

    def rnd(r, c):  # column-major r x c
        return torch.rand(c, r, generator=g, device="cuda", dtype=f64) - 0.5

    keep = []
    if case == "ozaki2":
        lib.xkb_tune_set(b"oz_2cta", 1.0)
    if case == "update256":
        m, k = 7680, 256
        P, C = rnd(m, k), rnd(m, m)
        keep += [P, C]
        ga = _GemmArgs(1, 0, 1, m, m, k, P.data_ptr(), m, P.data_ptr(), m, C.data_ptr(), m)
        ga.alpha[0], ga.beta[0], ga.uplo = -1.0, 1.0, 1
        for _ in range(2):
            assert lib.xkb_cuda_gemm(ctypes.byref(ga), sp) == 0
    elif case == "streamk":
        m, n, k = 640, 1280, 2048
        A, B, C = rnd(k, m), rnd(k, n), rnd(m, n)  # op(A) = A^T: A stored k x m
        keep += [A, B, C]
        ga = _GemmArgs(1, 1, 0, m, n, k, A.data_ptr(), k, B.data_ptr(), k, C.data_ptr(), m)
        ga.alpha[0] = ga.beta[0] = 1.0
        for _ in range(2):
            assert lib.xkb_cuda_gemm(ctypes.byref(ga), sp) == 0
    elif case in ("ozaki8192", "splitk"):
        m, n, k = (8192, 8192, 8192) if case == "ozaki8192" else (512, 512, 4096)
        A, B, C = rnd(m, k), rnd(k, n), rnd(m, n)
        keep += [A, B, C]
        ga = _GemmArgs(1, 0, 0, m, n, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m)
        ga.alpha[0] = 1.0
        for _ in range(2):
            rc = (lib.xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, sp) if case == "ozaki8192"
                  else lib.xkb_cuda_gemm(ctypes.byref(ga), sp))
            assert rc == 0, rc
    elif case in ("dmma", "ozaki", "ozaki2", "repack"):
        n = 4096
        ld = n + 1 if case == "repack" else n
        A, B, C = rnd(ld, n), rnd(ld, n), rnd(n, n)
        keep += [A, B, C]
        ga = _GemmArgs(1, 0, 0, n, n, n, A.data_ptr(), ld, B.data_ptr(), ld, C.data_ptr(), n)
        ga.alpha[0] = ga.beta[0] = 1.0
        for _ in range(2):
            rc = (lib.xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, sp) if case.startswith("ozaki")
                  else lib.xkb_cuda_gemm(ctypes.byref(ga), sp))
            assert rc == 0, rc
    elif case == "trsm":
        n = 4096
        L = torch.tril(rnd(n, n).t()) + n * torch.eye(n, device="cuda", dtype=f64)
        A, B = L.t().contiguous(), rnd(n, n)
        keep += [A, B]
        al = (ctypes.c_double * 2)(2.0, 0.0)
        for _ in range(2):
            assert lib.xkb_cuda_trsm(1, 0, 1, 0, 0, n, n,
                                     ctypes.cast(al, ctypes.POINTER(ctypes.c_double)),
                                     A.data_ptr(), n, B.data_ptr(), n, 0, sp) == 0
    elif case in ("potrf", "potrf8192"):
        n = 8192 if case == "potrf8192" else 4096
        Bm = rnd(n, n)
        A0 = Bm @ Bm.t() / n + torch.eye(n, device="cuda", dtype=f64)
        A = A0.clone()
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        keep += [A0, A, info]
        for _ in range(2):
            A.copy_(A0)
            assert lib.xkb_cuda_potrf(1, 1, n, A.data_ptr(), n, info.data_ptr(), 0, sp) == 0
    elif case in ("getrf", "getrf8192"):
        n = 8192 if case == "getrf8192" else 4096
        A0 = rnd(n, n) + n * torch.eye(n, device="cuda", dtype=f64)
        A = A0.clone()
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        keep += [A0, A, info]
        for _ in range(2):
            A.copy_(A0)
            assert lib.xkb_cuda_getrf_nopiv(1, n, A.data_ptr(), n, info.data_ptr(), 0, sp) == 0
    elif case == "batch":
        rng = np.random.default_rng(2024)

        def lu():
            return int(np.exp(rng.uniform(np.log(64), np.log(2048))))

        ops = []
        for _ in range(150):
            r = rng.random()
            o = X.BatchOp()
            if r < 0.7 or r >= 0.9:
                cplx = r >= 0.9
                m, n, k = lu(), lu(), lu()
                A, B, C = rnd(m, k), rnd(k, n), rnd(m, n)
                if cplx:
                    A, B, C = torch.complex(A, A), torch.complex(B, B), torch.complex(C, C)
                o.kind, o.dtype, o.M, o.N, o.K = 0, 3 if cplx else 1, m, n, k
                o.A, o.lda, o.B, o.ldb, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m
                o.alpha[0] = o.beta[0] = 1.0
                keep += [A, B, C]
            else:
                m, n = lu(), lu()
                L = torch.tril(rnd(m, m).t()) + m * torch.eye(m, device="cuda", dtype=f64)
                A, B = L.t().contiguous(), rnd(m, n)
                o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, 1, 0, 0, m, n
                o.A, o.lda, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), m
                o.alpha[0] = 1.0
                keep += [A, B]
            ops.append(o)
        arr = (X.BatchOp * len(ops))(*ops)
        for _ in range(2):
            assert lib.xkb_cuda_batch(arr, len(ops), 0, sp) == 0
    elif case == "copy":
        # HBM-bound helpers: beta scaling of C (k_scale, 8192^2), the
        # triangle and symmetric materialisations of TRMM / SYMM
        # (k_tri_fill, k_copy2d, k_sym_fill, 4096^2)
        n = 8192
        C = rnd(n, n)
        keep += [C]
        be = (ctypes.c_double * 2)(0.5, 0.0)
        bp = ctypes.cast(be, ctypes.POINTER(ctypes.c_double))
        for _ in range(2):
            assert lib.xkb_cuda_scale(1, n, n, bp, C.data_ptr(), n, 0, 0, 0, sp) == 0
        n = 4096
        A, B, D = rnd(n, n), rnd(n, n), rnd(n, n)
        keep += [A, B, D]
        al = (ctypes.c_double * 2)(1.0, 0.0)
        ap = ctypes.cast(al, ctypes.POINTER(ctypes.c_double))
        for _ in range(2):
            assert lib.xkb_cuda_trmm(1, 0, 1, 0, 0, n, n, ap, A.data_ptr(), n, B.data_ptr(), n, 0,
                                     sp) == 0
            assert lib.xkb_cuda_symm(1, 0, 0, 1, n, n, ap, A.data_ptr(), n, B.data_ptr(), n, bp,
                                     D.data_ptr(), n, 0, sp) == 0
    else:
        raise SystemExit("unknown case %r" % case)
    torch.cuda.synchronize()
    assert lib.xkb_cuda_take_device_error() == 0
    print("ok", case)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "dmma")
