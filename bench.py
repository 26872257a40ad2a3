"""Benchmark: FP64-accurate DGEMM TFLOP/s on one B200, Ozaki INT8 tensor-core
form vs the plain FP64 DMMA kernel, on the workload
"DGEMM NN M=N=K=16384 with wide exponent spread (a_ij = u*2^e, u ~ U[-1,1],
e ~ U{-20..20} per row of A and per column of B)".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0.  `value` = 2*M*N*K / device time of one Ozaki DGEMM
call (C ABI xkb_cuda_ozaki_gemm, inputs resident in HBM, 2 GiB each, so every
step streams from HBM rather than L2), with the moduli count the autotuner
measures for this K band (config.moduli_choice); error_vs_dd checks that
count against the double-double oracle in the same run, next to the plain
kernel and the K rule's count (ozaki_rule_moduli).  `e2e` = the same metric through the
public XKBlas API (xkblas_dgemm_async + xkblas_memory_coherent_async +
xkblas_sync with pinned host buffers; host->device copies of A and B and the
device->host copy of C inside the timed region, caches dropped every step).
Multi-GPU (torchrun): independent replicas, one per GPU, time = max over
ranks (weak scaling; the path has no exchange step).
Inputs are synthetic (seeded numpy generator); the CPU baseline and the
accuracy check against the double-double oracle use bounded samples.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = N = K = 16384
EMAX = 20
METRIC = "FP64-accurate TFLOP/s (DGEMM/DTRSM/DSYRK): Ozaki-TC vs plain DMMA, 1 B200"
WORKLOAD = "dgemm_nn_16384_expspread20_ozaki"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
            "fallback"


def gen_expspread(rows, cols, seed, by_col):
    """u * 2^e, u ~ U[-1,1], e ~ U{-EMAX..EMAX} per row (or per column)."""
    rng = np.random.default_rng(seed)
    e = rng.integers(-EMAX, EMAX + 1, size=cols if by_col else rows)
    A = np.asfortranarray(rng.uniform(-1.0, 1.0, size=(rows, cols)))
    if by_col:
        A *= np.ldexp(1.0, e)[None, :]
    else:
        A *= np.ldexp(1.0, e)[:, None]
    return A


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, idx):
        self.idx = idx
        self.proc = None
        self.out = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_rows(step_s):
    """Rows of the workload's A for one OpenBLAS dgemm_ row-block step of
    about step_s seconds on all host threads (multiple of 64, 256..M)."""
    import oracle as O
    O.blas_open(threads=os.cpu_count())
    B = gen_expspread(K, N, 2, True)
    rows = 256
    A = gen_expspread(rows, K, 1, False)
    C = np.zeros((rows, N), order="F")
    O.native_gemm(O.NOTRANS, O.NOTRANS, 1.0, A, B, 0.0, C)  # first call: thread start-up
    t0 = time.perf_counter()
    O.native_gemm(O.NOTRANS, O.NOTRANS, 1.0, A, B, 0.0, C)
    t1 = time.perf_counter() - t0
    rows = int(max(256, min(M, rows * step_s / max(t1, 1e-3)))) // 64 * 64
    return rows, B


def cpu_gemm_steps(rows, B, nsteps):
    """Seconds of each of nsteps OpenBLAS dgemm_ calls (the call
    xkblas_dgemm_native makes, restated by the oracle) on the first `rows`
    rows of the workload's A times its full B."""
    import oracle as O
    A = gen_expspread(rows, K, 1, False)
    C = np.zeros((rows, N), order="F")
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        O.native_gemm(O.NOTRANS, O.NOTRANS, 1.0, A, B, 0.0, C)
        times.append(time.perf_counter() - t0)
    return times


CPU_STEP_S = 2.0  # seconds of host BLAS per sampled step (both arms)


def cpu_sample_text(path, rows, t):
    return ("OpenBLAS %s dgemm_ (the call xkblas_dgemm_native makes) on a %d x %d x %d row "
            "block of the %d^3 workload per step, median step %.2f s"
            % (os.path.basename(path or "libopenblas"), rows, N, K, M, t))


def cpu_baseline(nsteps=3):
    """The reference's CPU path on the box's host cores: the same row-block
    steps as the reference arm (--impl reference), median of nsteps."""
    import oracle as O
    rows, B = cpu_rows(CPU_STEP_S)
    t = statistics.median(cpu_gemm_steps(rows, B, nsteps))
    return {"value": 2.0 * rows * N * K / t / 1e12, "unit": "TFLOP/s", "cores": os.cpu_count(),
            "kind": "port", "sample": cpu_sample_text(O.find_openblas(), rows, t)}


def dd_errors(A, B, Cs, nrow=16, ncol=256, seed=7):
    """Componentwise error |C - C_dd| / (|A||B|) on sampled entries, against
    the double-double oracle (checker only)."""
    import oracle as O
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(M, nrow, replace=False))
    cols = np.sort(rng.choice(N, ncol, replace=False))
    dd = O.gemm_dd(O.NOTRANS, O.NOTRANS, 1.0, A, B, 0.0, None, rows, cols)
    scale = np.abs(A[rows]) @ np.abs(B[:, cols])
    out = {}
    for name, C in Cs.items():
        e = np.abs(C[np.ix_(rows, cols)] - dd) / scale
        out[name] = {"max": float(e.max()), "mean": float(e.mean())}
    return out


from xkblas_b200 import GemmArgs, TraceRec  # include/xkb_cuda.h structs

def _cm(t):
    """Device tensor holding a column-major matrix (a row-major tensor of its
    transpose) -> Fortran-ordered host array of that matrix."""
    return np.asfortranarray(t.cpu().numpy().T)


def _pick(n, k, seed):
    return np.sort(np.random.default_rng(seed).choice(n, min(n, k), replace=False))


def dd_gemm_error(C, ta, tb, alpha, A, B, beta, C0, rows, cols, mask=None):
    """max |C - C_dd| / (|alpha||op(A)||op(B)| + |beta||C0|) over sampled
    entries (C_dd: the double-double oracle rounded once)."""
    import oracle as O
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    C0 = np.asfortranarray(C0) if C0 is not None else None
    dd = O.gemm_dd(ta, tb, alpha, A, B, beta, C0, rows, cols)
    opA = A if ta == O.NOTRANS else (A.T if ta == O.TRANS else A.conj().T)
    opB = B if tb == O.NOTRANS else (B.T if tb == O.TRANS else B.conj().T)
    scale = abs(alpha) * (np.abs(opA[rows]) @ np.abs(opB[:, cols]))
    if C0 is not None and beta != 0:
        scale = scale + abs(beta) * np.abs(C0[np.ix_(rows, cols)])
    e = np.abs(C[np.ix_(rows, cols)] - dd) / scale
    return float(e[mask].max() if mask is not None else e.max())


def dd_backward_error(L, R, P, rows, cols, alpha=1.0):
    """Componentwise backward error of a solve or factorization on sampled
    entries: |L R - alpha P| / (|L||R| + |alpha||P|), the residual in
    double-double (L R - alpha P = 0 defines the exact answer)."""
    import oracle as O
    L, R, P = np.asfortranarray(L), np.asfortranarray(R), np.asfortranarray(P)
    res = O.gemm_dd(O.NOTRANS, O.NOTRANS, 1.0, L, R, -alpha, P, rows, cols)
    den = np.abs(L[rows]) @ np.abs(R[:, cols]) + abs(alpha) * np.abs(P[np.ix_(rows, cols)])
    return float(np.max(np.abs(res) / den))



def other_configs(lib, torch, dev, sp, stream):
    """The remaining benchmark workloads, device resident, plain FP64
    DMMA vs Ozaki: DGEMM 1024^3 (alpha 1.5, beta -0.5), DTRSM L/L/N/N 4096
    (alpha 2, A lower + 4096 on the diagonal), DSYRK and ZHERK L/N
    N = K = 8192 (alpha = beta = 1).  Flops: reference blas/flops.h."""
    g = torch.Generator(device=dev).manual_seed(1234)
    out = {}

    def u(*shape, cplx=False):
        if cplx:
            return torch.complex(torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) - 0.5,
                                 torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) - 0.5)
        return torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) - 0.5

    def timed(fn, reps, reset=None):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        # the inputs were made on torch's default stream; the library's calls
        # (and the resets) run on `stream`
        torch.cuda.synchronize()
        if reset:
            reset()
        assert fn() == 0
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            if reset:
                reset()
            ev0.record(stream)
            assert fn() == 0
            ev1.record(stream)
            torch.cuda.synchronize()
            tot += ev0.elapsed_time(ev1)
        return tot / reps

    # config 1: DGEMM NN 1024^3
    n = 1024
    A, B, C0 = u(n, n), u(n, n), u(n, n)
    C = C0.clone()
    ga = GemmArgs(1, 0, 0, n, n, n, A.data_ptr(), n, B.data_ptr(), n, C.data_ptr(), n)
    ga.alpha[0], ga.beta[0] = 1.5, -0.5
    fl = 2.0 * n ** 3
    with torch.cuda.stream(stream):
        rs = lambda: C.copy_(C0)
        to = timed(lambda: lib.xkb_cuda_ozaki_gemm(ctypes.byref(ga), 0, sp), 10, rs)
        Co = _cm(C)
        tp = timed(lambda: lib.xkb_cuda_gemm(ctypes.byref(ga), sp), 10, rs)
        Cp = _cm(C)
    hA, hB, hC0 = _cm(A), _cm(B), _cm(C0)
    r, c = _pick(n, 64, 1), _pick(n, 64, 2)
    out["dgemm_nn_1024_nb256"] = {
        "plain_tflops": fl / tp / 1e9, "ozaki_tflops": fl / to / 1e9, "plain_ms": tp, "ozaki_ms": to,
        "error_vs_dd": {k: dd_gemm_error(X_, 111, 111, 1.5, hA, hB, -0.5, hC0, r, c)
                        for k, X_ in (("plain", Cp), ("ozaki", Co))},
        "error_kind": "componentwise |C - C_dd| / (|alpha||A||B| + |beta||C0|), 64 x 64 sampled"}
    del A, B, C, C0
    # config 2: DTRSM L/L/N/N 4096, alpha 2
    n = 4096
    A = torch.tril(u(n, n)) + n * torch.eye(n, device=dev, dtype=torch.float64)
    Acm = A.t().contiguous()  # row-major storage of the column-major lower matrix
    B0 = u(n, n)
    B = B0.clone()
    al = (ctypes.c_double * 2)(2.0, 0.0)
    al = ctypes.cast(al, ctypes.POINTER(ctypes.c_double))
    fl = float(n) * n * (n + 1)
    with torch.cuda.stream(stream):
        rs = lambda: B.copy_(B0)
        tp = timed(lambda: lib.xkb_cuda_trsm(1, 0, 1, 0, 0, n, n, al, Acm.data_ptr(), n,
                                             B.data_ptr(), n, 0, sp), 5, rs)
        Xp = _cm(B)
        to = timed(lambda: lib.xkb_cuda_trsm(1, 0, 1, 0, 0, n, n, al, Acm.data_ptr(), n,
                                             B.data_ptr(), n, 1024, sp), 5, rs)
        Xo = _cm(B)
    hA, hB0 = np.asfortranarray(A.cpu().numpy()), _cm(B0)
    r, c = _pick(n, 48, 3), _pick(n, 48, 4)
    out["dtrsm_llnn_4096"] = {
        "plain_tflops": fl / tp / 1e9, "ozaki_tflops": fl / to / 1e9, "plain_ms": tp, "ozaki_ms": to,
        "error_vs_dd": {k: dd_backward_error(hA, X_, hB0, r, c, alpha=2.0)
                        for k, X_ in (("plain", Xp), ("ozaki", Xo))},
        "error_kind": "componentwise backward error |A X - 2 B| / (|A||X| + 2|B|), residual in "
                      "double-double, 48 x 48 sampled"}
    del A, Acm, B, B0
    # config 3: DSYRK / ZHERK lower, no-trans, N = K = 8192
    n = 8192
    for name, cplx, code, mult in (("dsyrk_ln_8192", False, 1, 1.0), ("zherk_ln_8192", True, 3, 4.0)):
        A = u(n, n, cplx=cplx)
        # C symmetric / Hermitian with the same entry distribution: the lower
        # triangle of a uniform matrix mirrored (conjugated), real diagonal
        U = u(n, n, cplx=cplx)
        H = torch.tril(U) + torch.tril(U, -1).conj().t()
        if cplx:
            H.diagonal().imag.zero_()
        C0 = H.t().contiguous()  # column-major storage of H
        del U, H
        C = C0.clone()
        gs = GemmArgs(code, 0, 2 if cplx else 1, n, n, n, A.data_ptr(), n, A.data_ptr(), n,
                      C.data_ptr(), n)
        gs.alpha[0], gs.beta[0] = 1.0, 1.0
        gs.uplo = 1  # lower
        gs.herm_diag = 1 if cplx else 0
        fl = mult * n * (n + 1.0) * n
        with torch.cuda.stream(stream):
            rs = lambda: C.copy_(C0)
            tp = timed(lambda: lib.xkb_cuda_gemm(ctypes.byref(gs), sp), 2, rs)
            Cp = _cm(C)
            to = timed(lambda: lib.xkb_cuda_ozaki_gemm(ctypes.byref(gs), 0, sp), 3, rs)
            Co = _cm(C)
        hA, hC0 = _cm(A), _cm(C0)
        r = _pick(n, 64, 5)
        c = np.unique(np.concatenate([r[:32], _pick(n, 32, 6)]))
        low = r[:, None] >= c[None, :]
        out[name] = {
            "plain_tflops": fl / tp / 1e9, "ozaki_tflops": fl / to / 1e9, "plain_ms": tp,
            "ozaki_ms": to,
            "error_vs_dd": {k: dd_gemm_error(X_, 111, 113 if cplx else 112, 1.0, hA, hA, 1.0, hC0,
                                             r, c, mask=low)
                            for k, X_ in (("plain", Cp), ("ozaki", Co))},
            "error_kind": "componentwise, lower-triangle entries of a 64 x 64 sample"}
        del A, C, C0, Cp, Co, hA, hC0
    # Cholesky (a next-row driver on the same kernels): DPOTRF lower 8192,
    # A = B B^T / n + I; flops n^3/3 + n^2/2 + n/6 (reference flops.h)
    n = 8192
    Bm = u(n, n)
    A0 = Bm @ Bm.t() / n + torch.eye(n, device=dev, dtype=torch.float64)
    A = A0.clone()
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    with torch.cuda.stream(stream):
        rs = lambda: A.copy_(A0)
        tp = timed(lambda: lib.xkb_cuda_potrf(1, 1, n, ctypes.c_void_p(A.data_ptr()), n,
                                              ctypes.c_void_p(info.data_ptr()), 0, sp), 3, rs)
        info_p = int(info.item())
        Lp = np.tril(_cm(A))
        # tensor-op mode: updates with all dimensions >= 2048 in the Ozaki form
        to = timed(lambda: lib.xkb_cuda_potrf(1, 1, n, ctypes.c_void_p(A.data_ptr()), n,
                                              ctypes.c_void_p(info.data_ptr()), 2048, sp), 3, rs)
        Lo = np.tril(_cm(A))
    fl = n ** 3 / 3.0 + n * n / 2.0 + n / 6.0
    hA0 = _cm(A0)
    r, c = _pick(n, 48, 7), _pick(n, 48, 8)
    out["dpotrf_l_8192"] = {
        "plain_tflops": fl / tp / 1e9, "ozaki_tflops": fl / to / 1e9, "plain_ms": tp, "ozaki_ms": to,
        "info": max(info_p, int(info.item())),
        "error_vs_dd": {k: dd_backward_error(L_, np.asfortranarray(L_.T), hA0, r, c)
                        for k, L_ in (("plain", Lp), ("ozaki", Lo))},
        "error_kind": "componentwise backward error |L L^T - A| / (|L||L^T| + |A|), residual in "
                      "double-double, 48 x 48 sampled"}
    del Lp, Lo, hA0
    del Bm, A0, A, info
    # LU without pivoting (the zgetrf_nopiv tile driver): DGETRF 8192 on a
    # diagonally dominant matrix; flops 2n^3/3 - n^2/2 + 5n/6 (reference flops.h)
    A0 = u(n, n) + n * torch.eye(n, device=dev, dtype=torch.float64)
    A = A0.clone()
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    with torch.cuda.stream(stream):
        rs = lambda: A.copy_(A0)
        tp = timed(lambda: lib.xkb_cuda_getrf_nopiv(1, n, ctypes.c_void_p(A.data_ptr()), n,
                                                    ctypes.c_void_p(info.data_ptr()), 0, sp), 3, rs)
        info_p = int(info.item())
        LUp = _cm(A)
        to = timed(lambda: lib.xkb_cuda_getrf_nopiv(1, n, ctypes.c_void_p(A.data_ptr()), n,
                                                    ctypes.c_void_p(info.data_ptr()), 2048, sp), 3, rs)
        LUo = _cm(A)
    fl = 2.0 * n ** 3 / 3.0 - n * n / 2.0 + 5.0 * n / 6.0
    hA0 = _cm(A0)
    r, c = _pick(n, 48, 9), _pick(n, 48, 10)

    def lu_err(LU):
        L = np.asfortranarray(np.tril(LU, -1) + np.eye(n))
        return dd_backward_error(L, np.asfortranarray(np.triu(LU)), hA0, r, c)

    out["dgetrf_nopiv_8192"] = {
        "plain_tflops": fl / tp / 1e9, "ozaki_tflops": fl / to / 1e9, "plain_ms": tp, "ozaki_ms": to,
        "info": max(info_p, int(info.item())),
        "error_vs_dd": {"plain": lu_err(LUp), "ozaki": lu_err(LUo)},
        "error_kind": "componentwise backward error |L U - A| / (|L||U| + |A|), residual in "
                      "double-double, 48 x 48 sampled"}
    del LUp, LUo, hA0
    del A0, A, info
    torch.cuda.empty_cache()
    return out


class BatchOp(ctypes.Structure):
    """xkb_batch_op of include/xkb_cuda.h."""
    _fields_ = [("kind", ctypes.c_int), ("dtype", ctypes.c_int), ("opA", ctypes.c_int),
                ("opB", ctypes.c_int), ("side", ctypes.c_int), ("uplo", ctypes.c_int),
                ("trans", ctypes.c_int), ("diag", ctypes.c_int), ("M", ctypes.c_int),
                ("N", ctypes.c_int), ("K", ctypes.c_int),
                ("A", ctypes.c_void_p), ("lda", ctypes.c_long),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_long),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_long),
                ("alpha", ctypes.c_double * 2), ("beta", ctypes.c_double * 2)]


def batch_config(lib, torch, dev, sp, stream, ncalls=2000, seed=2024, reps=5):
    """The mixed-call workload: `ncalls` independent calls, 70% DGEMM NN,
    20% DTRSM left/lower/no-trans/non-unit with a diagonally dominant A, 10%
    ZGEMM NN; M, N, K log-uniform in [64, 2048] (one seeded generator),
    leading dimensions = row counts (mostly odd, so most operands are not
    16-byte aligned), alpha = beta = 1.  Run as ONE persistent launch of the
    tile-task executor (xkb_cuda_batch), device resident; reported: aggregate
    TFLOP/s (sum of flops, reference blas/flops.h, / launch time), per-call
    completion latency p50/p99 from the launch start (device timestamps), and
    the same calls issued one launch per call (xkb_cuda_gemm / xkb_cuda_trsm)
    on the same stream for comparison.  The timed submissions replay the
    batch's CUDA graph (kept from the second submission); the first
    submission, which builds and uploads the task list, is reported apart."""
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev).manual_seed(seed)
    f64, c128 = torch.float64, torch.complex128

    def lu():
        return int(np.exp(rng.uniform(np.log(64), np.log(2048))))

    def u(r, c):  # column-major r x c (a row-major c x r tensor)
        return torch.rand(c, r, generator=g, device=dev, dtype=f64) - 0.5

    ops, keep, flops = [], [], 0.0
    kinds = {"dgemm": 0, "dtrsm": 0, "zgemm": 0}
    for _ in range(ncalls):
        r = rng.random()
        o = BatchOp()
        if r < 0.7 or r >= 0.9:
            cplx = r >= 0.9
            m, n, k = lu(), lu(), lu()
            A, B, C = u(m, k), u(k, n), u(m, n)
            if cplx:
                A = torch.complex(A, u(m, k))
                B = torch.complex(B, u(k, n))
                C = torch.complex(C, u(m, n))
            o.kind, o.dtype, o.opA, o.opB, o.M, o.N, o.K = 0, 3 if cplx else 1, 0, 0, m, n, k
            o.A, o.lda, o.B, o.ldb, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m
            o.alpha[0] = 1.0
            o.beta[0] = 1.0
            flops += (8.0 if cplx else 2.0) * m * n * k
            kinds["zgemm" if cplx else "dgemm"] += 1
            keep.append((A, B, C))
        else:
            m, n = lu(), lu()
            L = torch.tril(u(m, m).t()) + m * torch.eye(m, device=dev, dtype=f64)
            A = L.t().contiguous()  # column-major storage of the lower L
            B = u(m, n)
            o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, 1, 0, 0, m, n
            o.A, o.lda, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), m
            o.alpha[0] = 1.0
            flops += float(n) * m * (m + 1)
            kinds["dtrsm"] += 1
            keep.append((A, B))
        ops.append(o)
    arr = (BatchOp * len(ops))(*ops)
    lib.xkb_cuda_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.xkb_cuda_batch_latency.argtypes = [ctypes.c_void_p, ctypes.c_int]
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # accuracy sample: the first calls of each kind, inputs copied before the
    # first submission (later submissions accumulate into the outputs)
    sample = {"dgemm": [], "dtrsm": [], "zgemm": []}
    for i, o in enumerate(ops):
        kind = "dtrsm" if o.kind == 1 else ("zgemm" if o.dtype == 3 else "dgemm")
        if len(sample[kind]) < 4:
            sample[kind].append((i, [_cm(t) for t in keep[i]]))
    # first submission: host task construction + task upload + launch; the
    # second is kept as a CUDA graph, later ones replay it
    lib.xkb_cuda_batch_release()
    torch.cuda.synchronize()
    ev0.record(stream)
    h0 = time.perf_counter()
    assert lib.xkb_cuda_batch(ctypes.addressof(arr), len(ops), 0, sp) == 0
    host_first = (time.perf_counter() - h0) * 1e3
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_first = ev0.elapsed_time(ev1)
    errs = {}
    for kind, lst in sample.items():
        e = 0.0
        for i, host in lst:
            out = _cm(keep[i][-1])
            r, c = _pick(out.shape[0], 16, i), _pick(out.shape[1], 16, i + 1)
            if kind == "dtrsm":
                # host[0]: the lower L (its column-major storage read back)
                e = max(e, dd_backward_error(host[0], out, host[1], r, c))
            else:
                A_, B_, C0_ = host
                e = max(e, dd_gemm_error(out, 111, 111, 1.0, A_, B_, 1.0, C0_, r, c))
        errs[kind] = e
    k0 = lib.xkb_cuda_kernel_count()
    for _ in range(3):  # warm-up
        assert lib.xkb_cuda_batch(ctypes.addressof(arr), len(ops), 0, sp) == 0
    torch.cuda.synchronize()
    times, host = [], []
    for _ in range(reps):
        ev0.record(stream)
        h0 = time.perf_counter()
        assert lib.xkb_cuda_batch(ctypes.addressof(arr), len(ops), 0, sp) == 0
        host.append((time.perf_counter() - h0) * 1e3)
        ev1.record(stream)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
    launches = (lib.xkb_cuda_kernel_count() - k0) // (reps + 3)
    cached = lib.xkb_cuda_batch_cached()
    lat = (ctypes.c_double * len(ops))()
    assert lib.xkb_cuda_batch_latency(ctypes.addressof(lat), len(ops)) == 0
    lat = np.array(list(lat))
    ms = statistics.median(times)
    # one launch per call, same calls and stream
    al = (ctypes.c_double * 2)(1.0, 0.0)
    alp = ctypes.cast(al, ctypes.POINTER(ctypes.c_double))
    gas = []
    for o in ops:
        if o.kind == 0:
            ga = GemmArgs(o.dtype, 0, 0, o.M, o.N, o.K, o.A, o.lda, o.B, o.ldb, o.C, o.ldc)
            ga.alpha[0] = 1.0
            ga.beta[0] = 1.0
            gas.append(ga)
        else:
            gas.append(None)

    def per_call():
        bad = 0
        for o, ga in zip(ops, gas):
            if ga is not None:
                bad += lib.xkb_cuda_gemm(ctypes.byref(ga), sp) != 0
            else:
                bad += lib.xkb_cuda_trsm(1, 0, 1, 0, 0, o.M, o.N, alp, o.A, o.lda, o.C, o.ldc, 0,
                                         sp) != 0
        return bad

    per_call()
    torch.cuda.synchronize()
    ev0.record(stream)
    rejected = per_call()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_seq = ev0.elapsed_time(ev1)
    del keep
    torch.cuda.empty_cache()
    return {"workload": "batch_%d_calls_70dgemm_20dtrsm_10zgemm_loguniform_64_2048" % ncalls,
            "calls": kinds, "gflop": flops / 1e9,
            "tflops": flops / ms / 1e9, "ms_per_batch": ms, "launches_per_batch": int(launches),
            "graph_replay": bool(cached), "host_ms_per_submission": statistics.median(host),
            "first_submission": {"ms": ms_first, "tflops": flops / ms_first / 1e9,
                                 "host_ms": host_first},
            "latency_ms_p50": float(np.percentile(lat, 50)),
            "latency_ms_p99": float(np.percentile(lat, 99)),
            "per_call_launches": {"tflops": flops / ms_seq / 1e9, "ms": ms_seq,
                                  "launches": len(ops), "rejected_calls": int(rejected)},
            "speedup_vs_per_call": ms_seq / ms,
            "error_vs_dd": errs,
            "error_kind": "max over the first 4 calls of each kind, 16 x 16 sampled entries each: "
                          "gemm componentwise |C - C_dd| / (|A||B| + |C0|), trsm componentwise "
                          "backward error with the residual in double-double"}


def batch_config_e2e(lib, torch, ncalls=2000, seed=2024, reps=2):
    """The mixed-call workload of batch_config (same sizes, same generator)
    through the public XKBlas API with host-resident, user-owned matrices:
    every call is xkblas_dgemm_async / xkblas_ztrsm... as the reference's
    users issue them, then memory_coherent_async on every output and one
    xkblas_sync, all inside the timed region (host->device copies of every
    operand and device->host copies of every output included; the device
    caches are dropped between repetitions).  The library queues the calls
    and runs them as executor batches."""
    rng = np.random.default_rng(seed)

    def lu():
        return int(np.exp(rng.uniform(np.log(64), np.log(2048))))

    plan = []
    for _ in range(ncalls):  # the same draw sequence as batch_config
        r = rng.random()
        if r < 0.7 or r >= 0.9:
            plan.append(("zgemm" if r >= 0.9 else "dgemm", lu(), lu(), lu()))
        else:
            plan.append(("dtrsm", lu(), lu(), 0))
    words = 0
    for kind, m, n, k in plan:
        w = 2 if kind == "zgemm" else 1
        words += w * ((m * k + k * n + m * n) if kind != "dtrsm" else (m * m + m * n))
    buf = torch.empty(words, dtype=torch.float64, pin_memory=True).numpy()
    fill = np.random.default_rng(seed + 1)
    for i in range(0, words, 1 << 26):
        seg = buf[i:i + (1 << 26)]
        fill.random(out=seg)
        seg -= 0.5
    mats, off, flops, h2d, d2h = [], 0, 0.0, 0, 0

    def take(rows, cols, cplx):
        nonlocal off
        w = 2 if cplx else 1
        a = buf[off:off + w * rows * cols]
        off += w * rows * cols
        a = a.view(np.complex128) if cplx else a
        return a.reshape(cols, rows).T  # Fortran-ordered rows x cols view

    for kind, m, n, k in plan:
        if kind == "dtrsm":
            A, B = take(m, m, False), take(m, n, False)
            A[np.arange(m), np.arange(m)] += m  # diagonally dominant lower triangle
            mats.append((kind, m, n, 0, A, None, B))
            flops += float(n) * m * (m + 1)
            h2d += 8 * (m * m + m * n)
            d2h += 8 * m * n
        else:
            c = kind == "zgemm"
            A, B, C = take(m, k, c), take(k, n, c), take(m, n, c)
            mats.append((kind, m, n, k, A, B, C))
            flops += (8.0 if c else 2.0) * m * n * k
            es = 16 if c else 8
            h2d += es * (m * k + k * n + m * n)
            d2h += es * m * n
    one_d = ctypes.c_double(1.0)
    one_z = (ctypes.c_double * 2)(1.0, 0.0)
    P = ctypes.c_void_p

    phases = {}

    def run():
        t0 = time.perf_counter()
        for kind, m, n, k, A, B, C in mats:
            if kind == "dgemm":
                r = lib.xkblas_dgemm_async(111, 111, m, n, k, ctypes.byref(one_d),
                                           P(A.ctypes.data), m, P(B.ctypes.data), k,
                                           ctypes.byref(one_d), P(C.ctypes.data), m)
            elif kind == "zgemm":
                r = lib.xkblas_zgemm_async(111, 111, m, n, k, one_z, P(A.ctypes.data), m,
                                           P(B.ctypes.data), k, one_z, P(C.ctypes.data), m)
            else:
                r = lib.xkblas_dtrsm_async(141, 122, 111, 131, m, n, ctypes.byref(one_d),
                                           P(A.ctypes.data), m, P(C.ctypes.data), m)
            assert r == 0, (kind, r)
        t1 = time.perf_counter()
        for kind, m, n, k, A, B, C in mats:
            es = 16 if kind == "zgemm" else 8
            assert lib.xkblas_memory_coherent_async(0, 0, ctypes.c_size_t(m), ctypes.c_size_t(n),
                                                    P(C.ctypes.data), ctypes.c_size_t(m),
                                                    ctypes.c_size_t(es)) == 0
        t2 = time.perf_counter()
        assert lib.xkblas_sync() == 0
        t3 = time.perf_counter()
        # host time to issue the calls, to issue the coherence requests, and
        # the wait in xkblas_sync
        phases.update(issue_ms=(t1 - t0) * 1e3, coherent_ms=(t2 - t1) * 1e3,
                      sync_wait_ms=(t3 - t2) * 1e3)

    import xkblas_b200 as X
    st = X.Stats()
    lib.xkblas_reset_stats()
    run()  # warm-up (allocations, pinned staging)
    lib.xkblas_memory_invalidate_caches()
    times, best = [], None
    for _ in range(reps):
        lib.xkblas_reset_stats()
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
        if times[-1] == min(times):
            best = dict(phases)
        lib.xkblas_get_stats(ctypes.byref(st))
        lib.xkblas_memory_invalidate_caches()
    sec = min(times)
    out = {"value": flops / sec / 1e12, "unit": "TFLOP/s", "ms": sec * 1e3,
           "h2d_bytes": h2d, "d2h_bytes": d2h, "batches": int(st.batches),
           "batched_calls": int(st.batched_calls),
           "phases_ms": {k: round(v, 2) for k, v in best.items()}}
    del mats, buf
    return out


def workload_config(world):
    """The `config` both arms print (the workload only)."""
    return {"workload": WORKLOAD, "M": M, "N": N, "K": K, "exp_spread": EMAX,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs 2 GiB each > 126 MB L2 (no flush needed)"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (the host BLAS
    through xkblas_dgemm_native's Fortran symbol), all host threads, on rank
    0: warm-up + timed steps of the same row block cpu_baseline uses; the
    value is the median step."""
    if rank != 0:
        return
    import oracle as O
    rows, B = cpu_rows(CPU_STEP_S)
    times = cpu_gemm_steps(rows, B, args.warmup + args.steps)[args.warmup:]
    t = statistics.median(times)
    v = 2.0 * rows * N * K / t / 1e12
    sample = cpu_sample_text(O.find_openblas(), rows, t)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(world),
            "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "step_ms": {"min": min(times) * 1e3, "median": t * 1e3, "max": max(times) * 1e3}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the CPU baseline and the double-double accuracy sample")
    ap.add_argument("--size", type=int, default=16384,
                    help="M = N = K (the benchmark workload is 16384; smaller sizes for profiling)")
    args = ap.parse_args()
    global M, N, K, WORKLOAD
    if args.size != M:
        M = N = K = args.size
        WORKLOAD = "dgemm_nn_%d_expspread20_ozaki" % args.size
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    os.environ["XKBLAS_GPUSET"] = str(local)
    import torch
    torch.cuda.set_device(local)
    from xkblas_b200.replicas import Replicas
    reps = Replicas(backend="nccl", timeout_s=300)  # one independent problem per GPU

    import xkblas_b200 as X
    lib = X.lib()
    X.init()
    lib.xkb_trace_take.argtypes = [ctypes.POINTER(TraceRec), ctypes.c_int]

    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    A = gen_expspread(M, K, 1 + 10 * rank, False)
    B = gen_expspread(K, N, 2 + 10 * rank, True)
    # column-major A (M x K) == row-major torch (K, M)
    dA = torch.from_numpy(A.T).to(f"cuda:{local}")
    dB = torch.from_numpy(B.T).to(f"cuda:{local}")
    dC = torch.zeros(N, M, dtype=torch.float64, device=f"cuda:{local}")
    dP = torch.zeros_like(dC)
    torch.cuda.synchronize()

    def args_for(C):
        g = GemmArgs(1, 0, 0, M, N, K, dA.data_ptr(), M, dB.data_ptr(), K, C.data_ptr(), M)
        g.alpha[0] = 1.0
        return g

    g_oz = args_for(dC)
    g_pl = args_for(dP)
    # moduli count: the autotuner's measured choice for this K band (the
    # smallest count at most half as far from a 16-moduli product as the
    # plain kernel, on a 1024 x 1024 x K sample of the same distribution);
    # the K rule's count is timed beside it in the extras
    from xkblas_b200.autotune import choose_moduli
    nmod_rule = lib.xkb_ozaki_default_moduli(K)
    nmod, tune_err_plain, tune_errs = choose_moduli(lib, K, 1024, 1024, sp)
    torch.cuda.synchronize()
    # the measured count becomes the tuning table's entry for this K band:
    # the floor of the data rule, which picks the count on the device from
    # the operands' concentration (nmod = 0 below)
    lib.xkb_tune_set(b"ozaki_moduli_k<=%d" % K, float(nmod))

    def barrier():
        reps.barrier(torch.cuda.synchronize)

    maxreduce = reps.max

    # the other configurations first: each is timed on its own, not in the
    # wake of the power-capped 16384^3 runs
    extras = {}
    if rank == 0 and not args.no_extra:
        extras = other_configs(lib, torch, f"cuda:{local}", sp, stream)
        extras["batch_2000_mixed"] = batch_config(lib, torch, f"cuda:{local}", sp, stream)
        extras["batch_2000_mixed"]["e2e_public_api"] = batch_config_e2e(lib, torch)
    X.ozaki_counts(reset=True)  # the reported counts cover the headline calls only

    # ---- device-resident Ozaki steps --------------------------------------
    k0 = lib.xkb_cuda_kernel_count()
    for _ in range(args.warmup):
        assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g_oz), 0, sp) == 0
    barrier()
    lib.xkb_trace_enable(1)
    lib.xkb_trace_take(None, 0)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    k1 = lib.xkb_cuda_kernel_count()
    with Clocks(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g_oz), 0, sp) == 0
        ev1.record(stream)
        barrier()
    launches = lib.xkb_cuda_kernel_count() - k1
    ms = maxreduce(ev0.elapsed_time(ev1) / args.steps)
    recs = (TraceRec * 256)()
    n = lib.xkb_trace_take(recs, 256)
    lib.xkb_trace_enable(0)
    gemm_ms = [recs[i].ms_gemm for i in range(n) if recs[i].op == b"ozaki_gemm"]
    conv_ms = [recs[i].ms_convert for i in range(n) if recs[i].op == b"ozaki_gemm"]
    crt_ms = [recs[i].ms_crt for i in range(n) if recs[i].op == b"ozaki_gemm"]
    flops = 2.0 * M * N * K
    value = world * flops / (ms * 1e-3) / 1e12
    deverr = lib.xkb_cuda_take_device_error()

    # ---- roofline of the dominant kernel (INT8 tensor-core GEMM, all moduli)
    pk, pk_src = peaks()
    # dense INT8 rate = 2x dense BF16 on B200.  The INT8 GEMM runs ~50 ms per
    # launch, back to back inside a long step under the 1 kW power cap: the
    # sustained BF16 figure is its denominator (the burst one is reported too)
    int8_peak = 2.0 * pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
    int8_peak_burst = 2.0 * pk["bf16_tflops"]
    gm = statistics.mean(gemm_ms) if gemm_ms else float("nan")
    # the count the device chose for the timed calls (same inputs every step)
    oz_calls, oz_msum, oz_fb, nm_chosen = X.ozaki_counts()
    int8_ops = 2.0 * M * N * K * nm_chosen  # algorithmic INT8 ops per launch (all moduli)
    achieved = int8_ops / (gm * 1e-3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("k_oz_gemm_bytes_per_launch_16384")
        except Exception:
            traffic = None

    # ---- plain DMMA reference point on the same inputs ---------------------
    lib.xkb_cuda_gemm(ctypes.byref(g_pl), sp)
    barrier()
    ev0.record(stream)
    steps_plain = 2
    for _ in range(steps_plain):
        lib.xkb_cuda_gemm(ctypes.byref(g_pl), sp)
    ev1.record(stream)
    barrier()
    ms_plain = maxreduce(ev0.elapsed_time(ev1) / steps_plain)
    plain_tflops = world * flops / (ms_plain * 1e-3) / 1e12
    fp64_nominal = 148 * 128 * 1.965e9 / 1e12  # DMMA: 64 FMA/clk/SM at max clock

    # ---- end to end through the public API ---------------------------------
    hA = X.pinned_empty((M, K), np.float64)
    hB = X.pinned_empty((K, N), np.float64)
    hC = X.pinned_empty((M, N), np.float64)
    hA[...] = A
    hB[...] = B
    X.set_modemath(X.XKBLAS_TENSOR_OP_MATH)
    # the same moduli count through the runtime: the tuning-table entry for
    # this K band (what XKBLAS_TUNE_FILE from the autotuner provides)
    one = np.array([1.0])
    zero = np.array([0.0])
    P = ctypes.c_void_p

    def e2e_step():
        r = lib.xkblas_dgemm_async(111, 111, M, N, K, P(one.ctypes.data), P(hA.ctypes.data), M,
                                   P(hB.ctypes.data), K, P(zero.ctypes.data), P(hC.ctypes.data),
                                   M)
        assert r == 0
        lib.xkblas_memory_coherent_async(0, 0, M, N, P(hC.ctypes.data), M, 8)
        assert lib.xkblas_sync() == 0
        lib.xkblas_memory_invalidate_caches()

    e2e_steps = args.steps
    for _ in range(2):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    t_e2e = maxreduce((time.perf_counter() - t0) / e2e_steps)
    X.set_modemath(X.XKBLAS_DEFAULT_MATH)
    e2e_value = world * flops / t_e2e / 1e12

    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(world),
        "ozaki": {"moduli": nm_chosen,
                  "moduli_choice": "chosen on the device per call (nmod = 0): the smallest count "
                                   "with H >= 53 + log2(2.31 rho_max sigma_max), at least the "
                                   "tuning table's %d for this K band" % nmod,
                  "tuned_floor": nmod,
                  "tuned_floor_choice": "xkblas_b200.autotune.choose_moduli on a 1024x1024x%d "
                                        "sample: plain err %.2e, %s" % (
                                            K, tune_err_plain,
                                            ", ".join("%d: %.2e" % e for e in tune_errs)),
                  "device_counts": {"calls": oz_calls, "moduli_sum": oz_msum,
                                    "plain_fallbacks": oz_fb}},
        "e2e": {"value": e2e_value, "unit": "TFLOP/s",
                "h2d_bytes_per_step": 2 * M * K * 8, "d2h_bytes_per_step": M * N * 8,
                "ms_per_step": t_e2e * 1e3},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "roofline": {"bound": "tensor", "kernel": "k_oz_gemm (INT8 tcgen05, all moduli)",
                     "achieved": achieved, "peak": int8_peak, "unit": "TFLOP/s",
                     "frac": achieved / int8_peak, "traffic": traffic,
                     "peak_source": "%s bf16 dense sustained x2 (INT8:BF16 dense rate 2:1)"
                                    % pk_src,
                     "peak_burst": int8_peak_burst, "frac_of_burst": achieved / int8_peak_burst,
                     "ms_per_launch": gm},
        "plain_dmma": {"value": plain_tflops, "unit": "TFLOP/s", "ms_per_step": ms_plain,
                       "frac_of_fp64_nominal": plain_tflops / fp64_nominal,
                       "fp64_nominal_tflops": fp64_nominal},
        "ozaki_speedup_vs_plain": ms_plain / ms,
        "ozaki_phases_ms": {"convert": statistics.mean(conv_ms) if conv_ms else None,
                            "int8_gemm": gm, "crt": statistics.mean(crt_ms) if crt_ms else None},
        "device_error": deverr,
    }
    if rank == 0 and not args.no_extra:
        line["other_configs"] = extras
        # the K rule's moduli count (worst-case bound, 16 at K = 16384): same
        # workload, timed apart
        d16 = torch.empty_like(dC)
        g16 = args_for(d16)
        for _ in range(2):
            assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g16), nmod_rule, sp) == 0
        torch.cuda.synchronize()
        t16 = []
        for _ in range(3):
            ev0.record(stream)
            assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(g16), nmod_rule, sp) == 0
            ev1.record(stream)
            torch.cuda.synchronize()
            t16.append(ev0.elapsed_time(ev1))
        line["ozaki_rule_moduli"] = {"moduli": nmod_rule,
                                     "value": flops / (min(t16) * 1e-3) / 1e12,
                                     "unit": "TFLOP/s", "ms": min(t16)}
        # accuracy against the double-double oracle and the CPU baseline
        # (bounded samples: the oracle only compares and times the CPU leg)
        Co = np.asfortranarray(dC.cpu().numpy().T)
        Cp = np.asfortranarray(dP.cpu().numpy().T)
        C16 = np.asfortranarray(d16.cpu().numpy().T)
        del d16
        line["error_vs_dd"] = dd_errors(A, B, {"ozaki": Co, "plain": Cp, "ozaki_rule_moduli": C16})
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    reps.close()


if __name__ == "__main__":
    main()
