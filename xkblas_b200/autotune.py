"""Autotuner: measures, on the B200 it runs on, the choices the library
otherwise makes by rule, and writes them as a tuning table that the runtime
loads at init (XKBLAS_TUNE_FILE):

    python -m xkblas_b200.autotune --out xkblas_tune.txt [--quick]
    XKBLAS_TUNE_FILE=xkblas_tune.txt ./app

Choices (keys of the table, see include/xkb_cuda.h):
  gemm_big_min_tiles      whole-matrix FP64 GEMM: 128-wide tiles from this many
                          tiles on (timed: both tile shapes on square DGEMMs);
  ozaki_min_dim           tensor-op mode: Ozaki from this size on (timed:
                          plain DMMA vs Ozaki on square DGEMMs);
  ozaki_moduli_k<=<K>     moduli count per inner-size band (measured error:
                          the smallest count whose error against a 16-moduli
                          product is at most half the plain FP64 kernel's on
                          inputs with exponents spread over [-20, 20] per row
                          of A and per column of B);
  oz_2cta                 Ozaki INT8 GEMM on single CTAs or CTA pairs (timed
                          on a square Ozaki DGEMM);
  ozaki_panel_cols        column width of the panels a public-API Ozaki DGEMM
                          streams through (timed end to end with pinned host
                          matrices, 8192^3, caches dropped per call);
  batch_schedule,         tile-task executor: claim order and 128-row tile
  batch_tile128_min_rows  threshold (timed on a mixed batch of uneven calls).

Each measurement uses seeded synthetic matrices and CUDA events (the panel
sweep: host clock around the public calls); the table records the measured
times beside each choice.
"""
import argparse
import ctypes
import math
import time
import sys

import numpy as np


from xkblas_b200 import GemmArgs as _GemmArgs  # xkb_gemm_args


def choose_moduli(lib, K, M=1024, N=1024, stream=None, gen=None):
    """The smallest moduli count whose Ozaki product, on M x K times K x N
    inputs with exponents spread over [-20, 20] per row of A and per column
    of B, is at most half as far from a 16-moduli product as the plain FP64
    kernel is (errors normalised by |a_i| |b_j| K).  Returns (count, plain
    error, [(count, error) tried]).  Runs on `stream` (a CUDA stream handle,
    ctypes) and synchronises the device around every call."""
    import torch as t
    g = gen if gen is not None else t.Generator(device="cuda").manual_seed(77)
    sp = stream if stream is not None else ctypes.c_void_p(0)

    def spread(r, c, by_col):
        u = 2 * t.rand(c, r, generator=g, device="cuda", dtype=t.float64) - 1
        shape = (c, 1) if by_col else (1, r)
        e = t.randint(-20, 21, shape, generator=g, device="cuda").double()
        return u * t.pow(2.0, e)

    A, B = spread(M, K, False), spread(K, N, True)
    C = t.zeros(N, M, device="cuda", dtype=t.float64)
    t.cuda.synchronize()
    a = _GemmArgs(1, 0, 0, M, N, K, A.data_ptr(), M, B.data_ptr(), K, C.data_ptr(), M)
    a.alpha[0] = 1.0
    assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(a), 16, sp) == 0
    t.cuda.synchronize()
    ref = C.clone()
    assert lib.xkb_cuda_gemm(ctypes.byref(a), sp) == 0
    t.cuda.synchronize()
    scale = (A.abs().amax(dim=0)[None, :] * B.abs().amax(dim=1)[:, None]) * K  # |a_i||b_j| K
    err_plain = ((C - ref).abs() / scale).max().item()
    choice, errs = 16, []
    for n in range(10, 16):
        C.zero_()
        t.cuda.synchronize()
        assert lib.xkb_cuda_ozaki_gemm(ctypes.byref(a), n, sp) == 0
        t.cuda.synchronize()
        err = ((C - ref).abs() / scale).max().item()
        errs.append((n, err))
        if err <= 0.5 * err_plain:
            choice = n
            break
    return choice, err_plain, errs


class Tuner:
    def __init__(self, quick=False, log=print):
        import torch
        import xkblas_b200 as X
        self.torch, self.X = torch, X
        self.lib = X.lib()
        X.init()
        self.quick = quick
        self.log = log
        # every tensor operation and every library call on one stream: the
        # library's own stream does not order against torch's default stream
        self.stream = torch.cuda.Stream()
        torch.cuda.set_stream(self.stream)
        self.sp = ctypes.c_void_p(self.stream.cuda_stream)
        self.g = torch.Generator(device="cuda").manual_seed(77)
        self.table = {}   # key -> (value, note)

    # -- helpers ---------------------------------------------------------------
    def rnd(self, r, c):
        t = self.torch
        return t.rand(c, r, generator=self.g, device="cuda", dtype=t.float64) - 0.5

    def spread(self, r, c, by_col):
        """u * 2^e, e uniform in [-20, 20] per row (A) or per column (B)."""
        t = self.torch
        u = 2 * t.rand(c, r, generator=self.g, device="cuda", dtype=t.float64) - 1
        if by_col:
            e = t.randint(-20, 21, (c, 1), generator=self.g, device="cuda").double()
        else:
            e = t.randint(-20, 21, (1, r), generator=self.g, device="cuda").double()
        return u * t.pow(2.0, e)

    def args(self, A, B, C, M, N, K):
        a = _GemmArgs(1, 0, 0, M, N, K, A.data_ptr(), M, B.data_ptr(), K, C.data_ptr(), M)
        a.alpha[0] = 1.0
        return a

    def time(self, fn, reps):
        t = self.torch
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        assert fn() == 0
        t.cuda.synchronize()
        best = math.inf
        for _ in range(reps):
            e0.record(self.stream)
            assert fn() == 0
            e1.record(self.stream)
            t.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    # -- choices ---------------------------------------------------------------
    def gemm_tiles(self):
        lib, sizes = self.lib, ([768, 1536, 3072] if self.quick else [512, 768, 1024, 1536, 2048, 3072, 4096])
        big_wins = []
        for n in sizes:
            A, B, C = self.rnd(n, n), self.rnd(n, n), self.rnd(n, n)
            a = self.args(A, B, C, n, n, n)
            tm = {}
            for shape, v in (("big", 0.0), ("small", 1e12)):
                lib.xkb_tune_set(b"gemm_big_min_tiles", v)
                tm[shape] = self.time(lambda: lib.xkb_cuda_gemm(ctypes.byref(a), self.sp), 5)
            tiles = math.ceil(n / 128) ** 2
            big_wins.append((tiles, tm["big"] <= tm["small"]))
            self.log("gemm %5d: tiles %5d big %.3f ms small %.3f ms" % (n, tiles, tm["big"], tm["small"]))
        # smallest tile count from which the big tile wins at every larger size
        thr = None
        for i, (tiles, win) in enumerate(big_wins):
            if all(w for _, w in big_wins[i:]):
                thr = tiles
                break
        lib.xkb_tune_set(b"gemm_big_min_tiles", float(thr if thr is not None else 1 << 30))
        self.table["gemm_big_min_tiles"] = (thr if thr is not None else 1 << 30,
                                            "tiles: " + ", ".join("%d%s" % (t, "B" if w else "s") for t, w in big_wins))

    def ozaki_crossover(self):
        lib = self.lib
        sizes = [1024, 2048, 4096] if self.quick else [512, 768, 1024, 1536, 2048, 3072, 4096]
        wins = []
        for n in sizes:
            A, B, C = self.rnd(n, n), self.rnd(n, n), self.rnd(n, n)
            a = self.args(A, B, C, n, n, n)
            tp = self.time(lambda: lib.xkb_cuda_gemm(ctypes.byref(a), self.sp), 5)
            to = self.time(lambda: lib.xkb_cuda_ozaki_gemm(ctypes.byref(a), 0, self.sp), 5)
            wins.append((n, to < tp))
            self.log("ozaki %5d: plain %.3f ms ozaki %.3f ms" % (n, tp, to))
        thr = None
        for i, (n, win) in enumerate(wins):
            if all(w for _, w in wins[i:]):
                thr = n
                break
        thr = thr if thr is not None else 1 << 30
        self.table["ozaki_min_dim"] = (thr, "sizes: " + ", ".join("%d%s" % (n, "O" if w else "p") for n, w in wins))

    def moduli(self):
        M = N = 512 if self.quick else 1024
        for K in ([1024, 16384] if self.quick else [256, 1024, 4096, 16384, 65536]):
            choice, err_plain, errs = choose_moduli(self.lib, K, M, N, self.sp, self.g)
            self.log("moduli K=%6d: plain %.2e, " % (K, err_plain)
                     + ", ".join("%d: %.2e" % e for e in errs) + " -> %d" % choice)
            self.table["ozaki_moduli_k<=%d" % K] = (choice, "plain err %.2e; %s" % (
                err_plain, ", ".join("%d: %.2e" % e for e in errs)))

    def batch(self):
        t, lib, X = self.torch, self.lib, self.X
        rng = np.random.default_rng(5)
        ops, keep = [], []
        ncalls = 120 if self.quick else 400

        def lu():
            return int(np.exp(rng.uniform(np.log(64), np.log(2048))))

        for _ in range(ncalls):
            r = rng.random()
            o = X.BatchOp()
            if r < 0.8:
                m, n, k = lu(), lu(), lu()
                A, B, C = self.rnd(m, k), self.rnd(k, n), self.rnd(m, n)
                o.kind, o.dtype, o.M, o.N, o.K = 0, 1, m, n, k
                o.A, o.lda, o.B, o.ldb, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m
                o.alpha[0] = o.beta[0] = 1.0
                keep += [A, B, C]
            else:
                m, n = lu(), lu()
                L = t.tril(self.rnd(m, m).t()) + m * t.eye(m, device="cuda", dtype=t.float64)
                A, B = L.t().contiguous(), self.rnd(m, n)
                o.kind, o.dtype, o.side, o.uplo, o.trans, o.diag, o.M, o.N = 1, 1, 0, 1, 0, 0, m, n
                o.A, o.lda, o.C, o.ldc = A.data_ptr(), m, B.data_ptr(), m
                o.alpha[0] = 1.0
                keep += [A, B]
            ops.append(o)
        arr = (X.BatchOp * len(ops))(*ops)
        best = None
        for sched in (0, 1):
            for rows in ((96, 1 << 20) if self.quick else (64, 96, 160, 1 << 20)):
                lib.xkb_tune_set(b"batch_tile128_min_rows", float(rows))
                lib.xkb_cuda_batch_release()
                ms = self.time(lambda: lib.xkb_cuda_batch(arr, len(ops), sched, self.sp), 3)
                self.log("batch schedule %d tile128 rows >= %d: %.2f ms" % (sched, rows, ms))
                if best is None or ms < best[0]:
                    best = (ms, sched, rows)
        lib.xkb_cuda_batch_release()
        self.table["batch_schedule"] = (best[1], "%.2f ms best of the sweep" % best[0])
        self.table["batch_tile128_min_rows"] = (best[2], "%.2f ms best of the sweep" % best[0])

    def ozaki_kernel(self):
        """Single-CTA or CTA-pair INT8 GEMM (oz_2cta)."""
        lib = self.lib
        n = 2048 if self.quick else 4096
        A, B, C = self.rnd(n, n), self.rnd(n, n), self.rnd(n, n)
        a = self.args(A, B, C, n, n, n)
        tm = {}
        for v in (0.0, 1.0):
            lib.xkb_tune_set(b"oz_2cta", v)
            tm[v] = self.time(lambda: lib.xkb_cuda_ozaki_gemm(ctypes.byref(a), 0, self.sp), 5)
        best = 1 if tm[1.0] < tm[0.0] else 0
        lib.xkb_tune_set(b"oz_2cta", float(best))
        self.log("ozaki %d: single CTA %.3f ms, CTA pair %.3f ms" % (n, tm[0.0], tm[1.0]))
        self.table["oz_2cta"] = (best, "%d^3: single %.3f ms, pair %.3f ms" % (n, tm[0.0], tm[1.0]))

    def ozaki_panels(self):
        """Column-panel width of the public-API Ozaki DGEMM (ozaki_panel_cols),
        timed end to end with pinned host matrices, caches dropped per call."""
        t, X, lib = self.torch, self.X, self.lib
        n = 4096 if self.quick else 8192
        hs = [t.empty((n, n), dtype=t.float64, pin_memory=True).numpy() for _ in range(3)]
        rng = np.random.default_rng(3)
        for h in hs[:2]:
            h[...] = rng.random((n, n)) - 0.5
        one, zero = np.array([1.0]), np.array([0.0])
        P = ctypes.c_void_p
        old_min = lib.xkb_tune_get(b"ozaki_min_dim", 2048.0)
        lib.xkb_tune_set(b"ozaki_min_dim", float(min(old_min, n)))
        X.set_modemath(X.XKBLAS_TENSOR_OP_MATH)

        def call():
            assert lib.xkblas_dgemm_async(111, 111, n, n, n, P(one.ctypes.data), P(hs[0].ctypes.data),
                                          n, P(hs[1].ctypes.data), n, P(zero.ctypes.data),
                                          P(hs[2].ctypes.data), n) == 0
            lib.xkblas_memory_coherent_async(0, 0, n, n, P(hs[2].ctypes.data), n, 8)
            assert lib.xkblas_sync() == 0
            lib.xkblas_memory_invalidate_caches()

        res = {}
        try:
            for cols in (512, 1024, 2048):
                if n // cols < 2:
                    continue
                lib.xkb_tune_set(b"ozaki_panel_cols", float(cols))
                call()
                best = math.inf
                for _ in range(2 if self.quick else 3):
                    t0 = time.perf_counter()
                    call()
                    best = min(best, time.perf_counter() - t0)
                res[cols] = best * 1e3
                self.log("ozaki panels %d^3, %d columns: %.2f ms" % (n, cols, res[cols]))
        finally:
            X.set_modemath(X.XKBLAS_DEFAULT_MATH)
            lib.xkb_tune_set(b"ozaki_min_dim", old_min)
        cols = min(res, key=res.get)
        lib.xkb_tune_set(b"ozaki_panel_cols", float(cols))
        self.table["ozaki_panel_cols"] = (cols, "%d^3 e2e: " % n + ", ".join(
            "%d: %.1f ms" % (c, v) for c, v in res.items()))

    def run(self):
        self.lib.xkb_tune_clear()
        self.gemm_tiles()
        self.ozaki_crossover()
        self.moduli()
        self.ozaki_kernel()
        self.ozaki_panels()
        self.batch()
        return self.table


def write_table(table, path, header=""):
    with open(path, "w") as f:
        f.write("# xkblas tuning table (python -m xkblas_b200.autotune)\n")
        if header:
            f.write("# %s\n" % header)
        for k, (v, note) in table.items():
            f.write("%-28s %-12s # %s\n" % (k, repr(v) if isinstance(v, float) else v, note))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True, help="tuning table to write")
    ap.add_argument("--quick", action="store_true", help="fewer sizes (about half a minute)")
    a = ap.parse_args(argv)
    import torch
    name = torch.cuda.get_device_name(0)
    table = Tuner(quick=a.quick).run()
    write_table(table, a.out, header="device: %s" % name)
    print("wrote", a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
