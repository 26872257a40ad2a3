"""Owner-computes distribution of a level-3 contraction over the GPUs of one
node, one process per GPU (torch.distributed: NCCL on GPUs, gloo on CPU).

The reference places the tiles of C on its GPUs 2D block-cyclically
(blas/xkblas.c:2596-2633 choose the grid, :850-905 the owner of tile (i, j))
and each GPU's tasks pull the A and B tiles they read by peer copies
(kaapi/kaapi_plugin_cuda.c:1174).  Here the same placement decides which
process computes which C tiles; the operands a process needs -- the row
panels of A for its tile rows, the column panels of B for its tile columns --
are moved into its own memory in one exchange step before any arithmetic,
so every kernel reads local memory only (no remote loads, no multicast).
A process then computes all of its tiles as ONE contraction on its packed
panels (the tiles of a block-cyclic set share their panels), through the
library's C ABI.

    plan = DistPlan(M, N, K, nb, world)
    a, b = plan.exchange(rank, held_a, held_b, group)   # the panels this rank needs
    tiles = plan.compute(rank, a, b, gemm)              # {(i, j): C tile}

`held_a` / `held_b` map panel index -> tensor for the panels a rank holds
before the call (their "home", by default panel p lives on rank p % world);
`group` is a torch.distributed process group (None: the default one); `gemm`
performs the local contraction (on GPUs, the library's device GEMM on CUDA
tensors: `library_gemm`).  Not run on more than one GPU here: the exchange
and the plan are tested with gloo ranks on CPU.
"""
import math

import numpy as np


def grid_shape(ngpus):
    """GPU grid Gm x Gn for a 2D block-cyclic placement: the most square
    factorisation, found as the reference does (blas/xkblas.c:2608-2626):
    Gm = floor(sqrt(n)); search g from Gm + 1 down for a divisor of n."""
    if ngpus < 1:
        raise ValueError("ngpus must be >= 1")
    gm = int(math.isqrt(ngpus))
    if gm == 0:
        return 1, ngpus
    g = gm + 1
    while g > 0 and ngpus % g != 0:
        g -= 1
    if g == 0:
        return ngpus, 1
    return g, ngpus // g


def tile_owner(i, j, gm, gn, bp=1, bq=1, count=None):
    """Owner of C tile (i, j): ((i / Bp) mod Gp) Gq + (j / Bq) mod Gq, modulo
    the device count (blas/xkblas.c:891)."""
    count = gm * gn if count is None else count
    return (((i // bp) % gm) * gn + (j // bq) % gn) % count


class OwnerMap:
    """Owners of the mt x nt tiles of C on `ngpus` processes."""

    def __init__(self, mt, nt, ngpus):
        self.mt, self.nt, self.ngpus = mt, nt, ngpus
        self.gm, self.gn = grid_shape(ngpus)
        ii, jj = np.meshgrid(np.arange(mt), np.arange(nt), indexing="ij")
        self.owner = tile_owner(ii, jj, self.gm, self.gn, count=ngpus)

    def tiles(self, rank):
        """(i, j) tiles of C that `rank` computes, column-major order."""
        jj, ii = np.nonzero(self.owner.T == rank)
        return list(zip(ii.tolist(), jj.tolist()))

    def row_panels(self, rank):
        """Tile rows of C (= row panels of op(A)) that `rank` has tiles in."""
        return sorted({i for i, _ in self.tiles(rank)})

    def col_panels(self, rank):
        """Tile columns of C (= column panels of op(B)) that `rank` has tiles in."""
        return sorted({j for _, j in self.tiles(rank)})


def default_home(npanels, world):
    """Where panel p lives before the call: rank p mod world."""
    return [p % world for p in range(npanels)]


class DistPlan:
    """The tile grid of C = alpha A B + beta C (A: M x K, B: K x N, tiles of
    nb x nb) on `world` processes, with the panel exchange that precedes the
    arithmetic."""

    def __init__(self, M, N, K, nb, world, a_home=None, b_home=None):
        self.M, self.N, self.K, self.nb, self.world = M, N, K, nb, world
        self.mt = (M + nb - 1) // nb
        self.nt = (N + nb - 1) // nb
        self.map = OwnerMap(self.mt, self.nt, world)
        self.a_home = a_home or default_home(self.mt, world)
        self.b_home = b_home or default_home(self.nt, world)

    def rows(self, i):
        return slice(i * self.nb, min(self.M, (i + 1) * self.nb))

    def cols(self, j):
        return slice(j * self.nb, min(self.N, (j + 1) * self.nb))

    def transfers(self):
        """Every panel move of the exchange: (kind, panel, src, dst), kind 'A'
        (row panel of A) or 'B' (column panel of B); a rank never sends to
        itself.  The order is the same on every rank."""
        out = []
        for dst in range(self.world):
            for i in self.map.row_panels(dst):
                if self.a_home[i] != dst:
                    out.append(("A", i, self.a_home[i], dst))
            for j in self.map.col_panels(dst):
                if self.b_home[j] != dst:
                    out.append(("B", j, self.b_home[j], dst))
        return out

    def bytes_moved(self, elsize=8):
        tot = 0
        for kind, p, _, _ in self.transfers():
            rows = self.rows(p) if kind == "A" else self.cols(p)
            tot += (rows.stop - rows.start) * self.K * elsize
        return tot

    def exchange(self, rank, held_a, held_b, group=None, dtype=None, device=None):
        """Run the exchange on this rank: send the panels it holds to the
        ranks that need them, receive the ones it needs.  `held_a[i]` is row
        panel i of A (rows x K), `held_b[j]` column panel j of B (K x cols),
        as torch tensors on this rank's device.  Returns (a, b): dicts of the
        panels this rank computes with.  One batched point-to-point step;
        every rank issues its operations in the same global order."""
        import torch
        import torch.distributed as dist
        held = list(held_a.values()) + list(held_b.values())
        dtype = dtype or (held[0].dtype if held else torch.float64)
        device = device or (held[0].device if held else "cpu")
        ops = []
        a = {i: held_a[i] for i in self.map.row_panels(rank) if self.a_home[i] == rank}
        b = {j: held_b[j] for j in self.map.col_panels(rank) if self.b_home[j] == rank}
        for kind, p, src, dst in self.transfers():
            if src == rank:
                t = (held_a if kind == "A" else held_b)[p].contiguous()
                ops.append(dist.P2POp(dist.isend, t, dst, group=group))
            elif dst == rank:
                shape = ((self.rows(p).stop - self.rows(p).start, self.K) if kind == "A"
                         else (self.K, self.cols(p).stop - self.cols(p).start))
                t = torch.empty(shape, dtype=dtype, device=device)
                (a if kind == "A" else b)[p] = t
                ops.append(dist.P2POp(dist.irecv, t, src, group=group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        return a, b

    def pack(self, rank, a, b):
        """This rank's operands of its one local contraction: its row panels
        of A stacked (rows x K) and its column panels of B side by side
        (K x cols), with the (row, col) offsets of each panel in the packed
        result."""
        import torch
        ri, cj = self.map.row_panels(rank), self.map.col_panels(rank)
        Ap = torch.cat([a[i] for i in ri], dim=0) if ri else None
        Bp = torch.cat([b[j] for j in cj], dim=1) if cj else None
        return Ap, Bp, ri, cj

    def compute(self, rank, a, b, gemm):
        """The C tiles of this rank: gemm(Ap, Bp) on its packed panels (one
        contraction: with Gm x Gn = world, a rank's block-cyclic tiles are
        exactly the cross product of its tile rows and tile columns);
        returns {(i, j): tile}."""
        Ap, Bp, ri, cj = self.pack(rank, a, b)
        if Ap is None or Bp is None:
            return {}
        Cp = gemm(Ap, Bp)
        out = {}
        roff, r0 = {}, 0
        for i in ri:
            roff[i] = r0
            r0 += self.rows(i).stop - self.rows(i).start
        coff, c0 = {}, 0
        for j in cj:
            coff[j] = c0
            c0 += self.cols(j).stop - self.cols(j).start
        for i, j in self.map.tiles(rank):
            h = self.rows(i).stop - self.rows(i).start
            w = self.cols(j).stop - self.cols(j).start
            out[(i, j)] = Cp[roff[i]:roff[i] + h, coff[j]:coff[j] + w]
        return out


def library_gemm(alpha=1.0, tensor_op=False):
    """The local contraction on this rank's GPU through the library's C ABI:
    row-major torch tensors Ap (m x k) and Bp (k x n) -> Cp = alpha Ap Bp
    (m x n, row-major), computed as the column-major product Cp^T = Bp^T Ap^T
    by xkb_cuda_gemm (FP64 DMMA) or xkb_cuda_ozaki_gemm (tensor-op mode)."""
    import ctypes
    import torch

    from . import GemmArgs, lib

    def run(Ap, Bp):
        m, k = Ap.shape
        n = Bp.shape[1]
        Ap, Bp = Ap.contiguous(), Bp.contiguous()
        Cp = torch.empty(m, n, dtype=Ap.dtype, device=Ap.device)
        # column-major views: Bp^T is n x k (ld n), Ap^T is k x m (ld k), Cp^T n x m (ld n)
        g = GemmArgs(1, 0, 0, n, m, k, Bp.data_ptr(), n, Ap.data_ptr(), k, Cp.data_ptr(), n)
        g.alpha[0] = alpha
        st = ctypes.c_void_p(torch.cuda.current_stream(Ap.device).cuda_stream)
        f = lib().xkb_cuda_ozaki_gemm if tensor_op else None
        r = f(ctypes.byref(g), 0, st) if f else lib().xkb_cuda_gemm(ctypes.byref(g), st)
        if r != 0:
            raise RuntimeError("local contraction failed: %d" % r)
        return Cp

    return run
