"""GLS map-making solve sharded over ranks: one process per GPU, torch.distributed
(NCCL on GPUs) for the exchanges.

Each rank holds the samples of some detectors and stationary intervals
(whole Toeplitz blocks, so N^-1 needs no halo).  The solve is the
single-process solve of the union of all ranks' data, as MAPPRAISER's MLmap
over MPI ranks (mappraiser/src/mappraiser.c:34-385, pcg_true.c:20-241,
precond.c:456-702):

* set-up: the global pixel set is the union of the ranks' pixels; the 3x3
  blocks (getlocalW on each rank) are summed over ranks (one all-reduce of
  9 doubles and one hit count per pixel); every rank inverts the same blocks
  and takes the same rcond cut; each rank rewrites its own samples of the
  pixels the cut removes (the pixel after each cut one when flagged samples
  exist, as the single-process cut does, precond.c:521 with
  mappraiser.c:130-142);
* iteration: each rank applies P^T N^-1 P to its samples with the library's
  kernels and the local maps are summed into the global map by one all-reduce
  of the map per operator application; map vectors are replicated, so the
  block-Jacobi apply and the dot products need no further exchange.

`solve(precision="fp64")` is PCG_GLS_true; `precision="mixed"` is the FP64
iterative refinement of mdp_gls_solve_mixed, with one all-reduce per inner
(FP32 operator) iteration and per FP64 residual.  Stop decisions are taken on
rank 0's scalars and broadcast, so every rank runs the same collectives.

`GpuShard` is a rank's data on its GPU; any object with the same methods
(pixels, trash, blocks, invert, cut, residual, apply) can stand in for it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch
import torch.distributed as dist


@dataclass
class DistInfo:
    iterations: int
    outer_iterations: int
    converged: bool
    res0: float
    res: float
    n_map: int
    n_cut: int


class GpuShard:
    """This rank's pointing, noise operator and TOD on its GPU."""

    def __init__(self, ctx, pix, weights, signal, noise, block_sizes, lam: int, invtt, idv=None):
        import midapack_b200 as mb
        self.mb = mb
        self.ctx = ctx
        self.m = int(signal.numel())
        self.P = mb.Pointing(ctx, pix, weights, self.m, 3)
        self.N = mb.Noise(ctx, block_sizes, lam, invtt, idv=idv)
        self.signal, self.noise = signal, noise
        self.device = signal.device

    def _shape(self):
        return self.P.shape()

    def pixels(self) -> torch.Tensor:
        sh = self._shape()
        lind = self.P.lindices().to(torch.int64)
        return (lind[3 * sh["trash_pix"]::3] // 3).contiguous()

    def trash(self) -> bool:
        return bool(self._shape()["trash_pix"])

    def blocks(self):
        mb = self.mb
        npix = self._shape()["n_map"] // 3
        W = torch.empty((npix, 9), dtype=torch.float64, device=self.device)
        hits = torch.empty(npix, dtype=torch.int32, device=self.device)
        mb.check(mb.lib().mdp_local_blocks(self.ctx.h, self.P.h, self.N.h, mb.ct.c_void_p(W.data_ptr()),
                                           mb.ct.c_void_p(hits.data_ptr())), "mdp_local_blocks")
        return W, hits

    def invert(self, W: torch.Tensor):
        mb = self.mb
        npix = W.shape[0]
        W = W.contiguous().clone()
        inv = torch.empty_like(W)
        rcond = torch.empty(npix, dtype=torch.float64, device=W.device)
        cut = torch.empty(npix, dtype=torch.int32, device=W.device)
        n = mb.ct.c_int64()
        mb.check(mb.lib().mdp_block_inverse(self.ctx.h, npix, mb.ct.c_void_p(W.data_ptr()),
                                            mb.ct.c_void_p(inv.data_ptr()), mb.ct.c_void_p(rcond.data_ptr()),
                                            mb.ct.c_void_p(cut.data_ptr()), mb.ct.byref(n)), "mdp_block_inverse")
        return inv, rcond, cut

    def cut(self, target: torch.Tensor) -> int:
        mb = self.mb
        t = target.to(torch.int32).contiguous()
        kept = mb.ct.c_int64()
        mb.check(mb.lib().mdp_pointing_cut(self.ctx.h, self.P.h, mb.ct.c_void_p(t.data_ptr()), mb.ct.byref(kept)),
                 "mdp_pointing_cut")
        return kept.value

    def residual(self, x_loc: torch.Tensor | None) -> torch.Tensor:
        mb = self.mb
        r = torch.empty(max(self._shape()["n_map"], 1), dtype=torch.float64, device=self.device)
        xp = mb.ct.c_void_p(x_loc.data_ptr()) if x_loc is not None else mb.ct.c_void_p(0)
        mb.check(mb.lib().mdp_gls_residual(self.ctx.h, self.P.h, self.N.h, mb.ct.c_void_p(self.signal.data_ptr()),
                                           mb.ct.c_void_p(self.noise.data_ptr()), xp, mb.ct.c_void_p(r.data_ptr())),
                 "mdp_gls_residual")
        return r[: self._shape()["n_map"]]

    def apply(self, h_loc: torch.Tensor, fp32: bool = False) -> torch.Tensor:
        mb = self.mb
        h = h_loc.contiguous()
        q = torch.empty(max(h.numel(), 1), dtype=torch.float64, device=self.device)
        mb.check(mb.lib().mdp_apply_op(self.ctx.h, self.P.h, self.N.h, mb.ct.c_void_p(h.data_ptr()),
                                       mb.ct.c_void_p(q.data_ptr()), 1 if fp32 else 0), "mdp_apply_op")
        return q[: h.numel()]

    def close(self):
        self.P.close()
        self.N.close()


class ShardedGLS:
    """The sharded solve over the ranks of `group` (default: the world)."""

    def __init__(self, shard, group=None):
        self.s = shard
        self.g = group
        self.dev = shard.device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.host_staging = dist.get_backend(group) == "gloo"

    # ---- collectives (device tensors go through host memory with gloo)
    def _stage(self, t: torch.Tensor) -> torch.Tensor:
        return t.cpu() if (t.is_cuda and self.host_staging) else t

    def _sum(self, t: torch.Tensor, op=None) -> torch.Tensor:
        u = self._stage(t)
        dist.all_reduce(u, op=op or dist.ReduceOp.SUM, group=self.g)
        if u is not t:
            t.copy_(u)
        return t

    def _flag(self, v: bool) -> bool:
        """Rank 0's decision, on every rank."""
        f = self._stage(torch.tensor([1 if v else 0], dtype=torch.int32, device=self.dev))
        dist.broadcast(f, src=dist.get_global_rank(self.g, 0) if self.g is not None else 0, group=self.g)
        return bool(f.item())

    def _union(self, pix: torch.Tensor) -> torch.Tensor:
        n = self._stage(torch.tensor([pix.numel()], dtype=torch.int64, device=self.dev))
        sizes = [torch.zeros_like(n) for _ in range(self.world)]
        dist.all_gather(sizes, n, group=self.g)
        mx = int(max(int(s.item()) for s in sizes))
        buf = torch.full((max(mx, 1),), -1, dtype=torch.int64, device=self.dev)
        buf[: pix.numel()] = pix
        buf = self._stage(buf)
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf, group=self.g)
        allp = torch.cat(parts).to(self.dev)
        return torch.unique(allp[allp >= 0])  # sorted

    # ---- set-up: pixel union, blocks, cut
    def setup(self):
        s = self.s
        pix = s.pixels()
        pg = self._union(pix)
        trash = torch.tensor([1 if s.trash() else 0], dtype=torch.int32, device=self.dev)
        self._sum(trash, dist.ReduceOp.MAX)
        l2g = torch.searchsorted(pg, pix)
        W_loc, hits_loc = s.blocks()
        W = torch.zeros((pg.numel(), 9), dtype=torch.float64, device=self.dev)
        W.index_add_(0, l2g, W_loc.reshape(-1, 9))
        hits = torch.zeros(pg.numel(), dtype=torch.int64, device=self.dev)
        hits.index_add_(0, l2g, hits_loc.to(torch.int64))
        self._sum(W)
        self._sum(hits)
        inv, rcond, cut = s.invert(W)
        cutb = cut.to(torch.bool)
        self.n_cut = int(cutb.sum().item())
        if self.n_cut:
            # samples rewritten: those of the pixel after each cut one when flagged
            # samples exist (the single-process numbering), else of the cut pixel
            target = torch.zeros(pg.numel(), dtype=torch.int32, device=self.dev)
            if int(trash.item()):
                target[1:] = cut[:-1]
            else:
                target = cut.clone()
            s.cut(target[l2g])
            kept_pix = pg[target == 0]
            inv, rcond, hits = inv[~cutb], rcond[~cutb], hits[~cutb]
            pad = kept_pix.numel() - inv.shape[0]
            if pad > 0:  # last pixel cut with flagged samples: unpaired blocks are zero
                inv = torch.cat([inv, torch.zeros((pad, 9), dtype=inv.dtype, device=self.dev)])
                rcond = torch.cat([rcond, torch.zeros(pad, dtype=rcond.dtype, device=self.dev)])
                hits = torch.cat([hits, torch.zeros(pad, dtype=hits.dtype, device=self.dev)])
            pg = kept_pix
            pix = s.pixels()
            l2g = torch.searchsorted(pg, pix)
        self.pg, self.l2g = pg, l2g
        self.inv = inv.reshape(-1, 3, 3)[: pg.numel()]
        self.rcond, self.hits = rcond[: pg.numel()], hits[: pg.numel()]
        self.n = 3 * pg.numel()

    # ---- map-domain helpers
    def _gather(self, x: torch.Tensor) -> torch.Tensor:
        return x.view(-1, 3)[self.l2g].reshape(-1)

    def _scatter_sum(self, q_loc: torch.Tensor) -> torch.Tensor:
        q = torch.zeros(self.n, dtype=torch.float64, device=self.dev)
        q.view(-1, 3).index_add_(0, self.l2g, q_loc.view(-1, 3))
        return self._sum(q)

    def _A(self, h: torch.Tensor, fp32: bool = False) -> torch.Tensor:
        return self._scatter_sum(self.s.apply(self._gather(h), fp32))

    def _residual(self, x: torch.Tensor | None) -> torch.Tensor:
        return self._scatter_sum(self.s.residual(None if x is None else self._gather(x)))

    def _M(self, g: torch.Tensor) -> torch.Tensor:
        return torch.bmm(self.inv, g.view(-1, 3, 1)).reshape(-1)

    def _pcg(self, b: torch.Tensor, tol2: float, maxiter: int, fp32: bool, on_iter=None):
        """Polak-Ribiere PCG on A x = b from x = 0 (pcg_true.c:20-241); stops when
        sum(g^2) <= tol2 or after maxiter iterations.  Returns x, iterations, res."""
        x = torch.zeros_like(b)
        g = b.clone()
        Cg = self._M(g)
        h = Cg.clone()
        g2pix = float(torch.dot(Cg, g))
        res = float(torch.dot(g, g))
        it = 0
        while it < maxiter:
            q = self._A(h, fp32)
            ro = g2pix / float(torch.dot(h, q))
            x += ro * h
            gp = g
            g = gp - ro * q
            Cg = self._M(g)
            g2pixp = g2pix
            g2pix = float(torch.dot(Cg, g))
            polak = float(torch.dot(Cg, g - gp))
            res = float(torch.dot(g, g))
            it += 1
            if on_iter:
                on_iter(res)
            if self._flag(not math.isfinite(res)):
                raise FloatingPointError(f"sharded PCG: residual became {res}")
            if self._flag(res <= tol2):
                break
            h = h * (polak / g2pixp) + Cg
        return x, it, res

    def solve(self, tol: float = 1e-8, maxiter: int = 500, precision: str = "fp64", inner_tol: float = 1e-4,
              inner_maxiter: int = 100, on_iter=None):
        """Returns (x over the global kept pixels, their global pixel ids, rcond, hits, DistInfo); x is
        replicated on every rank, pixel-major (I, Q, U).  on_iter(res) is called after each FP64 PCG
        iteration with its residual sum(g^2)."""
        if not hasattr(self, "pg"):
            self.setup()
        b = self._residual(None)
        res0 = float(torch.dot(b, b))
        if self._flag(res0 <= tol):  # the reference's initial test (pcg_true.c:113-118)
            x = torch.zeros_like(b)
            return x, self.pg, self.rcond, self.hits, DistInfo(0, 0, True, res0, res0, self.n, self.n_cut)
        tol2 = tol * tol * res0
        if precision == "fp64":
            x, it, res = self._pcg(b, tol2, maxiter - 1, False, on_iter)
            info = DistInfo(it, 0, res <= tol2, res0, res, self.n, self.n_cut)
            return x, self.pg, self.rcond, self.hits, info
        if precision != "mixed":
            raise ValueError(precision)
        x = torch.zeros_like(b)
        r, res = b, res0
        total = outer = 0
        while not self._flag(res <= tol2) and total < maxiter:
            need = 0.5 * tol / math.sqrt(res / res0)
            itol = max(inner_tol, min(need, 0.5))
            d, it, _ = self._pcg(r, itol * itol * res, min(inner_maxiter, maxiter - total), True)
            total += it
            outer += 1
            x += d
            r = self._residual(x)
            res = float(torch.dot(r, r))
            if self._flag(not math.isfinite(res)):
                raise FloatingPointError(f"sharded refinement: residual became {res}")
        info = DistInfo(total, outer, res <= tol2, res0, res, self.n, self.n_cut)
        return x, self.pg, self.rcond, self.hits, info
