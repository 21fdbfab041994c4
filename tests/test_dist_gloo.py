"""Sharded solve (midapack_b200.dist) on the CPU: two gloo ranks, each holding
half of the detectors, with the oracle's operators standing in for the GPU
shard; the replicated map must equal the oracle's single-process PCG of the
whole data (maps within 1e-8 relative per I/Q/U, same pixels, iteration count
+-1), for flagged samples, for a cut with flagged samples (the quirk of the
rewritten pixel, in global pixel order) and for the mixed-precision
refinement."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as tmp

from midapack_b200 import synth
from oracle import restate as R
from tests._cases import with_degenerate_pixels


class OracleShard:
    """A rank's samples with the oracle restatement's operators (CPU)."""

    device = torch.device("cpu")

    def __init__(self, pix, weights, signal, noise, block_sizes, lam, invtt):
        self.m = len(signal)
        self.A = R.local_shape(pix, weights, self.m, 3)
        self.sig = np.array(signal, dtype=np.float64)
        self.noise = np.asarray(noise, dtype=np.float64)
        self.bs, self.lam, self.invtt = np.asarray(block_sizes), lam, invtt

    def pixels(self):
        t = self.A.trash_pix
        return torch.from_numpy(self.A.lindices[3 * t::3].astype(np.int64) // 3)

    def trash(self):
        return bool(self.A.trash_pix)

    def blocks(self):
        W, hits = R.local_W(self.A, self.bs, self.lam, self.invtt)
        return torch.from_numpy(W.reshape(-1, 9).copy()), torch.from_numpy(np.asarray(hits, dtype=np.int32))

    def invert(self, W):
        rcond, inv = R.bj_blocks(W.numpy().reshape(-1, 3, 3))
        cut = ~(rcond > 1e-1)
        inv = np.where(cut[:, None, None], 0.0, inv)
        return (torch.from_numpy(inv.reshape(-1, 9).copy()), torch.from_numpy(rcond.copy()),
                torch.from_numpy(cut.astype(np.int32)))

    def cut(self, target):
        target = target.numpy().astype(bool)
        A = self.A
        idx = A.local.reshape(A.m, 3).astype(np.int64)
        valid = (idx[:, 0] != 0) if A.trash_pix else np.ones(A.m, dtype=bool)
        q = np.where(valid, idx[:, 0] // 3 - A.trash_pix, 0)
        rows = valid & target[q]
        gl = A.lindices[A.local.astype(np.int64)].astype(np.int32).reshape(A.m, 3)
        vals = A.values.copy().reshape(A.m, 3)
        gl[rows] = np.arange(3, dtype=np.int32) - 3
        vals[rows] = 0.0
        self.sig[rows] = 0.0
        if rows.any():
            self.A = R.local_shape(gl.reshape(-1), vals.reshape(-1), A.m, 3)
            self.A.trash_pix = 1
        return int((~target).sum())

    def _N(self, v):
        return R.stbmm(v, self.bs, self.lam, self.invtt)

    def residual(self, x_loc):
        d = self.sig + self.noise
        if x_loc is not None:
            d = d - R.matvec(self.A, x_loc.numpy())
        return torch.from_numpy(R.trmatvec(self.A, self._N(d)))

    def apply(self, h_loc, fp32=False):
        q = R.trmatvec(self.A, self._N(R.matvec(self.A, h_loc.numpy())))
        if fp32:  # a stand-in for the FP32 operator: the FP64 product rounded to FP32
            q = q.astype(np.float32).astype(np.float64)
        return torch.from_numpy(q)


def _split(wl, rank, world):
    """Detectors [rank*nd/world, (rank+1)*nd/world) of the workload, with their blocks."""
    nd = wl.n_det
    d0, d1 = rank * nd // world, (rank + 1) * nd // world
    s0, s1 = d0 * wl.n_samp, d1 * wl.n_samp
    nb_per = wl.n_samp // wl.block_len
    bs = wl.block_sizes[d0 * nb_per:d1 * nb_per]
    tt = wl.invtt[d0 * nb_per * wl.lam:d1 * nb_per * wl.lam]
    return (wl.pix[3 * s0:3 * s1], wl.weights[3 * s0:3 * s1], wl.signal[s0:s1], wl.noise[s0:s1], bs, wl.lam, tt)


def _worker(rank, world, port, case, precision, out):
    import torch.distributed as dist
    from midapack_b200.dist import ShardedGLS
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = _CASES[case]()
        shard = OracleShard(*_split(wl, rank, world))
        x, pix, rcond, hits, info = ShardedGLS(shard).solve(tol=1e-11, maxiter=600, precision=precision)
        out[rank] = (x.numpy(), pix.numpy(), hits.numpy(), info.iterations, info.converged, info.n_cut)
    finally:
        dist.destroy_process_group()


_CASES = {
    "gaps": lambda: synth.small(n_det=4, n_samp=2048, block_len=1024, lam=32, gap_frac=0.02, seed=41),
    "cut_gaps": lambda: with_degenerate_pixels(
        synth.small(n_det=4, n_samp=2048, block_len=1024, lam=32, gap_frac=0.02, seed=42), seed=3),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("case,precision", [("gaps", "fp64"), ("cut_gaps", "fp64"), ("gaps", "mixed")])
def test_two_gloo_ranks_match_single_process(case, precision):
    ctx = tmp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, case, precision, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        res = dict(out)
    wl = _CASES[case]()
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-11, maxiter=600)
    x0, pix0, hits0, it0, conv0, ncut0 = res[0]
    x1 = res[1][0]
    assert np.array_equal(x0, x1)  # replicated on every rank
    assert conv0
    lst = o.bj.A.lindices[3 * o.bj.A.trash_pix::3] // 3
    assert np.array_equal(pix0, lst)
    assert np.array_equal(hits0, np.asarray(o.bj.hits))
    if precision == "fp64":
        assert abs(it0 - o.iters) <= 1
    det = np.ones(len(x0), dtype=bool)
    if case == "cut_gaps":
        assert ncut0 > 0
        W, _ = R.local_W(o.bj.A, wl.block_sizes, wl.lam, wl.invtt)
        ev = np.linalg.eigvalsh(W)
        det = np.repeat(ev[:, 0] > 1e-6 * ev[:, 2], 3)
    for k in range(3):
        sel = det[k::3]
        assert _rel(x0[k::3][sel], o.x[k::3][sel]) < 1e-8, (k, _rel(x0[k::3][sel], o.x[k::3][sel]))


def _mlmap_worker(rank, world, port, outdir):
    """MLmap as a MAPPRAISER caller with one rank per process calls it: each rank
    passes data_size_proc (all ranks) and its own samples and blocks."""
    import torch.distributed as dist
    from midapack_b200 import mappraiser_wrapper as mw
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = _MLMAP_CASE()
        pix, w, sig, noi, bs, lam, tt = _split(wl, rank, world)
        dsp = np.array([len(_split(wl, r, world)[2]) for r in range(world)], dtype=np.int32)
        params = dict(path_output=outdir, ref="sh", solver=0, precond=0, Z_2lvl=0, ptcomm_flag=6, tol=1e-10,
                      maxiter=600, enlFac=1, ortho_alg=1, bs_red=0, nside=wl.nside, Lambda=lam)
        mw.MLmap(dist.group.WORLD, params, dsp, len(bs), bs, 3, pix, w, sig, noi, tt,
                 shard=OracleShard(pix, w, sig, noi, bs, lam, tt))
    finally:
        dist.destroy_process_group()


# 2 x 8 x 24 flat grid sized so that 12 nside^2 pixels cover it (nside 8)
_MLMAP_CASE = lambda: synth.make_workload("mlmap2", 32, 24, 4, 2048, 1024, 32, seed=43, gap_frac=0.02)  # noqa: E731


def test_mlmap_on_two_ranks_writes_the_reference_maps(ref_lib, tmp_path):
    """MLmap with a two-rank process group (gloo, CPU; the oracle's operators as
    each rank's shard): rank 0's FITS maps against the reference's own MLmap
    (oracle/_ref) on two forked ranks with the same split (mappraiser.c:64-88):
    Hits equal, Cond within 1e-12, I/Q/U within 1e-8 on the observed pixels."""
    from midapack_b200 import mappraiser_wrapper as mw
    wl = _MLMAP_CASE()
    assert wl.nside == 8
    ctx = tmp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_mlmap_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    maps = [mw.read_fits_map(str(tmp_path / f"{k}_sh.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    half = wl.n_samples // 2
    nb = len(wl.block_sizes)
    I, Q, U, Cond, Hits, res = ref_lib.mlmap(2, [half, half], [nb // 2, nb // 2], wl.block_sizes, wl.pix, wl.weights,
                                             wl.signal, wl.noise, wl.lam, wl.invtt, wl.nside, tol=1e-10, maxiter=600)
    np.testing.assert_array_equal(maps[4], Hits)
    obs = Hits > 0
    np.testing.assert_allclose(maps[3][obs], Cond[obs], rtol=1e-12, atol=0)
    for mine, theirs in zip(maps[:3], (I, Q, U)):
        assert _rel(mine[obs], theirs[obs]) < 1e-8
    rr = np.fromfile(str(tmp_path / "pcg_residuals_sh.dat"))
    assert rr[0] == 1.0 and abs(len(rr) - len(res)) <= 1
