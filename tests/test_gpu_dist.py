"""Sharded solve (midapack_b200.dist) with the GPU shard: one NCCL rank, and
two gloo ranks sharing the GPU (their collectives go through host memory, so
no kernel waits on another rank), each holding half of the detectors; the map
must equal the single-process device solve of the whole data (FP64: 1e-10
relative per I/Q/U; mixed precision: 1e-8)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from midapack_b200 import synth

pytestmark = pytest.mark.gpu


def _case():
    return synth.small(n_det=4, n_samp=4096, block_len=2048, lam=64, gap_frac=0.02, seed=51)


def _split(wl, rank, world):
    nd = wl.n_det
    d0, d1 = rank * nd // world, (rank + 1) * nd // world
    s0, s1 = d0 * wl.n_samp, d1 * wl.n_samp
    nb_per = wl.n_samp // wl.block_len
    bs = wl.block_sizes[d0 * nb_per:d1 * nb_per]
    tt = wl.invtt[d0 * nb_per * wl.lam:d1 * nb_per * wl.lam]
    return (wl.pix[3 * s0:3 * s1], wl.weights[3 * s0:3 * s1], wl.signal[s0:s1], wl.noise[s0:s1], bs, wl.lam, tt)


def _worker(rank, world, port, backend, precision, out):
    import torch
    import torch.distributed as dist
    import midapack_b200 as mb
    from midapack_b200.dist import GpuShard, ShardedGLS
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world)
    try:
        pix, w, sig, nz, bs, lam, tt = _split(_case(), rank, world)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        ctx = mb.Context(0)
        shard = GpuShard(ctx, d(pix), d(w), d(sig), d(nz), bs, lam, tt)
        x, pg, rcond, hits, info = ShardedGLS(shard).solve(tol=1e-12, maxiter=900, precision=precision)
        out[rank] = (x.cpu().numpy(), pg.cpu().numpy(), hits.cpu().numpy(), info.iterations, info.converged)
        shard.close()
        ctx.close()
    finally:
        dist.destroy_process_group()


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, backend, precision):
    ctx = tmp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, backend, precision, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(600)
            assert p.exitcode == 0
        return dict(out)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("world,backend,precision", [(1, "nccl", "fp64"), (2, "gloo", "fp64"), (2, "gloo", "mixed")])
def test_sharded_matches_single_process(gpu_ctx, world, backend, precision):
    import torch
    import midapack_b200 as mb
    res = _run(world, backend, precision)
    wl = _case()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), wl.n_samples, 3)
    N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
    x1, lst, cond, hits, _, info = mb.gls_solve(gpu_ctx, P, N, d(wl.signal), d(wl.noise), tol=1e-12, maxiter=900)
    x1, lst, hits = x1.cpu().numpy(), lst.cpu().numpy(), hits.cpu().numpy()
    x0, pg, h0, it0, conv = res[0]
    assert conv
    for r in range(1, world):
        assert np.array_equal(res[r][0], x0)  # replicated on every rank
    assert np.array_equal(pg, lst[0::3] // 3)
    assert np.array_equal(h0, hits)
    tol = 1e-10 if precision == "fp64" else 1e-8
    for k in range(3):
        assert _rel(x0[k::3], x1[k::3]) < tol, (k, _rel(x0[k::3], x1[k::3]))
