"""Multi-RHS mixed-precision solve: each column against the FP64 GPU solve of
the same column (maps within 1e-8 relative, max over I/Q/U), for 1, 2 and 4
slots with more columns than slots (converged columns leave their slot to the
next column), with and without the CUDA graph, with the timed slot choice,
and the signal column against the oracle."""
import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _case(nrhs):
    wl = synth.small(n_det=2, n_samp=4096, block_len=1024, lam=32, gap_frac=0.02, seed=31)
    noise = synth.mc_noise(wl.n_det, wl.n_samp, nrhs, wl.fknee, seed=5)
    return wl, noise


@pytest.mark.parametrize("slots,graph", [(1, True), (2, True), (4, True), (4, False), (0, True)])
def test_multi_matches_fp64_columns(gpu_ctx, slots, graph):
    import torch
    import midapack_b200 as mb
    nrhs = 5
    wl, noise = _case(nrhs)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    m = wl.n_samples
    P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), m, 3)
    N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
    x, lst, cond, hits, ci, info = mb.gls_solve_multi(gpu_ctx, P, N, d(noise), signal=d(wl.signal), signal_col=0,
                                                      tol=1e-12, maxiter=900, slots=slots, use_graph=graph)
    x = x.cpu().numpy()
    assert all(c.converged for c in ci)
    if slots:
        assert info.slots == slots
    assert info.graph == (1 if graph else 0)
    assert info.total_iterations == sum(c.iterations for c in ci)
    assert info.fp64_applications == sum(c.outer_iterations + 1 for c in ci)
    for r in range(nrhs):
        P1 = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), m, 3)
        N1 = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
        sig = wl.signal if r == 0 else np.zeros(m)
        x1, l1, c1, h1, _, i1 = mb.gls_solve(gpu_ctx, P1, N1, d(sig), d(noise[r].astype(np.float64)), tol=1e-12,
                                             maxiter=900)
        assert i1.converged
        assert np.array_equal(lst.cpu().numpy(), l1.cpu().numpy())
        assert np.array_equal(hits.cpu().numpy(), h1.cpu().numpy())
        x1 = x1.cpu().numpy()
        for k in range(3):
            assert _rel(x[r][k::3], x1[k::3]) < 1e-8, (r, k, _rel(x[r][k::3], x1[k::3]))
    o = R.pcg(wl.pix, wl.weights, wl.signal, noise[0].astype(np.float64), wl.block_sizes, wl.lam, wl.invtt,
              tol=1e-12, maxiter=900)
    for k in range(3):
        assert _rel(x[0][k::3], o.x[k::3]) < 1e-8


def test_multi_single_column(gpu_ctx):
    import torch
    import midapack_b200 as mb
    wl, noise = _case(1)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    m = wl.n_samples
    P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), m, 3)
    N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
    x, *_, ci, info = mb.gls_solve_multi(gpu_ctx, P, N, d(noise.astype(np.float64)), tol=1e-10, maxiter=500,
                                         slots=0)
    assert info.slots == 1 and ci[0].converged
    o = R.pcg(wl.pix, wl.weights, np.zeros(m), noise[0].astype(np.float64), wl.block_sizes, wl.lam, wl.invtt,
              tol=1e-12, maxiter=900)
    x = x.cpu().numpy()
    for k in range(3):
        assert _rel(x[0][k::3], o.x[k::3]) < 1e-6
