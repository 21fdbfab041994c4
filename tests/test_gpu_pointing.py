"""Pointing matrix on the GPU vs the oracle: index compression bit-exact,
P and P^T within 1e-13 (FP64); P^T by map bins bit-reproducible."""
import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _cases():
    yield "triplet", synth.small(n_det=2, n_samp=4096, block_len=2048, lam=32), 3
    yield "triplet_gaps", synth.small(n_det=3, n_samp=2048, block_len=1024, lam=16, gap_frac=0.05, seed=3), 3


@pytest.mark.parametrize("case", ["triplet", "triplet_gaps"])
def test_compression_and_products(gpu_ctx, case):
    import torch
    import midapack_b200 as mb
    name, wl, nnz = [c for c in _cases() if c[0] == case][0]
    m = wl.n_samples
    A = R.local_shape(wl.pix, wl.weights, m, nnz)
    g = _dev(wl.pix)
    w = _dev(wl.weights)
    P = mb.Pointing(gpu_ctx, g, w, m, nnz)
    sh = P.shape()
    assert sh["lcount"] == A.lcount and sh["trash_pix"] == A.trash_pix and sh["triplet"] == 1
    assert np.array_equal(P.lindices().cpu().numpy(), A.lindices)
    assert np.array_equal(P.local_indices().cpu().numpy(), A.local)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(A.n)
    y = _dev(np.zeros(m))
    P.matvec(_dev(x), y)
    torch.cuda.synchronize()
    yr = R.matvec(A, x)
    assert np.linalg.norm(y.cpu().numpy() - yr) <= 1e-13 * np.linalg.norm(yr)
    t = rng.standard_normal(m)
    xo = _dev(np.zeros(A.n))
    P.trmatvec(_dev(t), xo)
    torch.cuda.synchronize()
    xr = R.trmatvec(A, t)
    assert np.linalg.norm(xo.cpu().numpy() - xr) <= 1e-13 * np.linalg.norm(xr)


@pytest.mark.parametrize("nnz", [1, 2, 3])
def test_general_layout(gpu_ctx, nnz):
    """Arbitrary (non-triplet) indices go through the general kernels."""
    import torch
    import midapack_b200 as mb
    rng = np.random.default_rng(10 + nnz)
    m = 5000
    gidx = rng.integers(0, 700, size=(m, nnz)).astype(np.int32)
    flagged = rng.random(m) < 0.05  # whole rows flagged: every entry negative, the first the smallest
    gidx[flagged] = -nnz + np.arange(nnz)
    gidx = gidx.reshape(-1)
    vals = rng.standard_normal(m * nnz)
    A = R.local_shape(gidx, vals, m, nnz)
    P = mb.Pointing(gpu_ctx, _dev(gidx), _dev(vals), m, nnz)
    sh = P.shape()
    assert sh["lcount"] == A.lcount and sh["trash_pix"] == A.trash_pix
    assert np.array_equal(P.lindices().cpu().numpy(), A.lindices)
    assert np.array_equal(P.local_indices().cpu().numpy(), A.local)
    x = rng.standard_normal(A.n)
    y = _dev(np.zeros(m))
    P.matvec(_dev(x), y)
    yr = R.matvec(A, x)
    assert np.allclose(y.cpu().numpy(), yr, rtol=0, atol=1e-13 * np.abs(yr).max())
    t = rng.standard_normal(m)
    xo = _dev(np.zeros(A.n))
    P.trmatvec(_dev(t), xo)
    torch.cuda.synchronize()
    xr = R.trmatvec(A, t)
    assert np.linalg.norm(xo.cpu().numpy() - xr) <= 1e-13 * np.linalg.norm(xr)


def test_adjoint_full_size(gpu_ctx):
    """<P x, y> == <x, P^T y> on the 4 det x 2^20 workload (size-independent property)."""
    import torch
    import midapack_b200 as mb
    cfg = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"])
    wl = synth.make_workload("c1", **cfg)
    m = wl.n_samples
    P = mb.Pointing(gpu_ctx, _dev(wl.pix), _dev(wl.weights), m, 3)
    n = P.shape()["n_map"]
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(m, dtype=torch.float64, device="cuda", generator=g)
    Px = torch.empty(m, dtype=torch.float64, device="cuda")
    Pty = torch.empty(n, dtype=torch.float64, device="cuda")
    P.matvec(x, Px)
    P.trmatvec(y, Pty)
    a = float(torch.dot(Px, y))
    b = float(torch.dot(x, Pty))
    assert abs(a - b) <= 1e-12 * (float(Px.norm()) * float(y.norm()))


def test_rejects_negative_index_in_valid_row(gpu_ctx):
    """A non-trash row holding a flagged index would make the reference read
    before the map (mapmat.c:711-719); it is rejected on creation."""
    import midapack_b200 as mb
    m, nnz = 100, 2
    gidx = np.arange(m * nnz, dtype=np.int32) + 10
    gidx[0:2] = [-2, -1]    # a trash row
    gidx[11] = -1           # row 5, second entry: invalid
    with pytest.raises(mb.MidapackError):
        mb.Pointing(gpu_ctx, _dev(gidx), _dev(np.ones(m * nnz)), m, nnz)


@pytest.mark.parametrize("gaps", [0.0, 0.02])
def test_binned_transpose_large(gpu_ctx, gaps):
    """From 2^20 samples on, P^T runs by map bins (shared-memory sums): same
    result as the oracle within 1e-13, including a partial last bin."""
    import torch
    import midapack_b200 as mb
    wl = synth.make_workload("big", 300, 170, 2, 1 << 20, 1 << 20, 64, gap_frac=gaps, seed=12)
    m = wl.n_samples
    A = R.local_shape(wl.pix, wl.weights, m, 3)
    P = mb.Pointing(gpu_ctx, _dev(wl.pix), _dev(wl.weights), m, 3)
    t = np.random.default_rng(3).standard_normal(m)
    xo = _dev(np.zeros(A.n))
    for _ in range(2):  # the bin list is built on the first call and reused
        P.trmatvec(_dev(t), xo)
        torch.cuda.synchronize()
        xr = R.trmatvec(A, t)
        assert np.linalg.norm(xo.cpu().numpy() - xr) <= 1e-13 * np.linalg.norm(xr)


@pytest.mark.parametrize("grid", [(40, 30), (4, 3)])
@pytest.mark.parametrize("fp32", [False, True])
def test_binned_transpose_is_reproducible(gpu_ctx, fp32, grid):
    """P^T by map bins adds every row in a fixed order (time order within a bin,
    lane order for rows of one step on one pixel): repeated applications, and
    two pointing objects built from the same arrays, give bit-identical maps;
    FP64 P^T, and the FP32 operator P^T N^-1 P of the mixed solver.  On the
    4 x 3 grid every step of 32 rows revisits pixels (the lane-order path)."""
    import torch
    import midapack_b200 as mb
    wl = synth.make_workload("rep", grid[0], grid[1], 3, 1 << 19, 1 << 19, 32, gap_frac=0.01, seed=14)
    m = wl.n_samples
    rng = np.random.default_rng(5)
    t = rng.standard_normal(m)
    outs = []
    for _ in range(2):
        P = mb.Pointing(gpu_ctx, _dev(wl.pix), _dev(wl.weights), m, 3)
        n = P.shape()["n_map"]
        h = _dev(np.random.default_rng(6).standard_normal(n))
        N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt) if fp32 else None
        for _ in range(2):
            xo = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
            if fp32:
                mb.check(mb.lib().mdp_apply_op(gpu_ctx.h, P.h, N.h, h.data_ptr(), xo.data_ptr(), 1), "mdp_apply_op")
            else:
                P.trmatvec(_dev(t), xo)
            torch.cuda.synchronize()
            outs.append(xo.cpu().numpy())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    A = R.local_shape(wl.pix, wl.weights, m, 3)
    if fp32:
        hh = np.random.default_rng(6).standard_normal(A.n)
        xr = R.trmatvec(A, R.stbmm(R.matvec(A, hh), wl.block_sizes, wl.lam, wl.invtt))
        assert np.linalg.norm(outs[0] - xr) <= 1e-5 * np.linalg.norm(xr)
    else:
        xr = R.trmatvec(A, t)
        assert np.linalg.norm(outs[0] - xr) <= 1e-13 * np.linalg.norm(xr)
