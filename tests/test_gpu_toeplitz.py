"""N^-1 (block mean removal + banded Toeplitz, overlap-save FFT) on the GPU vs
the oracle's exact long-double banded product.  Tolerance: 1e-12 norm-wise
relative per application (FP64)."""

import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _run(gpu_ctx, block_sizes, lam, invtt, v, fft=None):
    import torch
    import midapack_b200 as mb
    N = mb.Noise(gpu_ctx, block_sizes, lam, invtt)
    if fft:
        N.set_plan(fft if isinstance(fft, str) else f"fft:{fft}")
    vin = torch.from_numpy(v).cuda()
    vout = torch.empty_like(vin)
    N.apply(vin, vout)
    torch.cuda.synchronize()
    return vout.cpu().numpy(), N.tile()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("lam,sizes,fft", [
    (1, [100, 37], None),            # white noise: diagonal scaling, no mean removal
    (2, [50, 9, 64], None),
    (16, [1000, 333], None),
    (64, [4096, 777, 130], None),     # ragged blocks, one shorter than a tile
    (300, [5000, 600], None),         # lambda not a power of two
    (100, [3000], 512),               # forced small tile: many tiles per block
    (2048, [20000, 4100], None),
    (4096, [40000], 16384),           # largest single-CTA tile
    (4096, [40000, 9000], 32768),     # 2-CTA cluster tile (distributed shared memory)
    (8192, [24000, 24000], None),     # the reference fixture's shape
    (8192, [70000], 65536),           # 4-CTA cluster tile
    (16384, [140000], 131072),        # 8-CTA cluster tile
    (4096, [40000, 9000], "c,2"),     # cluster four-step tiles: 2, 4, 8 CTAs (2C x 4096 points)
    (8192, [70000, 9000], "c,4"),
    (16384, [140000, 40000], "c,8"),
    (16384, [300000], "c,8"),         # four tiles of the at-scale plan: interior and edge tiles
    (100, [300000, 5000], "c,8"),     # narrow band: blocks shorter than a tile, windows past both ends
])
def test_stbmm_vs_exact(gpu_ctx, lam, sizes, fft):
    rng = np.random.default_rng(lam + len(sizes))
    t = np.zeros(lam)
    t[0] = 2.0
    if lam > 1:
        t[1:] = rng.standard_normal(lam - 1) * np.exp(-np.arange(1, lam) / (0.3 * lam))
    invtt = np.tile(t, len(sizes))
    v = rng.standard_normal(int(sum(sizes))) + 3.0
    out, tile = _run(gpu_ctx, sizes, lam, invtt, v, fft)
    ref = R.stbmm(v, np.array(sizes), lam, invtt, exact=True)
    assert _rel(out, ref) < TOL, (tile, _rel(out, ref))


def test_stbmm_distinct_blocks(gpu_ctx):
    """Blocks with different first rows get their own spectra."""
    rng = np.random.default_rng(4)
    lam, sizes = 128, [3000, 2500, 4000]
    invtt = np.concatenate([synth.invtt_row(4096, lam, fk) for fk in (0.1, 1.0, 5.0)])
    v = rng.standard_normal(sum(sizes))
    out, _ = _run(gpu_ctx, sizes, lam, invtt, v)
    ref = R.stbmm(v, np.array(sizes), lam, invtt, exact=True)
    assert _rel(out, ref) < TOL


def test_stbmm_noise_model_full_block(gpu_ctx):
    """The 1/f inverse-noise row of the 2^20-sample, lambda 2^12 workload, one block,
    against the oracle's FFT product (exact within FP64 rounding)."""
    n, lam = 1 << 20, 1 << 12
    row = synth.invtt_row(n, lam, 1.0)
    rng = np.random.default_rng(9)
    v = synth.noise_tod(n, 1.0, rng)
    out, tile = _run(gpu_ctx, [n], lam, row, v)
    ref = R.stbmm(v, np.array([n]), lam, row)
    assert _rel(out, ref) < TOL, tile


def test_stbmm_in_place(gpu_ctx):
    import torch
    import midapack_b200 as mb
    rng = np.random.default_rng(2)
    lam, sizes = 64, [2000, 1500]
    invtt = np.tile(synth.invtt_row(2048, lam, 1.0), 2)
    v = rng.standard_normal(sum(sizes))
    N = mb.Noise(gpu_ctx, sizes, lam, invtt)
    d = torch.from_numpy(v.copy()).cuda()
    N.apply(d, d)
    torch.cuda.synchronize()
    ref = R.stbmm(v, np.array(sizes), lam, invtt, exact=True)
    assert _rel(d.cpu().numpy(), ref) < TOL


def test_stbmm_rejects_band_wider_than_block(gpu_ctx):
    import midapack_b200 as mb
    with pytest.raises(mb.MidapackError):
        mb.Noise(gpu_ctx, [10], 64, np.ones(64))


@pytest.mark.parametrize("lam,sizes,plan", [
    (16, [1000, 333], "s,4,5"),              # smallest split tile: 16 x 32 points
    (64, [4096, 777, 130], "s,5,5"),          # ragged blocks, one shorter than a tile
    (300, [5000, 600], "s,5,6"),              # lambda not a power of two
    (2048, [20000, 4100], "s,6,8"),
    (4096, [40000, 9000], "s,7,8"),
    (8192, [70000], "s,8,8"),
    (16384, [140000, 3 * 16384], "s,8,9"),    # largest split tile: 256 x 512 points
    (64, [4096, 777, 130], "c,2"),            # cluster four-step tiles: blocks far shorter than a tile
    (2048, [20000, 4100, 65537], "c,4"),
    (16384, [140000, 3 * 16384], "c,8"),
])
def test_stbmm_split_plan_vs_exact(gpu_ctx, lam, sizes, plan):
    """The three-kernel (four-step FFT) tile plans and the cluster four-step
    plans, FP64 and FP32."""
    import torch
    import midapack_b200 as mb
    rng = np.random.default_rng(lam + 7)
    t = np.zeros(lam)
    t[0] = 2.0
    t[1:] = rng.standard_normal(lam - 1) * np.exp(-np.arange(1, lam) / (0.3 * lam))
    invtt = np.tile(t, len(sizes))
    v = rng.standard_normal(int(sum(sizes))) + 3.0
    N = mb.Noise(gpu_ctx, sizes, lam, invtt).set_plan(plan).set_plan(plan, fp32=True)
    tile, tile32 = N.tile(), N.tile_fp32()
    if plan[0] == "s":
        m1, m2 = (int(x) for x in plan.split(",")[1:])
        assert tile["split"] == [1 << m1, 1 << m2] and tile32["split"] == [1 << m1, 1 << m2]
    else:
        shape = [2 * int(plan.split(",")[1]), 4096]
        assert tile["cluster_four_step"] == shape and tile32["cluster_four_step"] == shape
    vin = torch.from_numpy(v).cuda()
    vout = torch.empty_like(vin)
    N.apply(vin, vout)
    v32 = vin.float()
    o32 = torch.empty_like(v32)
    N.apply_fp32(v32, o32)
    torch.cuda.synchronize()
    ref = R.stbmm(v, np.array(sizes), lam, invtt, exact=True)
    assert _rel(vout.cpu().numpy(), ref) < TOL
    ref32 = R.stbmm(v32.double().cpu().numpy(), np.array(sizes), lam, invtt, exact=True)
    assert _rel(o32.double().cpu().numpy(), ref32) < 1e-5


def test_split_plans_of_two_operators_share_kernels(gpu_ctx):
    """Two operators whose split plans launch the same column kernel with
    different shared-memory sizes (256 x 512 and 256 x 256 points): the plan
    built second must not break the launches of the first."""
    import torch
    import midapack_b200 as mb
    ops = []
    for lam, sizes, plan in [(16384, [140000], "s,8,9"), (8192, [70000], "s,8,8")]:
        rng = np.random.default_rng(lam)
        t = np.zeros(lam)
        t[0] = 2.0
        t[1:] = rng.standard_normal(lam - 1) * np.exp(-np.arange(1, lam) / (0.3 * lam))
        N = mb.Noise(gpu_ctx, sizes, lam, np.tile(t, len(sizes))).set_plan(plan).set_plan(plan, fp32=True)
        ops.append((N, sizes, lam, np.tile(t, len(sizes))))
    for N, sizes, lam, invtt in ops:
        v = np.random.default_rng(lam + 1).standard_normal(int(sum(sizes)))
        vin = torch.from_numpy(v).cuda()
        vout = torch.empty_like(vin)
        N.apply(vin, vout)
        o32 = torch.empty(vin.shape, dtype=torch.float32, device="cuda")
        N.apply_fp32(vin.float(), o32)
        torch.cuda.synchronize()
        ref = R.stbmm(v, np.array(sizes), lam, invtt, exact=True)
        assert _rel(vout.cpu().numpy(), ref) < TOL
        assert _rel(o32.double().cpu().numpy(), ref) < 1e-5
