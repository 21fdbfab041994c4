"""Device noise2invtt (libmidapack_b200: mdp_apod_window, mdp_periodogram,
mdp_noise2invtt) against the oracle (the scipy restatement of
mappraiser/python/TOAST_interface/utils.py:500-602) and against the golden
outputs of the reference's own function.

Tolerances: windows and periodograms are FP64 transforms of the same data,
checked to 1e-14 (absolute, windows peak at 1; the chebwin against a 30-digit
evaluation, since scipy's own chebwin is off by up to 5e-9) and 1e-12
(relative norm).  The
inverse-noise rows come out of a nonlinear fit: the device fit runs to the
least-squares minimum, so its cost is checked to be no higher than that of
curve_fit run to ftol = xtol = gtol = 1e-15 (times 1 + 1e-12), and its rows
against that fit's rows to 1e-6 (relative norm: the minimum is flat along
(alpha, fmin), where costs equal to 1e-14 still move the rows by ~1e-7); the
reference's own curve_fit stops at ftol = 1e-8, so its rows are checked to
1e-4."""
import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate
from tests._cases import noise_golden

pytestmark = pytest.mark.gpu
CASES = noise_golden()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("lam", [8, 64, 1000, 4096, 16384])
def test_chebwin_window(gpu_ctx, lam):
    """Against the 30-digit evaluation of the same window to 1e-14, and against
    scipy's (the reference's) window to scipy's own error plus 1e-14."""
    from midapack_b200 import noise
    got = noise.apod_window(lam, "chebwin", ctx=gpu_ctx).cpu().numpy()
    exact = restate.chebwin_exact(lam)
    ref = restate.apod_window(lam, "chebwin")
    assert np.abs(got - exact).max() <= 1e-14
    assert np.abs(got - ref).max() <= np.abs(ref - exact).max() + 1e-14


@pytest.mark.parametrize("lam", [8, 1000, 16384])
def test_gaussian_window(gpu_ctx, lam):
    from midapack_b200 import noise
    got = noise.apod_window(lam, "gaussian", ctx=gpu_ctx).cpu().numpy()
    assert np.abs(got - restate.apod_window(lam, "gaussian")).max() <= 1e-14


@pytest.mark.parametrize("sizes", [[16], [17], [1000, 1000], [1024, 1024, 1024], [4097], [8192, 8192], [65536],
                                   [100003], [1 << 20], [1024, 1000, 4097, 8192, 8192, 17]],
                         ids=lambda s: "-".join(map(str, s)))
def test_periodogram(gpu_ctx, sizes):
    from midapack_b200 import noise
    rng = np.random.default_rng(sum(sizes))
    total = sum(sizes)
    x = rng.standard_normal(total) + 3.0 + 1e-3 * np.arange(total)   # offset and trend: the detrend is exercised
    got = noise.periodogram(x, sizes, 37.0, ctx=gpu_ctx).cpu().numpy()
    assert got.size == sum(n // 2 + 1 for n in sizes)
    at = off = 0
    for n in sizes:
        _, ref = restate.periodogram(x[off:off + n], 37.0)
        g = got[at:at + n // 2 + 1]
        assert rel(g, ref) <= 1e-12, n
        assert np.abs(np.log10(g[1:]) - np.log10(ref[1:])).max() <= 1e-8, n
        at += n // 2 + 1
        off += n


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_noise2invtt_matches_oracle_and_reference(gpu_ctx, case):
    from midapack_b200 import noise
    n0 = gpu_ctx.launches
    out, params, evals = noise.invtt_blocks(case["noise"], [case["n"]], case["lam"], case["fsamp"], case["apod"],
                                            ctx=gpu_ctx, return_fit=True)
    got = out.cpu().numpy()
    tight, popt, psd = restate.noise2invtt(case["noise"], case["n"], case["lam"], case["fsamp"], case["apod"],
                                           tight=True)
    assert restate.fit_cost(psd, case["n"], case["fsamp"], params[0]) <= \
        restate.fit_cost(psd, case["n"], case["fsamp"], popt) * (1 + 1e-12)
    assert rel(got, tight) <= 1e-6
    assert rel(got, case["invtt"]) <= 1e-4
    assert 0 < evals[0] < 1000
    np.testing.assert_allclose(params[0][:3], popt[:3], rtol=1e-4)
    assert gpu_ctx.launches > n0


def test_compute_invtt_ragged_blocks(gpu_ctx):
    """compute_invtt over nobs x ndet blocks of different lengths (powers of two
    and not), written into the caller's buffer at (iobs*ndet + idet)*Lambda."""
    from midapack_b200 import noise
    sizes = [4096, 6000, 4096, 1000, 8192, 4096]
    lam = 256
    rng = np.random.default_rng(5)
    blocks = [synth.noise_tod(n, 0.3 + 0.5 * i, rng) for i, n in enumerate(sizes)]
    x = np.concatenate(blocks)
    buf = np.full(len(sizes) * lam + 3, -7.0)
    assert noise.compute_invtt(2, 3, x, np.array(sizes), lam, 100.0, buf, np.float64, ctx=gpu_ctx) is None
    for b, blk in enumerate(blocks):
        tight, _, _ = restate.noise2invtt(blk, sizes[b], lam, 100.0, "chebwin", tight=True)
        assert rel(buf[b * lam:(b + 1) * lam], tight) <= 1e-6, b
    assert np.all(buf[-3:] == -7.0)


def test_noise2invtt_interval_of_2p20_samples(gpu_ctx):
    """A stationary interval of 2^20 samples with lambda = 2^14 (the at-scale
    workload's block), twice in one batch: both rows equal bit for bit."""
    from midapack_b200 import noise
    n, lam = 1 << 20, 1 << 14
    x = synth.noise_tod(n, 1.0, np.random.default_rng(99))
    out = noise.invtt_blocks(np.concatenate([x, x]), [n, n], lam, 100.0, "chebwin", ctx=gpu_ctx).cpu().numpy()
    assert np.array_equal(out[:lam], out[lam:])
    tight, _, _ = restate.noise2invtt(x, n, lam, 100.0, "chebwin", tight=True)
    assert rel(out[:lam], tight) <= 1e-6


def test_noise2invtt_single_block_api(gpu_ctx):
    from midapack_b200 import noise
    c = CASES[1]
    got = noise.noise2invtt(c["noise"], c["n"], c["lam"], c["fsamp"], 0, np.float64, c["apod"], ctx=gpu_ctx)
    assert got.dtype == np.float64 and got.shape == (c["lam"],)
    assert rel(got, c["invtt"]) <= 1e-4


def test_noise2invtt_errors(gpu_ctx):
    from midapack_b200 import MidapackError, noise
    x = synth.noise_tod(4096, 1.0, np.random.default_rng(3))
    bad = x.copy()
    bad[100] = np.nan
    with pytest.raises(MidapackError, match="non-finite"):
        noise.invtt_blocks(bad, [4096], 64, 100.0, ctx=gpu_ctx)
    with pytest.raises(MidapackError, match="samples"):
        noise.invtt_blocks(np.zeros(16), [6, 10], 2, 100.0, ctx=gpu_ctx)
    n = (1 << 23) + 1   # not a power of two: its Bluestein transform would need 2^25 points
    with pytest.raises(MidapackError, match="unsupported"):
        noise.invtt_blocks(np.zeros(n), [n], 64, 100.0, ctx=gpu_ctx)
    # the context stays usable
    c = CASES[1]
    out = noise.invtt_blocks(c["noise"], [c["n"]], c["lam"], c["fsamp"], c["apod"], ctx=gpu_ctx).cpu().numpy()
    assert rel(out, c["invtt"]) <= 1e-4
