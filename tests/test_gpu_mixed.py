"""Mixed precision: the FP32 inverse-noise operator against the exact product
(FP32 tolerance 1e-5 norm-wise), and the mixed-precision solve (FP32 operator
inside FP64 iterative refinement) against the FP64 GPU solve and the oracle:
maps within 1e-8 relative, max over I/Q/U."""

import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R
from tests._cases import solver_cases

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("lam,sizes,fft", [
    (64, [5000, 777], None),
    (300, [9000], None),
    (2048, [40000, 5000], None),
    (4096, [70000], 32768),     # single FP32 CTA
    (8192, [70000], 65536),     # 2-CTA cluster
    (16384, [140000], 131072),  # 4-CTA cluster
    (16384, [300000], 262144),  # 8-CTA cluster
])
def test_stbmm_fp32_vs_exact(gpu_ctx, lam, sizes, fft):
    import torch
    import midapack_b200 as mb
    rng = np.random.default_rng(lam)
    invtt = np.tile(synth.invtt_row(max(4 * lam, 4096), lam, 1.0), len(sizes))
    v = rng.standard_normal(sum(sizes)) + 1.0
    N = mb.Noise(gpu_ctx, sizes, lam, invtt)
    if fft:
        N.set_plan(fft if isinstance(fft, str) else f"fft:{fft}", fp32=True)
    vin = torch.from_numpy(v).float().cuda()
    out = torch.empty_like(vin)
    N.apply_fp32(vin, out)
    torch.cuda.synchronize()
    ref = R.stbmm(v.astype(np.float32).astype(np.float64), np.array(sizes), lam, invtt,
                  exact=sum(sizes) * lam < 3e8)
    assert _rel(out.double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("plan32", [None, "s,5,5", "c,2"])
@pytest.mark.parametrize("case", ["gaps", "cut", "cut_gaps"])
def test_mixed_solve_matches_fp64(gpu_ctx, case, plan32):
    import torch
    import midapack_b200 as mb
    wl = solver_cases()[case]()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    m = wl.n_samples
    outs = []
    for mixed in (False, True):
        w = d(wl.weights)
        P = mb.Pointing(gpu_ctx, d(wl.pix), w, m, 3)
        N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
        if plan32:
            N.set_plan(plan32, fp32=True)
        if mixed:
            mb.prepare_fp32(gpu_ctx, P, N)
        fn = mb.gls_solve_mixed if mixed else mb.gls_solve
        # the map error is bounded by cond(A) x the residual: solve to 1e-12 to compare maps at 1e-8
        x, lst, cond, hits, res, info = fn(gpu_ctx, P, N, d(wl.signal), d(wl.noise), tol=1e-12, maxiter=900)
        assert info.converged
        outs.append((x.cpu().numpy(), lst.cpu().numpy(), hits.cpu().numpy(), info))
    (x64, l64, h64, i64), (x32, l32, h32, i32) = outs
    assert np.array_equal(l64, l32) and np.array_equal(h64, h32)
    assert i32.outer_iterations >= 1 and i32.fp64_applications == i32.outer_iterations + 1
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-12, maxiter=900)
    # With flagged samples the cut rewrites the samples of the pixel after the
    # rank-one one (precond.c:521 against mappraiser.c:130-142), so the rank-one
    # pixel stays in the system: its Q/U directions are an exact null space of
    # P^T N^-1 P, where every solver keeps whatever its rounding put there.  The
    # maps are compared on the determined pixels.
    W, _ = R.local_W(o.bj.A, wl.block_sizes, wl.lam, wl.invtt)
    ev = np.linalg.eigvalsh(W)
    det = np.repeat(ev[:, 0] > 1e-6 * ev[:, 2], 3)
    assert case != "cut_gaps" or not det.all()
    for k in range(3):
        sel = det[k::3]
        assert _rel(x32[k::3][sel], x64[k::3][sel]) < 1e-8, (k, _rel(x32[k::3][sel], x64[k::3][sel]))
        assert _rel(x32[k::3][sel], o.x[k::3][sel]) < 1e-8


@pytest.mark.parametrize("plan", [None, "s,4,5", "s,5,5", "c,2"])
@pytest.mark.parametrize("sizes", [[1001, 3095, 39], [4096, 4096], [35, 8190]])
def test_fp32_operator_ragged_blocks(gpu_ctx, sizes, plan):
    """The FP32 operator P^T N^-1 P (FP32 P with four samples per thread and
    the chunks' unaligned heads and tails one by one, FP32 N^-1, P^T) against
    the oracle's FP64 operator on blocks whose starts are not multiples of
    four, with the plan the tuner picks and with split plans: within 1e-5
    relative; prepare_fp32 ahead of it gives the same product."""
    import torch
    import midapack_b200 as mb
    m = int(sum(sizes))
    wl = synth.small(n_det=1, n_samp=m, block_len=m, lam=32, gap_frac=0.02, seed=71)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    invtt = np.tile(wl.invtt[:32], len(sizes))
    A = R.local_shape(wl.pix, wl.weights, m, 3)
    h = np.random.default_rng(3).standard_normal(A.n)
    ref = R.trmatvec(A, R.stbmm(R.matvec(A, h), np.array(sizes), 32, invtt, exact=True))
    hd = d(h)
    outs = []
    for prepare in (False, True):
        P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), m, 3)
        N = mb.Noise(gpu_ctx, sizes, 32, invtt)
        if plan:
            N.set_plan(plan, fp32=True)
        if prepare:
            mb.prepare_fp32(gpu_ctx, P, N)
        else:
            N.tile_fp32()
        if plan and plan[0] == "s":
            assert N.tile_fp32()["split"] == [1 << int(v) for v in plan.split(",")[1:]]
        if plan and plan[0] == "c":
            assert N.tile_fp32()["cluster_four_step"] == [2 * int(plan.split(",")[1]), 4096]
        q = torch.empty(A.n, dtype=torch.float64, device="cuda")
        mb.check(mb.lib().mdp_apply_op(gpu_ctx.h, P.h, N.h, hd.data_ptr(), q.data_ptr(), 1), "mdp_apply_op")
        torch.cuda.synchronize()
        outs.append(q.cpu().numpy())
    assert _rel(outs[0], ref) < 1e-5, _rel(outs[0], ref)
    assert _rel(outs[1], outs[0]) < 1e-12  # below 2^20 rows P^T adds with atomics
