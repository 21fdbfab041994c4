"""MTmap's TOD weighting on the device (mdp_templates_filter:
W x - W T B T^T W x, PCG_GLS_templates, mappraiser/src/pcg_true.c:301-365,
433-462) against the oracle restatement of the template classes
(oracle/restate.template_basis, pinned to the reference's compiled
templates.c).  The device sums the template amplitudes with atomic adds, so the
bound is a relative 1e-12 with the library's own kernels B and 1e-10 with
numpy's pseudo-inverses."""
import numpy as np
import pytest

from oracle import restate
from tests._cases import template_case

pytestmark = pytest.mark.gpu

VARIANTS = {
    "poly2_sss8_hwp2": dict(npoly=2, ground=1, n_sss_bins=8, nhwp=2),
    "poly3_only": dict(npoly=3, ground=0, n_sss_bins=0, nhwp=0),
    "sss16_only": dict(npoly=0, ground=1, n_sss_bins=16, nhwp=0),
    "poly1_hwp3": dict(npoly=1, ground=0, n_sss_bins=0, nhwp=3, delta_t=2.5),
}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _scan(sc):
    from midapack_b200 import templates
    return templates.Scan(sc.sweeps, sc.az, sc.az_min, sc.az_max, sc.hwp, sc.ndet, sc.npoly, sc.ground,
                          sc.n_sss_bins, sc.nhwp, sc.delta_t, sc.fs)


def numpy_filter(sc, invtt, x, kinv=None):
    out = np.empty_like(x)
    at = ka = 0
    for i in range(sc.nces):
        Phi = restate.template_basis(sc, i)
        L, nt = Phi.shape
        for j in range(sc.ndet):
            w = invtt[i * sc.ndet + j]
            if kinv is None:
                B = np.linalg.pinv(w * (Phi.T @ Phi), rcond=1e-12)
            else:
                B = kinv[ka:ka + nt * nt].reshape(nt, nt)
            u = w * x[at:at + L]
            out[at:at + L] = u - w * (Phi @ (B @ (Phi.T @ u)))
            at += L
            ka += nt * nt
    return out


@pytest.mark.parametrize("name", list(VARIANTS))
def test_filter_matches_oracle(gpu_ctx, name):
    import torch
    from midapack_b200 import templates
    sc, pix, w, sig, noi, invtt, nside = template_case(**VARIANTS[name])
    F = templates.Filter(gpu_ctx, _scan(sc), invtt)
    assert F.m == sig.size and F.n_amplitudes == sc.n_templates
    x = np.random.default_rng(3).standard_normal(sig.size) + noi
    xt = torch.from_numpy(x).cuda()
    n0 = gpu_ctx.launches
    got = F(xt).cpu().numpy()
    assert gpu_ctx.launches == n0 + 3
    kinv = templates.kernels(_scan(sc), invtt)
    assert rel(got, numpy_filter(sc, invtt, x, kinv)) <= 1e-12
    assert rel(got, numpy_filter(sc, invtt, x)) <= 1e-10
    y = xt.clone()
    F(y, out=y)   # in place
    assert rel(y.cpu().numpy(), got) <= 1e-13
    F.close()


def test_filter_removes_the_templates(gpu_ctx):
    import torch
    from midapack_b200 import templates
    sc, pix, w, sig, noi, invtt, nside = template_case()
    tau = np.random.default_rng(5).standard_normal(sc.n_templates)
    _, tod, _, _ = restate.templates_ops(sc, invtt, np.zeros(sig.size), tau)
    F = templates.Filter(gpu_ctx, _scan(sc), invtt)
    got = F(torch.from_numpy(tod).cuda()).cpu().numpy()
    wt = tod * np.repeat(invtt, sc.block_sizes)
    assert np.linalg.norm(got) <= 1e-10 * np.linalg.norm(wt)


def test_filter_rejects_too_many_amplitudes(gpu_ctx):
    from midapack_b200 import MidapackError, templates
    sc, *_ = template_case(npoly=1, ground=0, n_sss_bins=0, nhwp=1, delta_t=0.005)   # 2 x 8192 HWP chunks
    with pytest.raises(MidapackError, match="unsupported"):
        templates.Filter(gpu_ctx, _scan(sc), np.ones(sc.nces * sc.ndet))
