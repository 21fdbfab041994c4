"""The templates path (MTmap: algebra/src/templates/templates.c,
mappraiser/src/pcg_true.c:243-560, mappraiser/src/mappraiser.c:387-800): the
numpy restatement (oracle/restate.py) against the reference's own compiled code
(oracle/_ref, ref_templates_ops / ref_mtmap).  No GPU."""
import numpy as np
import pytest

from oracle import restate
from tests._cases import template_case

VARIANTS = {
    "poly2_sss8_hwp2": dict(npoly=2, ground=1, n_sss_bins=8, nhwp=2),
    "poly3_only": dict(npoly=3, ground=0, n_sss_bins=0, nhwp=0),
    "sss16_only": dict(npoly=0, ground=1, n_sss_bins=16, nhwp=0),
    "poly1_hwp3": dict(npoly=1, ground=0, n_sss_bins=0, nhwp=3, delta_t=2.5),
}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", list(VARIANTS))
def test_template_operators_match_reference(ref_lib, name):
    sc, pix, w, sig, noi, invtt, nside = template_case(**VARIANTS[name])
    rng = np.random.default_rng(2)
    d = rng.standard_normal(sig.size)
    tau = rng.standard_normal(sc.n_templates)
    amp, tod, kern, kinv = ref_lib.templates_ops(sc, invtt, d, tau)
    amp2, tod2, kern2, kinv2 = restate.templates_ops(sc, invtt, d, tau)
    assert rel(amp2, amp) <= 1e-13
    assert rel(tod2, tod) <= 1e-13
    assert rel(kern2, kern) <= 1e-12
    assert rel(kinv2, kinv) <= 1e-9


@pytest.mark.parametrize("name", ["poly2_sss8_hwp2", "poly3_only", "poly1_hwp3"])
def test_mtmap_matches_reference(ref_lib, name):
    sc, pix, w, sig, noi, invtt, nside = template_case(**VARIANTS[name])
    I, Q, U, Cond, Hits, res = ref_lib.mtmap(sc, pix, w, sig, noi, invtt, nside, tol=1e-10, maxiter=500)
    r = restate.pcg_templates(pix, w, sig, noi, sc, invtt, tol=1e-10, maxiter=500)
    assert r.iters == len(res) - 1
    np.testing.assert_allclose(r.res_rel, res, rtol=1e-6, atol=1e-14)
    A = r.bj.A
    mI, mQ, mU, _, _ = restate.x2map_pol(r.x, A.lindices[A.nnz * A.trash_pix:], np.zeros(r.x.size // 3),
                                         np.zeros(r.x.size // 3, dtype=np.int32), 12 * nside * nside)
    obs = Hits > 0
    for mine, theirs in ((mI, I), (mQ, Q), (mU, U)):
        assert rel(mine[obs], theirs[obs]) <= 1e-10


def test_filter_removes_the_template_space():
    """F = N^-1 - N^-1 T (T^T N^-1 T)^+ T^T N^-1 with white N: F T tau = 0."""
    sc, *_ = template_case()
    rng = np.random.default_rng(4)
    tau = rng.standard_normal(sc.n_templates)
    _, tod, _, kinv = restate.templates_ops(sc, np.ones(sc.nces * sc.ndet), np.zeros(sum(sc.block_sizes)), tau)
    at = ta = ka = 0
    for i in range(sc.nces):
        Phi = restate.template_basis(sc, i)
        L, nt = Phi.shape
        for _ in range(sc.ndet):
            B = kinv[ka:ka + nt * nt].reshape(nt, nt)
            v = tod[at:at + L]
            assert np.linalg.norm(v - Phi @ (B @ (Phi.T @ v))) <= 1e-10 * np.linalg.norm(v)
            at += L
            ta += nt
            ka += nt * nt
