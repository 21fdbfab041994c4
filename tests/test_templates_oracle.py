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


def _product_scan(sc):
    from midapack_b200 import templates
    return templates.Scan(sc.sweeps, sc.az, sc.az_min, sc.az_max, sc.hwp, sc.ndet, sc.npoly, sc.ground,
                          sc.n_sss_bins, sc.nhwp, sc.delta_t, sc.fs)


@pytest.mark.parametrize("name", list(VARIANTS))
def test_library_layout_matches_restatement(name):
    """mdp_template_layout (host set-up in the library) against the restated basis."""
    from midapack_b200 import templates
    sc, *_ = template_case(**VARIANTS[name])
    bins, wg, nt = templates.layout(_product_scan(sc))
    at = 0
    for i in range(sc.nces):
        Phi = restate.template_basis(sc, i)
        L = Phi.shape[0]
        assert nt[i] == Phi.shape[1]
        mine = np.zeros_like(Phi)
        for c in range(bins.shape[1]):
            np.add.at(mine, (np.arange(L), bins[at:at + L, c]), wg[at:at + L, c])
        assert np.abs(mine - Phi).max() <= 1e-14
        at += L


@pytest.mark.parametrize("name", list(VARIANTS))
def test_library_kernels_match_reference(ref_lib, name):
    """mdp_template_kernels against the reference's BuildKernel + InvKernel."""
    from midapack_b200 import templates
    sc, pix, w, sig, noi, invtt, nside = template_case(**VARIANTS[name])
    _, _, _, kinv = ref_lib.templates_ops(sc, invtt, np.zeros(sig.size), np.zeros(sc.n_templates))
    mine = templates.kernels(_product_scan(sc), invtt)
    assert rel(mine, kinv) <= 1e-9


def test_library_layout_rejects_bad_scans():
    from midapack_b200 import MidapackError, templates
    sc, *_ = template_case()
    bad = _product_scan(sc)
    bad.sweeps = [np.array([5, 600, 1200]), sc.sweeps[1]]
    with pytest.raises(MidapackError, match="sample 0"):
        templates.layout(bad)
    bad.sweeps = [np.array([0, 1, 1200]), sc.sweeps[1]]
    with pytest.raises(MidapackError, match="fewer than 2"):
        templates.layout(bad)
    bad = _product_scan(sc)
    bad.az_min = np.array([15.0, 10.0])
    with pytest.raises(MidapackError, match="below az_min"):
        templates.layout(bad)


def test_mtmap_with_library_kernels_matches_reference(ref_lib):
    """The templates solve with the library's kernels (mdp_template_kernels) in place
    of numpy's gives the reference MTmap's maps."""
    from midapack_b200 import templates
    sc, pix, w, sig, noi, invtt, nside = template_case()
    I, Q, U, Cond, Hits, res = ref_lib.mtmap(sc, pix, w, sig, noi, invtt, nside, tol=1e-10, maxiter=500)
    kinv = templates.kernels(_product_scan(sc), invtt)
    r = restate.pcg_templates(pix, w, sig, noi, sc, invtt, tol=1e-10, maxiter=500, kinv=kinv)
    assert r.iters == len(res) - 1
    A = r.bj.A
    mI, mQ, mU, _, _ = restate.x2map_pol(r.x, A.lindices[A.nnz * A.trash_pix:], np.zeros(r.x.size // 3),
                                         np.zeros(r.x.size // 3, dtype=np.int32), 12 * nside * nside)
    obs = Hits > 0
    for mine, theirs in ((mI, I), (mQ, Q), (mU, U)):
        assert rel(mine[obs], theirs[obs]) <= 1e-9
