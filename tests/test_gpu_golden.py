"""The CUDA path against the golden vectors produced by the reference's own
compiled code (tests/golden/): the reference's data_bin fixture (HEALPix
nside 512 pointing, lambda 8192) and seeded synthetic cases.  N^-1 is held to
1e-12 of the exact banded product; the gap to the reference's own output is
bounded by the reference's measured error on the same input (its
scmm_direct aliasing, toeplitz.c:585-589)."""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_gpu_matches_reference_golden(gpu_ctx, path):
    import torch
    import midapack_b200 as mb
    g = np.load(path)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    m = len(g["signal"])
    lam = int(g["lam"])
    w = d(g["weights"])
    P = mb.Pointing(gpu_ctx, d(g["pix"]), w, m, 3)
    assert np.array_equal(P.lindices().cpu().numpy(), g["lindices"])
    assert np.array_equal(P.local_indices().cpu().numpy(), g["local"])
    n = P.shape()["n_map"]
    y = torch.empty(m, dtype=torch.float64, device="cuda")
    P.matvec(d(g["x_in"]), y)
    assert _rel(y.cpu().numpy(), g["Px"]) < 1e-13
    xt = torch.empty(n, dtype=torch.float64, device="cuda")
    P.trmatvec(d(g["t_in"]), xt)
    assert _rel(xt.cpu().numpy(), g["Ptt"]) < 1e-13
    N = mb.Noise(gpu_ctx, g["block_sizes"], lam, g["invtt"])
    nv = torch.empty(m, dtype=torch.float64, device="cuda")
    N.apply(d(g["v_in"]), nv)
    from oracle import restate as R
    exact = R.stbmm(g["v_in"], g["block_sizes"], lam, g["invtt"], exact=True)
    ref_err = _rel(g["Nv"], exact)  # the reference's own error on this input
    assert _rel(nv.cpu().numpy(), exact) < 1e-12
    assert _rel(nv.cpu().numpy(), g["Nv"]) < max(1e-12, 2 * ref_err)
    P2 = mb.Pointing(gpu_ctx, d(g["pix"]), w, m, 3)
    x, lst, cond, hits, res, info = mb.gls_solve(gpu_ctx, P2, N, d(g["signal"]), d(g["noise"]), tol=float(g["tol"]),
                                                 maxiter=int(g["maxiter"]))
    assert np.array_equal(lst.cpu().numpy(), g["lstid"])
    assert np.array_equal(hits.cpu().numpy(), g["hits"])
    assert np.allclose(cond.cpu().numpy(), g["cond"], rtol=1e-12, atol=0)
    assert abs(info.iterations - (len(g["res_rel"]) - 1)) <= 1
    assert _rel(x.cpu().numpy(), g["x_sol"]) < max(1e-10, 1e3 * ref_err)
