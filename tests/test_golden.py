"""The oracle restatement against the golden vectors produced by the
reference's own compiled code (tests/golden/make_golden.py): index
compression bit-exact, P/P^T within 1e-13, N^-1 within 1e-12 of the exact
banded product, the PCG solution within 1e-10 with the same iteration count.
On the reference's own data (T0 ~ 1e7) the reference's stbmmProd itself
deviates from the exact product by ~4e-10: scmm_direct (toeplitz.c:585-589)
computes the imaginary part of the spectrum product from the already updated
real part, an error of the size of the spectrum's imaginary round-off.  The
gap to the reference is therefore bounded by that measured error.  CPU only."""
import glob
import os

import numpy as np
import pytest

from oracle import restate as R

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_restatement_matches_reference_golden(path):
    g = np.load(path)
    m = len(g["signal"])
    A = R.local_shape(g["pix"], g["weights"], m, 3)
    assert np.array_equal(A.lindices, g["lindices"])
    assert np.array_equal(A.local, g["local"])
    assert A.trash_pix == int(g["trash"])
    assert _rel(R.matvec(A, g["x_in"]), g["Px"]) < 1e-13
    assert _rel(R.trmatvec(A, g["t_in"]), g["Ptt"]) < 1e-13
    lam = int(g["lam"])
    exact = R.stbmm(g["v_in"], g["block_sizes"], lam, g["invtt"], exact=True)
    ref_err = _rel(g["Nv"], exact)  # the reference's own error (toeplitz.c:585-589 aliasing)
    ours = R.stbmm(g["v_in"], g["block_sizes"], lam, g["invtt"])
    assert _rel(ours, exact) < 1e-12
    assert _rel(ours, g["Nv"]) < max(1e-12, 2 * ref_err)
    o = R.pcg(g["pix"], g["weights"], g["signal"], g["noise"], g["block_sizes"], lam, g["invtt"], tol=float(g["tol"]),
              maxiter=int(g["maxiter"]))
    assert np.array_equal(o.bj.A.lindices[3 * o.bj.A.trash_pix:], g["lstid"])
    assert np.array_equal(o.bj.hits, g["hits"])
    assert np.allclose(o.bj.cond, g["cond"], rtol=1e-12, atol=0)
    assert abs(o.iters - (len(g["res_rel"]) - 1)) <= 1
    assert _rel(o.x, g["x_sol"]) < max(1e-10, 1e3 * ref_err)
