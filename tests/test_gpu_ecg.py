"""ECG (solver 1) on the GPU vs the restated enlarged CG (oracle/restate.ecg):
the same residual history over the first iterations (1e-6) and iteration
count (+-1); maps equal to the reference's PCG map (compiled reference, tol
1e-12) within 1e-8 on the determined pixels; Orthodir, the adaptive block
size, the host entry point ECG_GLS and MLmap with solver 1."""
import ctypes as ct
import os
import tempfile

import numpy as np
import pytest

from oracle import restate as R
from tests._cases import solver_cases

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _p(a, t):
    return a.ctypes.data_as(ct.POINTER(t))


def _gpu_ecg(ctx, wl, **kw):
    import torch
    import midapack_b200 as mb
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = mb.Pointing(ctx, d(wl.pix), d(wl.weights), wl.n_samples, 3)
    N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    x, lst, cond, hits, res, info = mb.gls_solve_ecg(ctx, P, N, d(wl.signal), d(wl.noise), **kw)
    return x.cpu().numpy(), lst.cpu().numpy(), cond.cpu().numpy(), hits.cpu().numpy(), res, info


def _determined(wl, A):
    W, _ = R.local_W(A, wl.block_sizes, wl.lam, wl.invtt)
    ev = np.linalg.eigvalsh(W)
    return np.repeat(ev[:, 0] > 1e-6 * ev[:, 2], 3)


@pytest.mark.parametrize("case", ["gaps", "cut_gaps"])
@pytest.mark.parametrize("enl,ortho,bs_red", [(1, 1, 0), (4, 1, 0), (8, 1, 1), (16, 1, 1)])
def test_ecg_orthomin(gpu_ctx, ref_lib, case, enl, ortho, bs_red):
    wl = solver_cases()[case]()
    x, lst, cond, hits, res, info = _gpu_ecg(gpu_ctx, wl, tol=1e-10, maxiter=800, enl_fac=enl, ortho_alg=ortho,
                                             bs_red=bs_red)
    e = R.ecg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=800,
              enl=enl, ortho_alg=ortho, bs_red=bs_red)
    xr, lstr, condr, hitsr, _ = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam,
                                            wl.invtt, tol=1e-12, maxiter=800)
    assert info.converged
    assert np.array_equal(lst, lstr) and np.array_equal(hits, hitsr)
    if not bs_red:  # with bs_red the directions dropped near the 1e-12 threshold may differ
        assert abs(info.iterations - e.iters) <= 1, (info.iterations, e.iters)
    k = min(6, len(res), len(e.res_rel))
    assert np.allclose(res[:k], e.res_rel[:k], rtol=1e-6)
    det = _determined(wl, e.bj.A) if case == "cut_gaps" else np.ones(len(xr), dtype=bool)
    for s in range(3):
        sel = det[s::3]
        assert _rel(x[s::3][sel], xr[s::3][sel]) < 1e-8, (s, _rel(x[s::3][sel], xr[s::3][sel]))


def test_ecg_orthodir_follows_restatement(gpu_ctx):
    """Orthodir's three-term block recurrence: same residual history as the
    restatement over its first iterations and the same (loose) convergence."""
    wl = solver_cases()["gaps"]()
    x, lst, cond, hits, res, info = _gpu_ecg(gpu_ctx, wl, tol=1e-4, maxiter=200, enl_fac=4, ortho_alg=0, bs_red=0)
    e = R.ecg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-4, maxiter=200,
              enl=4, ortho_alg=0, bs_red=0)
    assert info.converged and abs(info.iterations - e.iters) <= 1
    k = min(6, len(res))
    assert np.allclose(res[:k], e.res_rel[:k], rtol=1e-6)
    assert _rel(x, e.x) < 1e-3


def test_ecg_rejects_enlargement(gpu_ctx):
    import midapack_b200 as mb
    wl = solver_cases()["gaps"]()
    for enl in (0, 65):
        with pytest.raises(mb.MidapackError):
            _gpu_ecg(gpu_ctx, wl, enl_fac=enl)


def test_ecg_gls_host_entry_and_mlmap(gpu_ctx, ref_lib):
    """ECG_GLS through host pointers (cut mirrored on the host Mat and b, the
    rel_res file), and MLmap with solver 1 writing its FITS maps."""
    import midapack_b200 as mb
    from midapack_b200 import mappraiser_wrapper as mw
    from midapack_b200.mappraiser_wrapper import Mat
    from tests.test_gpu_dropin import _tpltz
    L = mb.lib()
    wl = solver_cases()["cut_gaps"]()
    m = wl.n_samples
    idx, vals, sig = wl.pix.copy(), wl.weights.copy(), wl.signal.copy()
    A = Mat()
    L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(vals, ct.c_double), 6, 0x44000000)
    invtt = wl.invtt.copy()
    T, blocks, bs = _tpltz(wl.block_sizes, wl.lam, invtt)
    n0 = A.lcount - 3 * A.trash_pix
    x = np.zeros(n0)
    cond = np.zeros(n0 // 3)
    hits = np.zeros(n0 // 3, dtype=np.int32)
    with tempfile.TemporaryDirectory() as td:
        rc = L.ECG_GLS(td.encode(), b"t", ct.byref(A), ct.byref(T), _p(x, ct.c_double), _p(sig, ct.c_double),
                       _p(wl.noise, ct.c_double), _p(cond, ct.c_double), _p(hits, ct.c_int32), 1e-10, 800, 4, 1, 0)
        assert rc == 0
        rel = np.loadtxt(os.path.join(td, "rel_res_t_enlfac_4_o=1.txt"))
    e = R.ecg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=800,
              enl=4, ortho_alg=1)
    n = A.lcount - 3 * A.trash_pix
    assert n == len(e.x)
    assert abs(len(rel) - len(e.res_rel)) <= 1 and rel[-1] < 1e-10
    det = _determined(wl, e.bj.A)
    assert _rel(x[:n][det], e.x[det]) < 1e-8
    assert np.count_nonzero(sig == 0) >= 1  # the cut zeroes b on the rewritten samples
    wl2 = solver_cases()["gaps"]()
    xr, lst, condr, hitsr, _ = ref_lib.pcg(wl2.pix, wl2.weights, wl2.signal, wl2.noise, wl2.block_sizes, wl2.lam,
                                           wl2.invtt, tol=1e-12, maxiter=800)
    refmaps = R.x2map_pol(xr, lst, condr, hitsr, 12 * wl2.nside ** 2)
    with tempfile.TemporaryDirectory() as td:
        params = dict(path_output=td, ref="run", solver=1, precond=0, Z_2lvl=0, ptcomm_flag=6, tol=1e-10,
                      maxiter=800, enlFac=4, ortho_alg=1, bs_red=0, nside=wl2.nside, Lambda=wl2.lam)
        mw.MLmap(None, params, np.array([wl2.n_samples], dtype=np.int32), len(wl2.block_sizes), wl2.block_sizes, 3,
                 wl2.pix, wl2.weights, wl2.signal, wl2.noise, wl2.invtt)
        maps = [mw.read_fits_map(os.path.join(td, f"{k}_run.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    for k in range(3):
        assert np.linalg.norm(maps[k] - refmaps[k]) <= 1e-8 * np.linalg.norm(refmaps[k])
    assert np.array_equal(maps[4], refmaps[4])
