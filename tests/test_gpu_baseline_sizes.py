"""Parity at the sizes of the benchmark workloads, through the reference-facing
C API (host arrays), against the reference's own compiled code (oracle/_ref).

* The CPU-runnable workload (4 detectors x 2^20 samples, 256x192 grid,
  lambda 2^12, one Toeplitz block per detector) with 1% flagged samples: the
  drop-in MLmap on the GPU against the reference's MLmap on 4 forked ranks
  (mappraiser.c:34-385), both to the workload's relative residual 1e-8.  Hits
  and the set of solved pixels bit-exact, Cond within 1e-12, I/Q/U within
  1e-10 on the observed pixels, same iteration count within one.
* A chunk of the at-scale workload (2 of its 64 detectors x 2^24 samples,
  2048x1536 grid, 2^20-sample blocks, lambda 2^14, 1% flagged samples):
  MatVecProd, stbmmProd and TrMatVecProd (mapmat.c:704-729, 819-859,
  toeplitz_wizard.c:80-111) against the reference's operators on the same
  inputs, 1e-12 per matvec; stbmmProd also against the exact long-double banded
  product on sampled rows (the reference's own FFT product carries the
  aliasing error of scmm_direct, toeplitz.c:585-589).

The reference's MLmap forks its ranks, so it runs in a fresh interpreter
(oracle.cpu_baseline) that never initialised CUDA.
"""
import ctypes as ct
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from midapack_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _p(a, t):
    return a.ctypes.data_as(ct.POINTER(t))


def test_c1_mlmap_matches_reference_on_4_ranks(gpu_ctx, ref_lib, tmp_path):
    from midapack_b200 import mappraiser_wrapper as mw
    cfg = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"], gap_frac=0.01)
    wl = synth.make_workload("c1", **cfg)
    tol, maxiter = 1e-8, 2000
    case, out = str(tmp_path / "case.npz"), str(tmp_path / "maps.npz")
    np.savez(case, pix=wl.pix, weights=wl.weights, signal=wl.signal, noise=wl.noise, block_sizes=wl.block_sizes,
             lam=wl.lam, invtt=wl.invtt, nside=wl.nside, tol=tol, maxiter=maxiter)
    r = subprocess.run([sys.executable, "-m", "oracle.cpu_baseline", "--mlmap", case, "4", out], cwd=ROOT,
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    rj = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    ref = np.load(out)
    gdir = tmp_path / "gpu"
    gdir.mkdir()
    params = dict(path_output=str(gdir), ref="c1", solver=0, precond=0, Z_2lvl=0, ptcomm_flag=6, tol=tol,
                  maxiter=maxiter, enlFac=1, ortho_alg=1, bs_red=0, nside=wl.nside, Lambda=wl.lam)
    mw.MLmap(None, params, np.array([wl.n_samples], dtype=np.int32), len(wl.block_sizes), wl.block_sizes, 3,
             wl.pix.copy(), wl.weights.copy(), wl.signal.copy(), wl.noise.copy(), wl.invtt.copy())
    mine = [mw.read_fits_map(str(gdir / f"{k}_c1.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    res = np.fromfile(str(gdir / "pcg_residuals_c1.dat"))
    assert abs((len(res) - 1) - rj["iterations"]) <= 1
    np.testing.assert_array_equal(mine[4], ref["Hits"])
    solved_ref = ref["Cond"] != 0
    np.testing.assert_array_equal(mine[3] != 0, solved_ref)
    np.testing.assert_allclose(mine[3][solved_ref], ref["Cond"][solved_ref], rtol=1e-12, atol=0)
    obs = ref["Hits"] > 0
    for k, name in enumerate("IQU"):
        d = np.linalg.norm(mine[k][obs] - ref[name][obs]) / np.linalg.norm(ref[name][obs])
        assert d <= 1e-10, f"{name}: {d:.3e}"


def _exact_rows(v, start, n, lam, T, rows):
    """Reference product on chosen rows of one block: mean removal
    (toeplitz_wizard.c:85-95) then the banded symmetric Toeplitz sum, in long double."""
    blk = v[start:start + n].astype(np.longdouble)
    blk = blk - blk.sum() / n
    t = T.astype(np.longdouble)
    out = []
    for r in rows:
        lo, hi = max(0, r - lam + 1), min(n, r + lam)
        j = np.arange(lo, hi)
        out.append(np.dot(t[np.abs(j - r)], blk[lo:hi]))
    return np.array(out, dtype=np.longdouble)


def test_c2_chunk_operators_match_reference(gpu_ctx, ref_lib):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Block, Flag, Mat, Tpltz
    L = mb.lib()
    cfg = dict(synth.CONFIGS["c2_64det_2p24_2048x1536_lam16384"], n_det=2)
    pix, w, bs, invtt = synth.make_pointing(**cfg)
    m, lam = pix.size // 3, cfg["lam"]
    rng = np.random.default_rng(20261215)

    # index compression and P / P^T through the drop-in Mat
    idx = pix.copy()
    A = Mat()
    A.trash_pix = 0
    assert L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(w, ct.c_double), 6, 0x44000000) == 0
    loc_r, lind_r, trash_r = ref_lib.local_shape(pix, m, 3)
    assert A.lcount == len(lind_r) and A.trash_pix == trash_r
    np.testing.assert_array_equal(np.ctypeslib.as_array(A.lindices, shape=(A.lcount,)), lind_r)
    np.testing.assert_array_equal(idx, loc_r)
    n = A.lcount - 3 * A.trash_pix
    x = rng.standard_normal(n)
    y = np.zeros(m)
    assert L.MatVecProd(ct.byref(A), _p(x, ct.c_double), _p(y, ct.c_double), 0) == 0
    yr = ref_lib.matvec(pix, w, x, m)
    assert np.linalg.norm(y - yr) <= 1e-12 * np.linalg.norm(yr)

    # stbmmProd on the TOD P x (in place, block means removed)
    nb = len(bs)
    blocks = (Block * nb)()
    tt = np.ascontiguousarray(invtt)
    bsa = np.ascontiguousarray(bs, dtype=np.int32)
    L.defineBlocks_avg(blocks, _p(tt, ct.c_double), nb, bsa.ctypes.data_as(ct.c_void_p), lam, 0)
    T = Tpltz()
    f = Flag()
    L.flag_stgy_init_auto(ct.byref(f))
    L.defineTpltz_avg.argtypes = [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int,
                                  ct.c_int64, ct.c_int, Flag, ct.c_int]
    L.defineTpltz_avg(ct.byref(T), m, 1, 1, blocks, nb, nb, 0, m, f, 0x44000000)
    v = y.copy()
    assert L.stbmmProd(ct.byref(T), _p(v, ct.c_double)) == 0
    vr = ref_lib.stbmm(y, bs, lam, invtt)
    # exact product on 64 rows of 4 blocks (first, last, two inside; rows near the edges included)
    gap_gpu = gap_ref = 0.0
    scale = 0.0
    for b in (0, 7, 20, nb - 1):
        s0, nn = b * cfg["block_len"], int(bs[b])
        rows = np.concatenate([[0, 1, lam - 2, lam, nn // 2, nn - lam, nn - 2, nn - 1],
                               rng.integers(0, nn, 56)])
        ex = _exact_rows(y, s0, nn, lam, invtt[b * lam:(b + 1) * lam], rows)
        gap_gpu += float(np.sum((v[s0 + rows] - ex) ** 2))
        gap_ref += float(np.sum((vr[s0 + rows] - ex) ** 2))
        scale += float(np.sum(ex ** 2))
    err_gpu, err_ref = np.sqrt(gap_gpu / scale), np.sqrt(gap_ref / scale)
    assert err_gpu <= 1e-12, f"GPU N^-1 vs exact product: {err_gpu:.3e}"
    d = np.linalg.norm(v - vr) / np.linalg.norm(vr)
    assert d <= max(1e-12, 4 * err_ref), f"GPU vs reference stbmmProd: {d:.3e} (reference vs exact {err_ref:.3e})"

    # P^T on the weighted TOD
    xo = np.zeros(n)
    assert L.TrMatVecProd(ct.byref(A), _p(vr, ct.c_double), _p(xo, ct.c_double), 0) == 0
    xr = ref_lib.trmatvec(pix, w, vr, m, n)
    assert np.linalg.norm(xo - xr) <= 1e-12 * np.linalg.norm(xr)
    L.MatFree(ct.byref(A))
