"""The reference-compatible C API (host pointers) of libmidapack_b200, called
through ctypes exactly as a MAPPRAISER caller would, vs the reference's own
compiled operators (oracle/_ref)."""
import ctypes as ct
import os
import tempfile

import numpy as np
import pytest

from midapack_b200 import synth
from tests._cases import solver_cases

pytestmark = pytest.mark.gpu


def _p(a, t):
    return a.ctypes.data_as(ct.POINTER(t))


def test_matinit_matvec_trmatvec(gpu_ctx, ref_lib):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Mat
    L = mb.lib()
    wl = synth.small(n_det=2, n_samp=4096, block_len=2048, lam=32, gap_frac=0.03, seed=31)
    m = wl.n_samples
    idx = wl.pix.copy()
    vals = wl.weights.copy()
    A = Mat()
    A.trash_pix = 0
    assert L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(vals, ct.c_double), 6, 0x44000000) == 0
    loc_r, lind_r, trash_r = ref_lib.local_shape(wl.pix, m, 3)
    assert A.lcount == len(lind_r) and A.trash_pix == trash_r
    assert np.array_equal(idx, loc_r)  # in-place rewrite to local indices
    assert np.array_equal(np.ctypeslib.as_array(A.lindices, shape=(A.lcount,)), lind_r)
    n = A.lcount - 3 * A.trash_pix
    rng = np.random.default_rng(0)
    x = rng.standard_normal(n)
    y = np.zeros(m)
    assert L.MatVecProd(ct.byref(A), _p(x, ct.c_double), _p(y, ct.c_double), 0) == 0
    yr = ref_lib.matvec(wl.pix, wl.weights, x, m)
    assert np.linalg.norm(y - yr) <= 1e-13 * np.linalg.norm(yr)
    t = rng.standard_normal(m)
    xo = np.zeros(n)
    assert L.TrMatVecProd(ct.byref(A), _p(t, ct.c_double), _p(xo, ct.c_double), 0) == 0
    xr = ref_lib.trmatvec(wl.pix, wl.weights, t, m, n)
    assert np.linalg.norm(xo - xr) <= 1e-13 * np.linalg.norm(xr)
    L.MatFree(ct.byref(A))


def _tpltz(block_sizes, lam, invtt):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Block, Flag, Tpltz
    L = mb.lib()
    nb = len(block_sizes)
    blocks = (Block * nb)()
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32)
    L.defineBlocks_avg(blocks, _p(invtt, ct.c_double), nb, bs.ctypes.data_as(ct.c_void_p), lam, 0)
    T = Tpltz()
    f = Flag()
    L.flag_stgy_init_auto(ct.byref(f))
    L.defineTpltz_avg.argtypes = [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int,
                                  ct.c_int64, ct.c_int, Flag, ct.c_int]
    L.defineTpltz_avg(ct.byref(T), int(bs.sum()), 1, 1, blocks, nb, nb, 0, int(bs.sum()), f, 0x44000000)
    return T, blocks, bs


def test_stbmmprod(gpu_ctx, ref_lib):
    import midapack_b200 as mb
    L = mb.lib()
    wl = synth.small(n_det=2, n_samp=8192, block_len=4096, lam=256, seed=33)
    invtt = wl.invtt.copy()
    T, blocks, bs = _tpltz(wl.block_sizes, wl.lam, invtt)
    v = np.random.default_rng(1).standard_normal(wl.n_samples)
    out = v.copy()
    assert L.stbmmProd(ct.byref(T), _p(out, ct.c_double)) == 0
    ref = ref_lib.stbmm(v, wl.block_sizes, wl.lam, wl.invtt)
    assert np.linalg.norm(out - ref) <= 1e-12 * np.linalg.norm(ref)


def test_pcg_gls_true(gpu_ctx, ref_lib):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Mat
    L = mb.lib()
    wl = solver_cases()["cut"]()
    m = wl.n_samples
    idx = wl.pix.copy()
    vals = wl.weights.copy()
    sig = wl.signal.copy()
    A = Mat()
    L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(vals, ct.c_double), 6, 0x44000000)
    invtt = wl.invtt.copy()
    T, blocks, bs = _tpltz(wl.block_sizes, wl.lam, invtt)
    n0 = A.lcount - 3 * A.trash_pix
    x = np.zeros(n0)
    cond = np.zeros(n0 // 3)
    hits = np.zeros(n0 // 3, dtype=np.int32)
    with tempfile.TemporaryDirectory() as td:
        rc = L.PCG_GLS_true(td.encode(), b"t", ct.byref(A), ct.byref(T), _p(x, ct.c_double), _p(sig, ct.c_double),
                            _p(wl.noise, ct.c_double), _p(cond, ct.c_double), _p(hits, ct.c_int32), 1e-10, 400, 0, 0)
        assert rc == 0
        res = np.fromfile(os.path.join(td, "pcg_residuals_t.dat"))
    xr, lstr, condr, hitsr, resr = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam,
                                               wl.invtt, tol=1e-10, maxiter=400)
    n = A.lcount - 3 * A.trash_pix
    assert n == len(xr)
    lst = np.ctypeslib.as_array(A.lindices, shape=(A.lcount,))[3 * A.trash_pix:]
    assert np.array_equal(lst, lstr)
    assert np.array_equal(hits[:n // 3], hitsr)
    assert np.linalg.norm(x[:n] - xr) <= 1e-10 * np.linalg.norm(xr)
    assert abs(len(res) - len(resr)) <= 1
    # the cut zeroes b on the rewritten samples, as the reference does
    assert np.count_nonzero(sig == 0) >= 1


def test_mlmap_writes_fits_maps(gpu_ctx, ref_lib):
    from midapack_b200 import mappraiser_wrapper as mw
    wl = solver_cases()["gaps"]()
    with tempfile.TemporaryDirectory() as td:
        params = dict(path_output=td, ref="run", solver=0, precond=0, Z_2lvl=0, ptcomm_flag=6, tol=1e-10,
                      maxiter=400, enlFac=1, ortho_alg=1, bs_red=0, nside=wl.nside, Lambda=wl.lam)
        mw.MLmap(None, params, np.array([wl.n_samples], dtype=np.int32), len(wl.block_sizes), wl.block_sizes, 3,
                 wl.pix, wl.weights, wl.signal, wl.noise, wl.invtt)
        maps = [mw.read_fits_map(os.path.join(td, f"{k}_run.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    ref = ref_lib.mlmap(1, [wl.n_samples], [len(wl.block_sizes)], wl.block_sizes, wl.pix, wl.weights, wl.signal,
                        wl.noise, wl.lam, wl.invtt, wl.nside, tol=1e-10, maxiter=400)
    for k in range(3):
        assert np.linalg.norm(maps[k] - ref[k]) <= 1e-10 * np.linalg.norm(ref[k])
    assert np.array_equal(maps[4], ref[4])
    assert np.allclose(maps[3], ref[3], rtol=1e-12, atol=0)
