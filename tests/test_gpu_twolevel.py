"""Two-level preconditioners (precond 1: a priori build_Z columns; precond 2:
a posteriori Lanczos Ritz vectors) on the GPU vs the reference's own C code
(oracle/_ref, its LAPACK calls restated in the shim) and the numpy
restatement: same pixels, iteration count +-1, residual history to 1e-6,
maps within 1e-10 relative per I/Q/U.  Also the reference-compatible host
entry points (build_precond / apply_precond / PCG_GLS_true / MLmap)."""
import ctypes as ct
import os
import tempfile

import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R
from tests._cases import solver_cases

pytestmark = pytest.mark.gpu
MAP_TOL = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _p(a, t):
    return a.ctypes.data_as(ct.POINTER(t))


def _gpu_solve(ctx, wl, tol, maxiter, precond, zn):
    import torch
    import midapack_b200 as mb
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = mb.Pointing(ctx, d(wl.pix), d(wl.weights), wl.n_samples, 3)
    N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    x, lst, cond, hits, res, info = mb.gls_solve(ctx, P, N, d(wl.signal), d(wl.noise), tol=tol, maxiter=maxiter,
                                                 precond=precond, z_2lvl=zn)
    return x.cpu().numpy(), lst.cpu().numpy(), cond.cpu().numpy(), hits.cpu().numpy(), res, info


@pytest.mark.parametrize("case", ["gaps", "cut_gaps"])
@pytest.mark.parametrize("precond,zn", [(1, 0), (1, 4), (1, 6), (2, 0), (2, 4), (2, 8)])
def test_two_level_vs_reference(gpu_ctx, ref_lib, case, precond, zn):
    wl = solver_cases()[case]()
    x, lst, cond, hits, res, info = _gpu_solve(gpu_ctx, wl, 1e-10, 400, precond, zn)
    xr, lstr, condr, hitsr, resr = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam,
                                               wl.invtt, tol=1e-10, maxiter=400, precond=precond, z_2lvl=zn)
    assert info.converged
    assert np.array_equal(lst, lstr)
    assert np.array_equal(hits, hitsr)
    assert abs(info.iterations - (len(resr) - 1)) <= 1, (info.iterations, len(resr) - 1)
    k = min(len(res), len(resr), 10)
    assert np.allclose(res[:k], resr[:k], rtol=1e-6)
    for s in range(3):
        assert _rel(x[s::3], xr[s::3]) < MAP_TOL, (s, _rel(x[s::3], xr[s::3]))


@pytest.mark.parametrize("precond,zn", [(1, 16), (2, 24)])
def test_two_level_many_columns_vs_restatement(gpu_ctx, precond, zn):
    """More columns on a larger case (the Gram matrix over several entry tiles,
    Ritz combinations of 24 Lanczos vectors)."""
    wl = synth.small(n_det=4, n_samp=16384, block_len=4096, lam=128, gap_frac=0.01, seed=61)
    x, lst, cond, hits, res, info = _gpu_solve(gpu_ctx, wl, 1e-10, 500, precond, zn)
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=500,
              precond=precond, z_2lvl=zn)
    assert info.converged
    assert np.array_equal(lst, o.bj.A.lindices[3 * o.bj.A.trash_pix:])
    assert abs(info.iterations - o.iters) <= 1, (info.iterations, o.iters)
    for s in range(3):
        assert _rel(x[s::3], o.x[s::3]) < MAP_TOL


def test_two_level_rejected_arguments(gpu_ctx):
    import torch
    import midapack_b200 as mb
    wl = solver_cases()["gaps"]()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), wl.n_samples, 3)
    N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
    with pytest.raises(mb.MidapackError):
        mb.gls_solve(gpu_ctx, P, N, d(wl.signal), d(wl.noise), precond=2, z_2lvl=129)
    with pytest.raises(mb.MidapackError):
        mb.gls_solve(gpu_ctx, P, N, d(wl.signal), d(wl.noise), precond=3)


_PRECOND = []


def _precond_struct():
    """The reference's Precond (precond.h:6-22) as a ctypes structure."""
    if not _PRECOND:
        from midapack_b200.mappraiser_wrapper import Mat

        class Precond(ct.Structure):
            _fields_ = [("precond", ct.c_int), ("n", ct.c_int), ("Zn", ct.c_int), ("BJ_inv", Mat), ("BJ", Mat),
                        ("pixpond", ct.POINTER(ct.c_double)), ("Z", ct.POINTER(ct.POINTER(ct.c_double))),
                        ("AZ", ct.POINTER(ct.POINTER(ct.c_double))), ("Em1", ct.POINTER(ct.c_double)),
                        ("Qg", ct.POINTER(ct.c_double)), ("AQg", ct.POINTER(ct.c_double)),
                        ("Qtx", ct.POINTER(ct.c_double)), ("w", ct.POINTER(ct.c_double))]
        _PRECOND.append(Precond)
    return _PRECOND[0]


def _tp(block_sizes, lam, invtt):
    from tests.test_gpu_dropin import _tpltz
    return _tpltz(block_sizes, lam, invtt)


@pytest.mark.parametrize("precond,zn", [(1, 4), (2, 6)])
def test_build_and_apply_precond_host_api(gpu_ctx, precond, zn):
    """build_precond fills the reference's Precond fields (Z, AZ, Em1 with the
    Zn columns) and apply_precond on host arrays equals the restatement's
    two-level product."""
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Mat
    Pc = _precond_struct()
    L = mb.lib()
    wl = solver_cases()["cut_gaps"]()
    m = wl.n_samples
    idx, vals, sig = wl.pix.copy(), wl.weights.copy(), wl.signal.copy()
    A = Mat()
    L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(vals, ct.c_double), 6, 0x44000000)
    invtt = wl.invtt.copy()
    T, blocks, bs = _tp(wl.block_sizes, wl.lam, invtt)
    n0 = A.lcount - 3 * A.trash_pix
    x = np.zeros(n0)
    cond = np.zeros(n0 // 3)
    hits = np.zeros(n0 // 3, dtype=np.int32)
    pp = ct.POINTER(Pc)()
    pixpond = ct.POINTER(ct.c_double)()
    n = ct.c_int()
    xp = ct.cast(x.ctypes.data, ct.POINTER(ct.c_double))
    L.build_precond.argtypes = [ct.POINTER(ct.POINTER(Pc)), ct.POINTER(ct.POINTER(ct.c_double)),
                                ct.POINTER(ct.c_int), ct.c_void_p, ct.c_void_p,
                                ct.POINTER(ct.POINTER(ct.c_double)), ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                ct.c_void_p, ct.c_double, ct.c_int, ct.c_int]
    L.build_precond(ct.byref(pp), ct.byref(pixpond), ct.byref(n), ct.byref(A), ct.byref(T), ct.byref(xp),
                    sig.ctypes.data, wl.noise.ctypes.data, cond.ctypes.data, hits.ctypes.data, 1e-10, zn, precond)
    assert bool(pp)
    p = pp.contents
    assert p.precond == precond and p.Zn == zn and p.n == n.value
    nn = n.value
    # the restatement on the same (cut) system
    o = R.precond_blockjacobi(R.local_shape(wl.pix, wl.weights, m, 3), wl.signal, wl.block_sizes, wl.lam, wl.invtt)
    Ao = o.A
    assert Ao.n == nn
    op = lambda v: R.trmatvec(Ao, R.stbmm(R.matvec(Ao, v), wl.block_sizes, wl.lam, wl.invtt))  # noqa: E731
    if precond == 1:
        Z = R.build_Z(Ao, zn)
        AZ = R.build_AZ(op, Z)
    else:
        g0 = R.trmatvec(Ao, R.stbmm(o.signal + wl.noise, wl.block_sizes, wl.lam, wl.invtt))
        Z, AZ = R.lanczos_eig(op, g0, zn)
    tl = R.TwoLevel(Z, AZ, R.build_Em1(Z, AZ))
    Zh = np.stack([np.ctypeslib.as_array(p.Z[j], shape=(nn,)) for j in range(zn)])
    AZh = np.stack([np.ctypeslib.as_array(p.AZ[j], shape=(nn,)) for j in range(zn)])
    if precond == 1:
        assert np.array_equal(Zh, Z)  # integer counts over the same rows
        assert _rel(AZh, AZ) < 1e-11
    g = np.random.default_rng(5).standard_normal(nn)
    Cg = np.zeros(nn)
    L.apply_precond.argtypes = [ct.POINTER(Pc), ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.apply_precond(pp, ct.byref(A), ct.byref(T), g.ctypes.data, Cg.ctypes.data)
    ref = R.apply_2lvl(tl, o.inv, g)
    assert _rel(Cg, ref) < 1e-8
    L.free_precond.argtypes = [ct.POINTER(ct.POINTER(Pc))]
    L.free_precond(ct.byref(pp))
    assert not bool(pp)


def test_pcg_gls_true_and_mlmap_two_level(gpu_ctx, ref_lib):
    """PCG_GLS_true(precond = 2, Z_2lvl = 4) through host pointers, and MLmap
    with the same preconditioner writing its FITS maps, vs the reference's
    PCG with that preconditioner."""
    import midapack_b200 as mb
    from midapack_b200 import mappraiser_wrapper as mw
    from midapack_b200.mappraiser_wrapper import Mat
    L = mb.lib()
    wl = solver_cases()["cut_gaps"]()
    m = wl.n_samples
    idx, vals, sig = wl.pix.copy(), wl.weights.copy(), wl.signal.copy()
    A = Mat()
    L.MatInit(ct.byref(A), m, 3, _p(idx, ct.c_int32), _p(vals, ct.c_double), 6, 0x44000000)
    invtt = wl.invtt.copy()
    T, blocks, bs = _tp(wl.block_sizes, wl.lam, invtt)
    n0 = A.lcount - 3 * A.trash_pix
    x = np.zeros(n0)
    cond = np.zeros(n0 // 3)
    hits = np.zeros(n0 // 3, dtype=np.int32)
    xr, lstr, condr, hitsr, resr = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam,
                                               wl.invtt, tol=1e-10, maxiter=400, precond=2, z_2lvl=4)
    with tempfile.TemporaryDirectory() as td:
        rc = L.PCG_GLS_true(td.encode(), b"t", ct.byref(A), ct.byref(T), _p(x, ct.c_double), _p(sig, ct.c_double),
                            _p(wl.noise, ct.c_double), _p(cond, ct.c_double), _p(hits, ct.c_int32), 1e-10, 400, 2, 4)
        assert rc == 0
        res = np.fromfile(os.path.join(td, "pcg_residuals_t.dat"))
    n = A.lcount - 3 * A.trash_pix
    assert n == len(xr)
    assert np.linalg.norm(x[:n] - xr) <= MAP_TOL * np.linalg.norm(xr)
    assert abs(len(res) - len(resr)) <= 1
    wl2 = solver_cases()["gaps"]()
    xr2, lst2, cond2, hits2, _ = ref_lib.pcg(wl2.pix, wl2.weights, wl2.signal, wl2.noise, wl2.block_sizes, wl2.lam,
                                            wl2.invtt, tol=1e-10, maxiter=400, precond=2, z_2lvl=3)
    refmaps = R.x2map_pol(xr2, lst2, cond2, hits2, 12 * wl2.nside ** 2)
    with tempfile.TemporaryDirectory() as td:
        params = dict(path_output=td, ref="run", solver=0, precond=2, Z_2lvl=3, ptcomm_flag=6, tol=1e-10,
                      maxiter=400, enlFac=1, ortho_alg=1, bs_red=0, nside=wl2.nside, Lambda=wl2.lam)
        mw.MLmap(None, params, np.array([wl2.n_samples], dtype=np.int32), len(wl2.block_sizes), wl2.block_sizes, 3,
                 wl2.pix, wl2.weights, wl2.signal, wl2.noise, wl2.invtt)
        maps = [mw.read_fits_map(os.path.join(td, f"{k}_run.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    for k in range(3):
        assert np.linalg.norm(maps[k] - refmaps[k]) <= MAP_TOL * np.linalg.norm(refmaps[k])
    assert np.array_equal(maps[4], refmaps[4])


@pytest.mark.parametrize("case", ["gaps", "cut_gaps"])
@pytest.mark.parametrize("precond,zn", [(1, 4), (2, 8)])
def test_two_level_mixed_precision(gpu_ctx, case, precond, zn):
    """The two-level preconditioners inside the mixed-precision solve (columns
    built with the FP64 operator, inner PCGs on the FP32 operator): the map
    equals the FP64 block-Jacobi solve within 1e-8 on the determined pixels
    (both to 1e-12)."""
    import torch
    import midapack_b200 as mb
    wl = solver_cases()[case]()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    outs = []
    for mixed in (False, True):
        P = mb.Pointing(gpu_ctx, d(wl.pix), d(wl.weights), wl.n_samples, 3)
        N = mb.Noise(gpu_ctx, wl.block_sizes, wl.lam, wl.invtt)
        if mixed:
            r = mb.gls_solve_mixed(gpu_ctx, P, N, d(wl.signal), d(wl.noise), tol=1e-12, maxiter=900, precond=precond,
                                   z_2lvl=zn)
        else:
            r = mb.gls_solve(gpu_ctx, P, N, d(wl.signal), d(wl.noise), tol=1e-12, maxiter=900)
        assert r[5].converged
        outs.append((r[0].cpu().numpy(), r[1].cpu().numpy()))
    (x64, l64), (x32, l32) = outs
    assert np.array_equal(l64, l32)
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=400)
    W, _ = R.local_W(o.bj.A, wl.block_sizes, wl.lam, wl.invtt)
    ev = np.linalg.eigvalsh(W)
    det = np.repeat(ev[:, 0] > 1e-6 * ev[:, 2], 3)
    for s in range(3):
        sel = det[s::3]
        assert _rel(x32[s::3][sel], x64[s::3][sel]) < 1e-8, (s, _rel(x32[s::3][sel], x64[s::3][sel]))
