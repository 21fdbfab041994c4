"""Pins the numpy restatement to the reference's own compiled C
(oracle/_ref): compression bit-exact, P and P^T bit-exact (same summation
order), N^-1 within 1e-13, the full PCG within 1e-12, and the rcond cut
(including the reference's behaviour with flagged samples).  Plus the
project LAPACK shim against scipy's LAPACK.  CPU only."""
import ctypes as ct
import os

import numpy as np
import pytest

from midapack_b200 import synth
from oracle import restate as R
from tests._cases import solver_cases


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("case", list(solver_cases()))
def test_operators_bitexact(ref_lib, case):
    wl = solver_cases()[case]()
    m = wl.n_samples
    A = R.local_shape(wl.pix, wl.weights, m, 3)
    loc, lind, trash = ref_lib.local_shape(wl.pix, m, 3)
    assert np.array_equal(A.lindices, lind) and np.array_equal(A.local, loc) and A.trash_pix == trash
    x = np.random.default_rng(0).standard_normal(A.n)
    assert np.array_equal(R.matvec(A, x), ref_lib.matvec(wl.pix, wl.weights, x, m))
    y = np.random.default_rng(1).standard_normal(m)
    assert np.array_equal(R.trmatvec(A, y), ref_lib.trmatvec(wl.pix, wl.weights, y, m, A.n))
    v = np.random.default_rng(2).standard_normal(m)
    assert _rel(R.stbmm(v, wl.block_sizes, wl.lam, wl.invtt, exact=True),
                ref_lib.stbmm(v, wl.block_sizes, wl.lam, wl.invtt)) < 1e-13


@pytest.mark.parametrize("case", list(solver_cases()))
def test_pcg_and_cut(ref_lib, case):
    wl = solver_cases()[case]()
    maxiter = 12 if case == "plain" else 400  # gap-free: singular operator, compare fixed iterates
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=maxiter)
    xr, lst, cond, hits, res = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt,
                                           tol=1e-10, maxiter=maxiter)
    assert np.array_equal(o.bj.A.lindices[3 * o.bj.A.trash_pix:], lst)
    # entries past the kept blocks are stale memory in the reference (see restate.precond_blockjacobi)
    kb = int((~o.bj.cut).sum())
    assert np.array_equal(o.bj.hits[:kb], hits[:kb])
    assert np.allclose(o.bj.cond[:kb], cond[:kb], rtol=1e-13, atol=0)
    assert min(o.iters, maxiter - 1) == len(res) - 1
    assert _rel(o.x, xr) < 1e-12


def test_mlmap_multirank_matches_single(ref_lib):
    """The fork/shared-memory MPI stand-in: 4-rank MLmap == 1-rank MLmap."""
    wl = synth.small(n_det=4, n_samp=2048, block_len=1024, lam=32, seed=51, gap_frac=0.02)
    args = (wl.block_sizes, wl.pix, wl.weights, wl.signal, wl.noise, wl.lam, wl.invtt, wl.nside)
    one = ref_lib.mlmap(1, [wl.n_samples], [len(wl.block_sizes)], *args, tol=1e-10, maxiter=300)
    per = wl.n_samples // 4
    four = ref_lib.mlmap(4, [per] * 4, [len(wl.block_sizes) // 4] * 4, *args, tol=1e-10, maxiter=300)
    for k in range(3):
        assert _rel(four[k], one[k]) < 1e-10
    assert np.array_equal(four[4], one[4])


def test_shim_lapack_vs_scipy(ref_lib):
    from scipy.linalg import lapack
    L = ct.CDLL(os.path.join(os.path.dirname(ref_lib.LIB_PATH), "libmidapack_ref_shims.so"))
    L.LAPACKE_dgetrf.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.POINTER(ct.c_double), ct.c_int,
                                 ct.POINTER(ct.c_int)]
    L.LAPACKE_dgecon.argtypes = [ct.c_int, ct.c_char, ct.c_int, ct.POINTER(ct.c_double), ct.c_int, ct.c_double,
                                 ct.POINTER(ct.c_double)]
    L.LAPACKE_dgetri.argtypes = [ct.c_int, ct.c_int, ct.POINTER(ct.c_double), ct.c_int, ct.POINTER(ct.c_int)]
    rng = np.random.default_rng(3)
    for trial in range(300):
        w = rng.standard_normal((rng.integers(1, 40), 3))
        w[:, 0] = 1.0
        a = (w[:, :, None] * w[:, None, :]).sum(0) * rng.uniform(0.5, 2e7)
        if trial % 7 == 0:
            a = np.outer(w[0], w[0])  # rank one
        anorm = np.abs(a).sum(axis=0).max()
        m = np.ascontiguousarray(a.copy())
        ipiv = np.zeros(3, dtype=np.int32)
        L.LAPACKE_dgetrf(101, 3, 3, m.ctypes.data_as(ct.POINTER(ct.c_double)), 3,
                         ipiv.ctypes.data_as(ct.POINTER(ct.c_int)))
        rc = ct.c_double()
        L.LAPACKE_dgecon(101, b"1", 3, m.ctypes.data_as(ct.POINTER(ct.c_double)), 3, anorm, ct.byref(rc))
        lu, piv, _ = lapack.dgetrf(np.asfortranarray(a))
        rs, _ = lapack.dgecon(lu, anorm, norm="1")
        assert np.array_equal(ipiv - 1, piv)
        assert np.allclose(m, lu, rtol=1e-13, atol=1e-13 * np.abs(a).max())
        assert (rc.value > 0.1) == (rs > 0.1)
        if rs > 1e-8:
            assert abs(rc.value - rs) <= 1e-12 * rs
        if rs > 0.1:
            L.LAPACKE_dgetri(101, 3, m.ctypes.data_as(ct.POINTER(ct.c_double)), 3,
                             ipiv.ctypes.data_as(ct.POINTER(ct.c_int)))
            inv, _ = lapack.dgetri(lu, piv)
            assert np.allclose(m, inv, rtol=1e-12, atol=1e-12 * np.abs(inv).max())


def test_shim_dsyev_dgelss_vs_numpy(ref_lib):
    """The shim's Jacobi dsyev / dgelss (two-level preconditioners) against
    numpy's LAPACK: eigenvalues, eigenvectors up to sign, pseudo-inverse with
    the rcond cut, rank."""
    L = ct.CDLL(os.path.join(os.path.dirname(ref_lib.LIB_PATH), "libmidapack_ref_shims.so"))
    dp = ct.POINTER(ct.c_double)
    L.LAPACKE_dsyev.argtypes = [ct.c_int, ct.c_char, ct.c_char, ct.c_int, dp, ct.c_int, dp]
    L.LAPACKE_dgelss.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_int, dp, ct.c_int, dp, ct.c_int, dp, ct.c_double,
                                 ct.POINTER(ct.c_int)]
    rng = np.random.default_rng(11)
    for n in (1, 2, 5, 16, 40):
        off = rng.standard_normal(n - 1)
        t = np.diag(rng.uniform(1, 10, n)) + np.diag(off, 1) + np.diag(off, -1)  # a Lanczos-like tridiagonal matrix
        a = np.ascontiguousarray(t.copy())
        w = np.zeros(n)
        assert L.LAPACKE_dsyev(101, b"V", b"U", n, a.ctypes.data_as(dp), n, w.ctypes.data_as(dp)) == 0
        ev, ey = np.linalg.eigh(t)
        assert np.allclose(w, ev, rtol=1e-12, atol=1e-12 * np.abs(ev).max())
        assert np.allclose(np.abs(a.T @ ey), np.eye(n), atol=1e-10)  # same eigenvectors up to sign
        # dgelss(E, I): full rank and rank deficient (one exact null direction)
        for deficient in (False, True):
            z = rng.standard_normal((n, n + 3))
            e = z @ z.T
            if deficient and n > 1:
                v = rng.standard_normal(n)
                e = e - np.outer(e @ v, e @ v) / (v @ e @ v)  # e v = 0
            ea = np.ascontiguousarray(e.copy())
            b = np.ascontiguousarray(np.eye(n))
            s = np.zeros(n)
            rank = ct.c_int()
            assert L.LAPACKE_dgelss(101, n, n, n, ea.ctypes.data_as(dp), n, b.ctypes.data_as(dp), n,
                                    s.ctypes.data_as(dp), 1e-10, ct.byref(rank)) == 0
            sv = np.linalg.svd(e, compute_uv=False)
            assert np.allclose(s, sv, rtol=1e-10, atol=1e-10 * sv[0])
            assert rank.value == int((sv > 1e-10 * sv[0]).sum())
            assert np.allclose(b, np.linalg.pinv(e, rcond=1e-10), rtol=1e-8, atol=1e-8 * np.abs(b).max())


@pytest.mark.parametrize("case", ["gaps", "cut_gaps"])
@pytest.mark.parametrize("precond,zn", [(1, 0), (1, 4), (1, 6), (2, 0), (2, 4), (2, 8)])
def test_pcg_two_level(ref_lib, case, precond, zn):
    """The two-level preconditioners: build_Z (with the reference's column
    index), build_AZ, the dgelss pseudo-inverse of E, Lanczos_eig (with its
    first three-term update), apply_precond; same iterations and residual
    history as the compiled reference, maps within 1e-11."""
    wl = solver_cases()[case]()
    o = R.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=400,
              precond=precond, z_2lvl=zn)
    xr, lst, cond, hits, res = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt,
                                           tol=1e-10, maxiter=400, precond=precond, z_2lvl=zn)
    assert np.array_equal(o.bj.A.lindices[3 * o.bj.A.trash_pix:], lst)
    assert o.iters == len(res) - 1
    k = min(8, len(res))
    assert np.allclose(o.res_rel[:k], res[:k], rtol=1e-8, atol=0)
    assert _rel(o.x, xr) < 1e-11


@pytest.mark.parametrize("case", ["gaps", "cut_gaps"])
@pytest.mark.parametrize("enl,ortho,bs_red", [(1, 1, 0), (4, 1, 0), (8, 1, 1), (16, 1, 1)])
def test_ecg_restatement_solves_the_reference_system(ref_lib, case, enl, ortho, bs_red):
    """ECG's iteration comes from preAlps, which the reference does not ship:
    the restated enlarged CG is pinned through the solution, which is unique
    on the determined pixels -- it must equal the compiled reference's PCG
    map (tol 1e-12) within 1e-8, with the same pixels."""
    wl = solver_cases()[case]()
    e = R.ecg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, tol=1e-10, maxiter=800,
              enl=enl, ortho_alg=ortho, bs_red=bs_red)
    xr, lst, cond, hits, res = ref_lib.pcg(wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam,
                                           wl.invtt, tol=1e-12, maxiter=800)
    assert e.res_rel[-1] < 1e-10
    assert np.array_equal(e.bj.A.lindices[3 * e.bj.A.trash_pix:], lst)
    det = np.ones(len(xr), dtype=bool)
    if case == "cut_gaps":  # the rewritten pixel of the cut is an exact null direction
        W, _ = R.local_W(e.bj.A, wl.block_sizes, wl.lam, wl.invtt)
        ev = np.linalg.eigvalsh(W)
        det = np.repeat(ev[:, 0] > 1e-6 * ev[:, 2], 3)
    for k in range(3):
        s = det[k::3]
        assert _rel(e.x[k::3][s], xr[k::3][s]) < 1e-8


def test_cpu_baseline_mlmap_mode(ref_lib, tmp_path):
    """bench.py's reference-MLmap leg (python -m oracle.cpu_baseline --mlmap):
    its maps equal the in-process reference MLmap on the same case."""
    import json
    import subprocess
    import sys
    wl = synth.small(n_det=2, n_samp=2048, block_len=1024, lam=32, seed=52, gap_frac=0.02)
    case, out = tmp_path / "case.npz", tmp_path / "maps.npz"
    np.savez(case, pix=wl.pix, weights=wl.weights, signal=wl.signal, noise=wl.noise, block_sizes=wl.block_sizes,
             lam=wl.lam, invtt=wl.invtt, nside=wl.nside, tol=1e-10, maxiter=300)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-m", "oracle.cpu_baseline", "--mlmap", str(case), "2", str(out)], cwd=root,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["ranks"] == 2 and line["iterations"] > 0
    m = np.load(out)
    ref = ref_lib.mlmap(2, [wl.n_samples // 2] * 2, [len(wl.block_sizes) // 2] * 2, wl.block_sizes, wl.pix, wl.weights,
                        wl.signal, wl.noise, wl.lam, wl.invtt, wl.nside, tol=1e-10, maxiter=300)
    for k, name in enumerate(("I", "Q", "U")):
        assert np.array_equal(m[name], ref[k])
