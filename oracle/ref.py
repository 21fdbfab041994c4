"""ctypes access to the reference's own compiled operators (oracle/_ref).

TEST INFRASTRUCTURE ONLY (see oracle/restate.py).  The library is built from
the reference sources by oracle/build_ref.sh; this module never builds it.
"""
from __future__ import annotations

import ctypes as ct
import os
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libmidapack_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (run oracle/build_ref.sh)")
        _lib = ct.CDLL(LIB_PATH)
    return _lib


def _p(a, ctype):
    return a.ctypes.data_as(ct.POINTER(ctype))


I32 = ct.c_int
F64 = ct.c_double


def local_shape(gindices: np.ndarray, m: int, nnz: int):
    idx = np.ascontiguousarray(gindices, dtype=np.int32).copy()
    vals = np.zeros(m * nnz)
    cap = idx.size
    lind = np.zeros(cap, dtype=np.int32)
    trash = ct.c_int(0)
    lc = lib().ref_local_shape(m, nnz, _p(idx, I32), _p(vals, F64), _p(lind, I32), cap, ct.byref(trash))
    return idx, lind[:lc].copy(), trash.value


def matvec(gindices, values, x, m, nnz=3):
    idx = np.ascontiguousarray(gindices, dtype=np.int32).copy()
    v = np.ascontiguousarray(values, dtype=np.float64).copy()
    xx = np.ascontiguousarray(x, dtype=np.float64).copy()
    y = np.zeros(m)
    lib().ref_matvec(m, nnz, _p(idx, I32), _p(v, F64), _p(xx, F64), _p(y, F64))
    return y


def trmatvec(gindices, values, y, m, n, nnz=3):
    idx = np.ascontiguousarray(gindices, dtype=np.int32).copy()
    v = np.ascontiguousarray(values, dtype=np.float64).copy()
    yy = np.ascontiguousarray(y, dtype=np.float64).copy()
    x = np.zeros(max(n, 1))
    lib().ref_trmatvec(m, nnz, _p(idx, I32), _p(v, F64), _p(yy, F64), _p(x, F64))
    return x[:n]


def stbmm(V, block_sizes, lam, invtt):
    """apply_weights (pcg_true.c:578-600) on the Toeplitz blocks of one rank:
    stbmmProd, or the white weighting when lam == 1."""
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32).copy()
    tt = np.ascontiguousarray(invtt, dtype=np.float64).copy()
    out = np.ascontiguousarray(V, dtype=np.float64).copy()
    lib().ref_stbmm(len(bs), _p(bs, I32), lam, _p(tt, F64), _p(out, F64))
    return out


class Flag(ct.Structure):
    """The reference's Flag (toeplitz.h:169-182)."""
    _fields_ = [(n, ct.c_int) for n in ("flag_bs", "flag_nfft", "flag_fftw", "flag_no_rshp", "flag_nofft",
                                        "flag_blockingcomm", "fixed_nfft", "fixed_bs", "flag_verbose",
                                        "flag_skip_build_gappy_blocks", "flag_param_distmin_fixed",
                                        "flag_precompute_lvl")]


def define_blocksize(n, lam, bs_flag, fixed_bs=0):
    """The reference's define_blocksize (toeplitz.c:168-253)."""
    f = lib().define_blocksize
    f.restype = ct.c_int
    return int(f(n, lam, bs_flag, fixed_bs))


def tpltz_init(n, lam, T, flag_bs=0, fixed_bs=0, flag_nfft=0, fixed_nfft=0):
    """The reference's tpltz_init (toeplitz.c:298-367): (nfft, blocksize, T_fft as
    complex [bs/2+1]); its arrays are released with tpltz_cleanup."""
    L = lib()
    fl = Flag()
    L.flag_stgy_init_auto(ct.byref(fl))
    fl.flag_bs, fl.fixed_bs, fl.flag_nfft, fl.fixed_nfft = flag_bs, fixed_bs, flag_nfft, fixed_nfft
    tt = np.ascontiguousarray(T, dtype=np.float64).copy()
    nfft, bs = ct.c_int(0), ct.c_int(0)
    tf, vf, vr = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
    pf, pb = ct.c_void_p(), ct.c_void_p()
    L.tpltz_init.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                             ct.c_void_p, ct.c_void_p, ct.c_void_p, Flag]
    rc = L.tpltz_init(n, lam, ct.byref(nfft), ct.byref(bs), ct.byref(tf), _p(tt, F64), ct.byref(vf), ct.byref(vr),
                      ct.byref(pf), ct.byref(pb), fl)
    if rc != 0:
        raise RuntimeError(f"reference tpltz_init failed (status {rc})")
    h = bs.value // 2 + 1
    out = np.ctypeslib.as_array(ct.cast(tf, ct.POINTER(F64)), shape=(2 * h,)).copy()
    L.tpltz_cleanup(ct.byref(tf), ct.byref(vf), ct.byref(vr), ct.byref(pf), ct.byref(pb))
    return nfft.value, bs.value, out[0::2] + 1j * out[1::2]


def apply_weights(block_sizes, lam, invtt, tod):
    """The reference's apply_weights (pcg_true.c:578-600) on one rank: white
    weighting for lambda 1, stbmmProd otherwise."""
    return stbmm(tod, block_sizes, lam, invtt)  # ref_stbmm calls apply_weights itself


def pcg(gindices, values, signal, noise, block_sizes, lam, invtt, tol=1e-8, maxiter=500, nnz=3, precond=0,
        z_2lvl=0):
    """Single-rank MLmap set-up + PCG_GLS_true (precond 0: block Jacobi, 1/2: the
    two-level preconditioners with z_2lvl columns). Returns (x, lstid, cond, hits, res_rel)."""
    m = len(signal)
    idx = np.ascontiguousarray(gindices, dtype=np.int32).copy()
    v = np.ascontiguousarray(values, dtype=np.float64).copy()
    sig = np.ascontiguousarray(signal, dtype=np.float64).copy()
    noi = np.ascontiguousarray(noise, dtype=np.float64).copy()
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32).copy()
    tt = np.ascontiguousarray(invtt, dtype=np.float64).copy()
    cap = int(np.unique(idx).size)
    x = np.zeros(cap)
    lstid = np.zeros(cap, dtype=np.int32)
    cond = np.zeros(cap // 3 + 1)
    hits = np.zeros(cap // 3 + 1, dtype=np.int32)
    with tempfile.TemporaryDirectory() as td:
        n = lib().ref_pcg_precond(m, nnz, _p(idx, I32), _p(v, F64), _p(sig, F64), _p(noi, F64), len(bs),
                                  _p(bs, I32), lam, _p(tt, F64), F64(tol), maxiter, precond, z_2lvl, td.encode(),
                                  b"oracle", _p(x, F64), _p(lstid, I32), _p(cond, F64), _p(hits, I32), cap)
        res = np.fromfile(os.path.join(td, "pcg_residuals_oracle.dat"), dtype=np.float64)
    return x[:n].copy(), lstid[:n].copy(), cond[:n // 3].copy(), hits[:n // 3].copy(), res


def mlmap(nranks, data_size_proc, nb_blocks_proc, block_sizes, pix, weights, signal, noise, lam, invtt, nside,
          tol=1e-8, maxiter=500, nnz=3):
    """MLmap on `nranks` forked ranks; returns the I, Q, U, Cond, Hits maps."""
    dsp = np.ascontiguousarray(data_size_proc, dtype=np.int32)
    nbp = np.ascontiguousarray(nb_blocks_proc, dtype=np.int32)
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32)
    px = np.ascontiguousarray(pix, dtype=np.int32)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    s = np.ascontiguousarray(signal, dtype=np.float64)
    nz = np.ascontiguousarray(noise, dtype=np.float64)
    tt = np.ascontiguousarray(invtt, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        rc = lib().ref_mlmap(nranks, td.encode(), b"oracle", F64(tol), maxiter, nside, nnz, lam, _p(dsp, I32),
                             _p(nbp, I32), _p(bs, I32), _p(px, I32), _p(w, F64), _p(s, F64), _p(nz, F64),
                             _p(tt, F64))
        if rc != 0:
            raise RuntimeError(f"reference MLmap failed (status {rc})")
        rd = lambda name, dt: np.fromfile(os.path.join(td, f"{name}_oracle.fits"), dtype=dt)  # noqa: E731
        out = (rd("mapI", np.float64), rd("mapQ", np.float64), rd("mapU", np.float64), rd("Cond", np.float64),
               rd("Hits", np.int32))
        res = np.fromfile(os.path.join(td, "pcg_residuals_oracle.dat"), dtype=np.float64)
    return out + (res,)


def operator_time(nranks, data_size_proc, nb_blocks_proc, block_sizes, pix, weights, lam, invtt, reps=1, nnz=3,
                  each=False):
    """Seconds per P^T N^-1 P application (max over ranks), reference code on host cores:
    the mean over `reps` applications, or (each=True) the list of their times."""
    dsp = np.ascontiguousarray(data_size_proc, dtype=np.int32)
    nbp = np.ascontiguousarray(nb_blocks_proc, dtype=np.int32)
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32)
    px = np.ascontiguousarray(pix, dtype=np.int32)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    tt = np.ascontiguousarray(invtt, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "t.bin")
        rc = lib().ref_operator_time(nranks, nnz, lam, reps, _p(dsp, I32), _p(nbp, I32), _p(bs, I32), _p(px, I32),
                                     _p(w, F64), _p(tt, F64), path.encode())
        if rc != 0:
            raise RuntimeError(f"reference operator timing failed (status {rc})")
        t = np.fromfile(path, dtype=np.float64)
        return [float(v) for v in t] if each else float(t.mean())


def _scan_args(sc):
    nsweeps = np.array([len(s) - 1 for s in sc.sweeps], dtype=np.int32)
    flat = lambda rows, dt: np.ascontiguousarray(np.concatenate([np.asarray(r) for r in rows]), dtype=dt)  # noqa: E731
    sweeps = flat(sc.sweeps, np.int32)
    az = flat(sc.az, np.float64) if sc.ground else np.zeros(int(sum(sc.ces_length(i) for i in range(sc.nces))))
    hwp = flat(sc.hwp, np.float64) if sc.nhwp else np.zeros_like(az)
    azmin = np.ascontiguousarray(sc.az_min, dtype=np.float64)
    azmax = np.ascontiguousarray(sc.az_max, dtype=np.float64)
    return nsweeps, sweeps, az, azmin, azmax, hwp


def templates_ops(sc, w_block, d, tau):
    """The reference's TrTVecProd, TVecProd, BuildKernel and InvKernel on the template
    classes MTmap builds (ref_templates_ops).  Returns (T^T d, T tau, kernels,
    pseudo-inverses), kernels block after block."""
    nsw, sw, az, azmin, azmax, hwp = _scan_args(sc)
    wb = np.ascontiguousarray(w_block, dtype=np.float64)
    dd = np.ascontiguousarray(d, dtype=np.float64)
    tt = np.ascontiguousarray(tau, dtype=np.float64)
    amp = np.zeros(sc.n_templates)
    tod = np.zeros(dd.size)
    kern = np.zeros(sc.kernel_size)
    kinv = np.zeros(sc.kernel_size)
    r = lib().ref_templates_ops(sc.nces, sc.ndet, _p(nsw, I32), _p(sw, I32), _p(az, F64), _p(azmin, F64),
                                _p(azmax, F64), _p(hwp, F64), sc.npoly, sc.ground, sc.n_sss_bins, sc.nhwp,
                                F64(sc.delta_t), F64(sc.fs), _p(wb, F64), _p(dd, F64), _p(tt, F64), _p(amp, F64),
                                _p(tod, F64), _p(kern, F64), _p(kinv, F64))
    if r != sc.n_templates:
        raise RuntimeError(f"reference built {r} templates, expected {sc.n_templates}")
    return amp, tod, kern, kinv


def mtmap(sc, pix, weights, signal, noise, invtt, nside, tol=1e-8, maxiter=500, nnz=3):
    """MTmap on one rank (ref_mtmap); returns the I, Q, U, Cond, Hits maps and the
    residual history."""
    nsw, sw, az, azmin, azmax, hwp = _scan_args(sc)
    px = np.ascontiguousarray(pix, dtype=np.int32)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    s = np.ascontiguousarray(signal, dtype=np.float64)
    nz = np.ascontiguousarray(noise, dtype=np.float64)
    tt = np.ascontiguousarray(invtt, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        rc = lib().ref_mtmap(td.encode(), b"oracle", sc.nces, sc.ndet, _p(nsw, I32), _p(sw, I32), _p(az, F64),
                             _p(azmin, F64), _p(azmax, F64), _p(hwp, F64), sc.npoly, sc.ground, sc.n_sss_bins,
                             sc.nhwp, F64(sc.delta_t), F64(sc.fs), F64(tol), maxiter, nside, nnz, _p(px, I32),
                             _p(w, F64), _p(s, F64), _p(nz, F64), _p(tt, F64))
        if rc != 0:
            raise RuntimeError(f"reference MTmap failed (status {rc})")
        rd = lambda name, dt: np.fromfile(os.path.join(td, f"{name}_oracle.fits"), dtype=dt)  # noqa: E731
        out = (rd("mapI", np.float64), rd("mapQ", np.float64), rd("mapU", np.float64), rd("Cond", np.float64),
               rd("Hits", np.int32))
        res = np.fromfile(os.path.join(td, "pcg_residuals_oracle.dat"), dtype=np.float64)
    return out + (res,)
