"""Set-up of MTmap's template-filtered solve (host side, in libmidapack_b200.so).

MTmap (mappraiser/src/mappraiser.c:387-800) marginalises per-block template
amplitudes (algebra/src/templates/templates.c): Legendre polynomials per sweep,
the azimuth-binned ground signal, HWP harmonics over delta_t chunks.  ``layout``
gives the template matrix of every CES in ELL form (one (bin, weight) pair per
class per sample), ``kernels`` the per-block pseudo-inverses
``pinv(w_b T_b^T T_b)`` that MTmap's PCG applies (both on the host, as in the
reference); ``Filter`` applies MTmap's weighting ``W - W T B T^T W`` to a TOD on
the device.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np

from . import Context, _ptr, check, lib


class _ScanC(ct.Structure):
    _fields_ = [("nces", ct.c_int), ("ndet", ct.c_int), ("npoly", ct.c_int), ("ground", ct.c_int),
                ("n_sss_bins", ct.c_int), ("nhwp", ct.c_int), ("delta_t", ct.c_double), ("fs", ct.c_double),
                ("nsweeps", ct.c_void_p), ("sweeps", ct.c_void_p), ("az", ct.c_void_p), ("az_min", ct.c_void_p),
                ("az_max", ct.c_void_p), ("hwp", ct.c_void_p)]


@dataclass
class Scan:
    """MTmap's scan arguments: per CES the sweep stamps (nsweeps + 1, the last =
    the CES length), boresight azimuth and its range, HWP angle; the template set."""
    sweeps: list
    az: list | None
    az_min: np.ndarray | None
    az_max: np.ndarray | None
    hwp: list | None
    ndet: int
    npoly: int
    ground: int
    n_sss_bins: int
    nhwp: int
    delta_t: float
    fs: float

    @property
    def nces(self) -> int:
        return len(self.sweeps)

    @property
    def n_class(self) -> int:
        return self.npoly + self.ground + 2 * self.nhwp

    def _c(self):
        keep = {}
        f64 = lambda rows: np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64) for r in rows]))  # noqa: E731
        keep["nsweeps"] = np.array([len(s) - 1 for s in self.sweeps], dtype=np.int32)
        keep["sweeps"] = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.int32) for s in self.sweeps]))
        if self.ground:
            keep["az"] = f64(self.az)
            keep["az_min"] = np.ascontiguousarray(self.az_min, dtype=np.float64)
            keep["az_max"] = np.ascontiguousarray(self.az_max, dtype=np.float64)
        if self.nhwp:
            keep["hwp"] = f64(self.hwp)
        s = _ScanC(self.nces, self.ndet, self.npoly, self.ground, self.n_sss_bins, self.nhwp, float(self.delta_t),
                   float(self.fs), *(keep[k].ctypes.data if k in keep else None
                                     for k in ("nsweeps", "sweeps", "az", "az_min", "az_max", "hwp")))
        return s, keep

    def n_samples_ces(self) -> int:
        return int(sum(int(s[-1]) for s in self.sweeps))


def layout(scan: Scan):
    """(bins [samples of all CESs, n_class] int32, weights [same] f64, nt [nces])."""
    s, keep = scan._c()
    M = scan.n_samples_ces()
    bins = np.zeros((M, scan.n_class), dtype=np.int32)
    wg = np.zeros((M, scan.n_class))
    nt = np.zeros(scan.nces, dtype=np.int32)
    check(lib().mdp_template_layout(ct.addressof(s), bins.ctypes.data, wg.ctypes.data, nt.ctypes.data),
          "mdp_template_layout")
    return bins, wg, nt


def kernels(scan: Scan, w_block):
    """The pseudo-inverted kernels pinv(w_b T_b^T T_b), block after block (flat)."""
    s, keep = scan._c()
    _, _, nt = layout(scan)
    w = np.ascontiguousarray(w_block, dtype=np.float64)
    if w.size != scan.nces * scan.ndet:
        raise ValueError("one weight per block (nces * ndet)")
    out = np.zeros(int(scan.ndet * (nt.astype(np.int64) ** 2).sum()))
    check(lib().mdp_template_kernels(ct.addressof(s), w.ctypes.data, out.ctypes.data), "mdp_template_kernels")
    return out


class Filter:
    """MTmap's TOD weighting on the device (mdp_templates_filter):
    ``y = W x - W T B T^T W x`` with W the white-noise weight of each block."""

    def __init__(self, ctx: Context, scan: Scan, w_block):
        self.ctx = ctx
        s, keep = scan._c()
        w = np.ascontiguousarray(w_block, dtype=np.float64)
        if w.size != scan.nces * scan.ndet:
            raise ValueError("one weight per block (nces * ndet)")
        self.h = ct.c_void_p()
        check(lib().mdp_templates_create(ctx.h, ct.addressof(s), w.ctypes.data, ct.byref(self.h)),
              "mdp_templates_create")
        m, na = ct.c_int64(), ct.c_int64()
        check(lib().mdp_templates_samples(self.h, ct.byref(m), ct.byref(na)), "mdp_templates_samples")
        self.m, self.n_amplitudes = m.value, na.value

    def __call__(self, x, out=None):
        """Filtered copy of the CUDA float64 tensor x (or into `out`, which may be x)."""
        import torch
        if x.numel() != self.m or x.dtype != torch.float64:
            raise ValueError(f"expected {self.m} float64 samples")
        y = torch.empty_like(x) if out is None else out
        check(lib().mdp_templates_filter(self.ctx.h, self.h, ct.c_void_p(_ptr(x)), ct.c_void_p(_ptr(y))),
              "mdp_templates_filter")
        return y

    def close(self):
        if self.h:
            lib().mdp_templates_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def solve(ctx: Context, A, N, F: Filter, signal, noise, tol=1e-8, maxiter=500, verbose=False):
    """MTmap's template-filtered PCG on device tensors (mdp_gls_solve_templates): N is
    the white noise operator (``midapack_b200.Noise(ctx, block_sizes, 1, w_block)``), F
    the filter built from the same weights.  Returns (x, lstid, cond, hits, res_rel,
    info) like ``midapack_b200.gls_solve``."""
    import torch
    from . import SolveInfo, SolveParams, c_f64p
    n0 = A.shape()["n_map"]
    x = torch.empty(max(n0, 1), dtype=torch.float64, device="cuda")
    lst = torch.empty(max(n0, 1), dtype=torch.int32, device="cuda")
    cond = torch.empty(max(n0 // 3, 1), dtype=torch.float64, device="cuda")
    hits = torch.empty(max(n0 // 3, 1), dtype=torch.int32, device="cuda")
    res = np.zeros(maxiter + 1)
    prm = SolveParams(tol, maxiter, 1 if verbose else 0, 0, 0)
    info = SolveInfo()
    check(lib().mdp_gls_solve_templates(ctx.h, A.h, N.h, F.h, ct.c_void_p(_ptr(signal)), ct.c_void_p(_ptr(noise)),
                                        ct.byref(prm), ct.c_void_p(x.data_ptr()), ct.c_void_p(lst.data_ptr()),
                                        ct.c_void_p(cond.data_ptr()), ct.c_void_p(hits.data_ptr()),
                                        res.ctypes.data_as(c_f64p), ct.byref(info)), "mdp_gls_solve_templates")
    n = info.n_map
    return x[:n], lst[:n], cond[:n // 3], hits[:n // 3], res[:info.iterations + 1], info
