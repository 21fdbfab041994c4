"""Set-up of MTmap's template-filtered solve (host side, in libmidapack_b200.so).

MTmap (mappraiser/src/mappraiser.c:387-800) marginalises per-block template
amplitudes (algebra/src/templates/templates.c): Legendre polynomials per sweep,
the azimuth-binned ground signal, HWP harmonics over delta_t chunks.  ``layout``
gives the template matrix of every CES in ELL form (one (bin, weight) pair per
class per sample), ``kernels`` the per-block pseudo-inverses
``pinv(w_b T_b^T T_b)`` that MTmap's PCG applies.  Both run on the host, as in
the reference.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import numpy as np

from . import check, lib


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
