"""Python mirror of MAPPRAISER's ctypes wrapper, backed by libmidapack_b200.

Same call as ``mappraiser/python/mappraiser_wrapper/__init__.py:125-189``::

    MLmap(comm, params, data_size_proc, nb_blocks_loc, local_blocks_sizes, nnz,
          pixels, pixweights, signal, noise, invtt)

with the same dtypes (int32 pixels, float64 weights/signal/noise/invtt,
``__init__.py:23-28``) and the same ``params`` keys (path_output, ref, solver,
precond, Z_2lvl, ptcomm_flag, tol, maxiter, enlFac, ortho_alg, bs_red, nside,
Lambda).  ``comm`` is accepted for signature compatibility; this build runs one
rank on one GPU (an mpi4py communicator of size > 1 is rejected).

Also the reference's C structs (Mat, Block, Flag, Tpltz) as ctypes
structures, for callers that drive MatInit / stbmmProd / PCG_GLS_true
directly (algebra/include/mapmat/mapmat.h:46-69,
algebra/include/toeplitz/toeplitz.h:152-203).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import check, lib

SIGNAL_TYPE = np.float64
PIXEL_TYPE = np.int32
WEIGHT_TYPE = np.float64
INVTT_TYPE = np.float64

available = True


class Mat(ct.Structure):
    _fields_ = [("flag", ct.c_int), ("m", ct.c_int), ("nnz", ct.c_int), ("trash_pix", ct.c_int),
                ("indices", ct.POINTER(ct.c_int)), ("values", ct.POINTER(ct.c_double)),
                ("id_last_pix", ct.POINTER(ct.c_int)), ("ll", ct.POINTER(ct.c_int)), ("lcount", ct.c_int),
                ("lindices", ct.POINTER(ct.c_int)), ("comm", ct.c_int), ("com_indices", ct.POINTER(ct.c_int)),
                ("com_count", ct.c_int), ("steps", ct.c_int), ("nS", ct.POINTER(ct.c_int)),
                ("nR", ct.POINTER(ct.c_int)), ("R", ct.POINTER(ct.POINTER(ct.c_int))),
                ("S", ct.POINTER(ct.POINTER(ct.c_int)))]


class Block(ct.Structure):
    _fields_ = [("idv", ct.c_int64), ("T_block", ct.POINTER(ct.c_double)), ("lambda_", ct.c_int), ("n", ct.c_int)]


class Flag(ct.Structure):
    _fields_ = [(n, ct.c_int) for n in ("flag_bs", "flag_nfft", "flag_fftw", "flag_no_rshp", "flag_nofft",
                                        "flag_blockingcomm", "fixed_nfft", "fixed_bs", "flag_verbose",
                                        "flag_skip_build_gappy_blocks", "flag_param_distmin_fixed",
                                        "flag_precompute_lvl")]


class Tpltz(ct.Structure):
    _fields_ = [("nrow", ct.c_int64), ("m_cw", ct.c_int), ("m_rw", ct.c_int), ("tpltzblocks", ct.POINTER(Block)),
                ("nb_blocks_loc", ct.c_int), ("nb_blocks_tot", ct.c_int), ("idp", ct.c_int64),
                ("local_V_size", ct.c_int), ("flag_stgy", Flag), ("comm", ct.c_int)]


MPI_COMM_WORLD = 0x44000000


def _comm_size(comm) -> int:
    if comm is None or isinstance(comm, int):
        return 1
    size = getattr(comm, "size", None)
    return int(size) if size is not None else 1


def MLmap(comm, params, data_size_proc, nb_blocks_loc, local_blocks_sizes, nnz, pixels, pixweights, signal, noise,
          invtt):
    """Compute the GLS estimator assuming a Toeplitz-structured noise covariance (one GPU)."""
    if _comm_size(comm) != 1:
        raise RuntimeError("midapack_b200 MLmap runs one rank per process on one GPU")
    L = lib()
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
    dsp, lbs, pix = i32(data_size_proc), i32(local_blocks_sizes), i32(pixels)
    w, s, nz, tt = f64(pixweights), f64(signal), f64(noise), f64(invtt)
    P = lambda a, t: a.ctypes.data_as(ct.POINTER(t))  # noqa: E731
    L.MLmap(MPI_COMM_WORLD, params["path_output"].encode("ascii"), params["ref"].encode("ascii"), params["solver"],
            params["precond"], params["Z_2lvl"], params["ptcomm_flag"], params["tol"], params["maxiter"],
            params["enlFac"], params["ortho_alg"], params["bs_red"], params["nside"], P(dsp, ct.c_int32),
            nb_blocks_loc, P(lbs, ct.c_int32), nnz, P(pix, ct.c_int32), P(w, ct.c_double), P(s, ct.c_double),
            P(nz, ct.c_double), params["Lambda"], P(tt, ct.c_double))


def read_fits_map(path: str) -> np.ndarray:
    """Reads the single-column HEALPix binary table MLmap writes."""
    with open(path, "rb") as f:
        raw = f.read()
    hdrs = []
    pos = 0
    for _ in range(2):
        while True:
            block = raw[pos:pos + 2880]
            pos += 2880
            cards = [block[i:i + 80].decode("ascii") for i in range(0, 2880, 80)]
            hdrs.append(cards)
            if any(c.startswith("END") for c in cards):
                break
    cards = [c for blk in hdrs for c in blk]
    get = lambda k: [c for c in cards if c.startswith(k.ljust(8) + "=")][-1].split("=")[1].split("/")[0].strip()  # noqa
    nrow = int(get("NAXIS2"))
    form = get("TFORM1").strip("'").strip()
    dt = ">f8" if form.endswith("D") else ">i4"
    return np.frombuffer(raw, dtype=dt, count=nrow, offset=pos).astype(dt[1:])
