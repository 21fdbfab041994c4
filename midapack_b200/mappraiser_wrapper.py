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
    """Ranks of `comm`: None or an MPI handle (int) is one rank; a
    torch.distributed process group is its size."""
    if comm is None or isinstance(comm, int):
        return 1
    import torch.distributed as dist
    if isinstance(comm, dist.ProcessGroup):
        return dist.get_world_size(comm)
    size = getattr(comm, "size", None)
    return int(size() if callable(size) else size) if size is not None else 1


def MLmap(comm, params, data_size_proc, nb_blocks_loc, local_blocks_sizes, nnz, pixels, pixweights, signal, noise,
          invtt, shard=None):
    """Compute the GLS estimator assuming a Toeplitz-structured noise covariance.

    With one rank (comm None or an MPI handle) the whole solve runs through the
    C entry point MLmap on this process's GPU.  With a torch.distributed process
    group of several ranks (one process per GPU), each rank passes its own
    samples exactly as the reference's callers do (data_size_proc: the samples
    of every rank; local_blocks_sizes: this rank's Toeplitz blocks; pixels,
    weights, signal, noise, invtt: this rank's arrays; mappraiser.c:64-88), the
    solve is the sharded PCG of midapack_b200.dist (one map all-reduce per
    operator application) and rank 0 writes the five maps and the residual
    history.  `shard` optionally replaces this rank's GPU shard by an object
    with the same methods (tests)."""
    if _comm_size(comm) > 1:
        return _mlmap_sharded(comm, params, data_size_proc, nb_blocks_loc, local_blocks_sizes, nnz, pixels,
                              pixweights, signal, noise, invtt, shard)
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


def _mlmap_sharded(group, params, data_size_proc, nb_blocks_loc, local_blocks_sizes, nnz, pixels, pixweights, signal,
                   noise, invtt, shard=None):
    import os

    import torch
    import torch.distributed as dist

    from midapack_b200.dist import GpuShard, ShardedGLS
    rank = dist.get_rank(group)
    dsp = np.asarray(data_size_proc, dtype=np.int64)
    m = int(dsp[rank])
    lbs = np.ascontiguousarray(np.asarray(local_blocks_sizes, dtype=np.int32)[:nb_blocks_loc])
    lam = int(params["Lambda"])
    if params["solver"] != 0 or params["precond"] != 0 or nnz != 3:
        raise ValueError("several ranks: solver 0 with precond 0 (block Jacobi) and Nnz 3")
    if len(pixels) != nnz * m or len(signal) != m or int(lbs.sum()) != m or len(invtt) < lam * nb_blocks_loc:
        raise ValueError(f"rank {rank}: arrays do not match data_size_proc[{rank}] = {m} and the local blocks")
    own = None
    if shard is None:
        import midapack_b200 as mb
        ctx = mb.Context(torch.cuda.current_device())
        dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()  # noqa: E731
        shard = own = GpuShard(ctx, dev(pixels, np.int32), dev(pixweights, np.float64), dev(signal, np.float64),
                               dev(noise, np.float64), lbs, lam, np.ascontiguousarray(invtt[:lam * nb_blocks_loc]))
    hist = []
    x, pg, rcond, hits, info = ShardedGLS(shard, group).solve(tol=params["tol"], maxiter=params["maxiter"],
                                                              precision="fp64", on_iter=hist.append)
    if own is not None:
        own.close()
    if rank == 0:
        nside = int(params["nside"])
        npix = 12 * nside * nside
        p = pg.cpu().numpy().astype(np.int64)
        xs = x.cpu().numpy()
        maps = [np.zeros(npix) for _ in range(4)] + [np.zeros(npix, dtype=np.int32)]
        for k in range(3):
            maps[k][p] = xs[k::3]
        maps[3][p] = rcond.cpu().numpy()
        maps[4][p] = hits.cpu().numpy().astype(np.int32)
        out, ref = params["path_output"], params["ref"]
        for name, mp in zip(("mapI", "mapQ", "mapU", "Cond", "Hits"), maps):
            data = np.ascontiguousarray(mp)
            lib().write_map(data.ctypes.data, 31 if name == "Hits" else 82, nside,
                            os.path.join(out, f"{name}_{ref}.fits").encode(), b"\x01", b"C")
        res0 = info.res0
        rr = np.sqrt(np.array([res0] + hist) / res0) if res0 > 0 else np.zeros(1)
        rr.astype(np.float64).tofile(os.path.join(out, f"pcg_residuals_{ref}.dat"))
    return info


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
