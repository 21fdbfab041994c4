"""midapack_b200: the GLS map-making hot path of MIDAPACK/MAPPRAISER on one B200.

The numerical work lives in ``libmidapack_b200.so`` (CUDA, sm_100a), reached
through its C ABI (``include/midapack_b200.h`` for device pointers,
``include/{mapmat,toeplitz,mappraiser}.h`` for the reference-compatible host
API).  This module is a thin ctypes layer: it never computes anything itself
and raises if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmidapack_b200.so")

MDP_OK = 0
MDP_ENOCONV = 7
_lib = None

c_i32p = ct.POINTER(ct.c_int32)
c_f64p = ct.POINTER(ct.c_double)


class MidapackError(RuntimeError):
    pass


class SolveParams(ct.Structure):
    _fields_ = [("tol", ct.c_double), ("maxiter", ct.c_int), ("verbose", ct.c_int), ("precond", ct.c_int),
                ("z_2lvl", ct.c_int)]


class SolveInfo(ct.Structure):
    _fields_ = [("iterations", ct.c_int), ("converged", ct.c_int), ("res0", ct.c_double), ("res", ct.c_double),
                ("n_map", ct.c_int64), ("n_cut", ct.c_int64), ("precond_seconds", ct.c_double),
                ("solve_seconds", ct.c_double), ("outer_iterations", ct.c_int), ("fp64_applications", ct.c_int)]


class ECGParams(ct.Structure):
    _fields_ = [("tol", ct.c_double), ("maxiter", ct.c_int), ("enl_fac", ct.c_int), ("ortho_alg", ct.c_int),
                ("bs_red", ct.c_int), ("verbose", ct.c_int)]


class MultiParams(ct.Structure):
    _fields_ = [("tol", ct.c_double), ("maxiter", ct.c_int), ("inner_tol", ct.c_double), ("inner_maxiter", ct.c_int),
                ("slots", ct.c_int), ("use_graph", ct.c_int), ("verbose", ct.c_int)]


class MultiColInfo(ct.Structure):
    _fields_ = [("iterations", ct.c_int), ("outer_iterations", ct.c_int), ("converged", ct.c_int),
                ("res0", ct.c_double), ("res", ct.c_double)]


class MultiInfo(ct.Structure):
    _fields_ = [("slots", ct.c_int), ("graph", ct.c_int), ("total_iterations", ct.c_int),
                ("batched_iterations", ct.c_int), ("fp64_applications", ct.c_int), ("n_map", ct.c_int64),
                ("n_cut", ct.c_int64), ("precond_seconds", ct.c_double), ("solve_seconds", ct.c_double)]


# exported symbols of include/*.h, with their ctypes signatures
_SIGS = {
    # device API (include/midapack_b200.h)
    "mdp_strerror": (ct.c_char_p, [ct.c_int]),
    "mdp_last_error": (ct.c_char_p, []),
    "mdp_context_create": (ct.c_int, [ct.c_int, ct.POINTER(ct.c_void_p)]),
    "mdp_context_destroy": (None, [ct.c_void_p]),
    "mdp_context_trim": (ct.c_int, [ct.c_void_p]),
    "mdp_context_set_stream": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "mdp_context_stream": (ct.c_void_p, [ct.c_void_p]),
    "mdp_synchronize": (ct.c_int, [ct.c_void_p]),
    "mdp_launch_count": (ct.c_uint64, [ct.c_void_p]),
    "mdp_profile_enable": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "mdp_profile_read": (ct.c_int, [ct.c_void_p, c_f64p, ct.POINTER(ct.c_int64)]),
    "mdp_pointing_create": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_void_p, ct.c_void_p,
                                       ct.POINTER(ct.c_void_p)]),
    "mdp_pointing_destroy": (None, [ct.c_void_p]),
    "mdp_pointing_shape": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int),
                                      ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int)]),
    "mdp_pointing_lindices": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_pointing_local_indices": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_matvec": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_trmatvec": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_noise_create": (ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(ct.c_int64), c_i32p, ct.c_int, c_f64p,
                                    ct.POINTER(ct.c_void_p)]),
    "write_map": (None, [ct.c_void_p, ct.c_int, ct.c_long, ct.c_char_p, ct.c_char, ct.c_char_p]),
    "mdp_noise_set_plan": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_char_p]),
    "mdp_noise_destroy": (None, [ct.c_void_p]),
    "mdp_stbmm": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_stbmm_noalloc": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_stbmm_fp32": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_prepare_fp32": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_noise_tile_fp32": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                                       ct.POINTER(ct.c_int64)]),
    "mdp_noise_tile": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int64)]),
    "mdp_gls_solve_multi": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int,
                                       ct.c_int64, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_local_blocks": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_block_inverse": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                     ct.POINTER(ct.c_int64)]),
    "mdp_pointing_cut": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_int64)]),
    "mdp_gls_residual": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                    ct.c_void_p]),
    "mdp_apply_op": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int]),
    "mdp_noise_plan": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                                  ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                                  ct.POINTER(ct.c_int)]),
    "mdp_gls_solve": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                 ct.POINTER(SolveParams), ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                 c_f64p, ct.POINTER(SolveInfo)]),
    "mdp_gls_solve_mixed": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                       ct.POINTER(SolveParams), ct.c_double, ct.c_int, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, ct.c_void_p, c_f64p, ct.POINTER(SolveInfo)]),
    "mdp_ecg_solve": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                 ct.POINTER(ECGParams), ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                 c_f64p, ct.POINTER(SolveInfo)]),
    "mdp_apod_window": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p]),
    "mdp_periodogram": (ct.c_int, [ct.c_void_p, ct.c_int, c_i32p, ct.c_void_p, ct.c_double, ct.c_void_p]),
    "mdp_noise2invtt": (ct.c_int, [ct.c_void_p, ct.c_int, c_i32p, ct.c_void_p, ct.c_int, ct.c_double, ct.c_int,
                                   ct.c_void_p, c_f64p, c_i32p]),
    "mdp_template_layout": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_template_kernels": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_templates_create": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_void_p)]),
    "mdp_templates_destroy": (None, [ct.c_void_p]),
    "mdp_templates_samples": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)]),
    "mdp_templates_filter": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mdp_gls_solve_templates": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p, ct.POINTER(SolveParams), ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p, ct.c_void_p, c_f64p, ct.POINTER(SolveInfo)]),
    # reference-compatible host API (include/mapmat.h, toeplitz.h, mappraiser.h)
    "MatInit": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, c_i32p, c_f64p, ct.c_int, ct.c_int]),
    "MatSetIndices": (None, [ct.c_void_p, ct.c_int, ct.c_int, c_i32p]),
    "MatSetValues": (None, [ct.c_void_p, ct.c_int, ct.c_int, c_f64p]),
    "MatFree": (None, [ct.c_void_p]),
    "MatLocalShape": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "MatComShape": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
    "MatVecProd": (ct.c_int, [ct.c_void_p, c_f64p, c_f64p, ct.c_int]),
    "TrMatVecProd": (ct.c_int, [ct.c_void_p, c_f64p, c_f64p, ct.c_int]),
    "greedyreduce": (ct.c_int, [ct.c_void_p, c_f64p]),
    "tpltz_init": (ct.c_int, None),
    "tpltz_cleanup": (ct.c_int, None),
    "flag_stgy_init_auto": (ct.c_int, [ct.c_void_p]),
    "flag_stgy_init_zeros": (ct.c_int, [ct.c_void_p]),
    "define_blocksize": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int, ct.c_int]),
    "stbmmProd": (ct.c_int, [ct.c_void_p, c_f64p]),
    "apply_weights": (ct.c_int, [ct.c_void_p, c_f64p]),
    "defineTpltz_avg": (ct.c_int, None),
    "defineBlocks_avg": (ct.c_int, [ct.c_void_p, c_f64p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int64]),
    "precondblockjacobilike": (ct.c_int, None),
    "build_precond": (None, None),
    "apply_precond": (None, None),
    "free_precond": (None, None),
    "get_pixshare_pond": (None, [ct.c_void_p, c_f64p]),
    "PCG_GLS_true": (ct.c_int, [ct.c_char_p, ct.c_char_p, ct.c_void_p, ct.c_void_p, c_f64p, c_f64p, c_f64p, c_f64p,
                                c_i32p, ct.c_double, ct.c_int, ct.c_int, ct.c_int]),
    "ECG_GLS": (ct.c_int, [ct.c_char_p, ct.c_char_p, ct.c_void_p, ct.c_void_p, c_f64p, c_f64p, c_f64p, c_f64p,
                           c_i32p, ct.c_double, ct.c_int, ct.c_int, ct.c_int, ct.c_int]),
    "MLmap": (None, [ct.c_int, ct.c_char_p, ct.c_char_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                     ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, c_i32p, ct.c_int, c_i32p, ct.c_int, c_i32p,
                     c_f64p, c_f64p, c_f64p, ct.c_int, c_f64p]),
    "MTmap": (None, None),
    "MLmap_b200": (ct.c_int, [ct.c_int, ct.c_int, ct.c_double, ct.c_int, ct.c_int, ct.c_int, ct.c_int, c_i32p,
                              ct.c_int, c_i32p, c_f64p, c_f64p, c_f64p, ct.c_int, c_f64p, c_f64p, c_f64p, c_f64p,
                              c_f64p, c_i32p, ct.POINTER(ct.c_int), c_f64p]),
}


def lib():
    """The loaded CUDA library.  Raises if it was not built (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MidapackError(f"{LIB_PATH} is missing: build it with `python -m midapack_b200.build`")
        L = ct.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            if args is not None:
                f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != MDP_OK:
        L = lib()
        raise MidapackError(f"{what}: {L.mdp_strerror(rc).decode()} ({L.mdp_last_error().decode()})")


def _ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (or an int address)."""
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise MidapackError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise MidapackError("expected a contiguous tensor")
    return t.data_ptr()


class Context:
    """One device, one stream (by default the current torch stream)."""

    def __init__(self, device: int = 0, use_torch_stream: bool = True):
        self.h = ct.c_void_p()
        check(lib().mdp_context_create(device, ct.byref(self.h)), "mdp_context_create")
        if use_torch_stream:
            import torch
            s = torch.cuda.current_stream(device).cuda_stream
            # torch's default stream is the legacy default stream, handle 0; the
            # C API reads NULL as "own stream", so name it explicitly (cudaStreamLegacy)
            check(lib().mdp_context_set_stream(self.h, ct.c_void_p(s if s else 1)), "mdp_context_set_stream")

    def synchronize(self):
        check(lib().mdp_synchronize(self.h), "mdp_synchronize")

    def profile(self, enable: bool = True):
        check(lib().mdp_profile_enable(self.h, 1 if enable else 0), "mdp_profile_enable")

    def profile_read(self):
        ms = (ct.c_double * 4)()
        n = (ct.c_int64 * 4)()
        check(lib().mdp_profile_read(self.h, ms, n), "mdp_profile_read")
        return {k: (ms[i], n[i]) for i, k in enumerate(("P", "Ninv", "Pt", "vec"))}

    def trim(self):
        """Frees the work buffers the context keeps between solves."""
        check(lib().mdp_context_trim(self.h), "mdp_context_trim")

    @property
    def launches(self) -> int:
        return int(lib().mdp_launch_count(self.h))

    def close(self):
        if self.h:
            lib().mdp_context_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pointing:
    """Device pointing matrix (reference Mat) built from global indices on the GPU."""

    def __init__(self, ctx: Context, gindices, values, m: int, nnz: int = 3):
        self.ctx = ctx
        self._values = values  # borrowed by the library: keep alive
        self.h = ct.c_void_p()
        check(lib().mdp_pointing_create(ctx.h, m, nnz, ct.c_void_p(_ptr(gindices)), ct.c_void_p(_ptr(values)),
                                        ct.byref(self.h)), "mdp_pointing_create")
        self.m, self.nnz = m, nnz

    def shape(self):
        lc, tr, n, trip = ct.c_int64(), ct.c_int(), ct.c_int64(), ct.c_int()
        check(lib().mdp_pointing_shape(self.h, ct.byref(lc), ct.byref(tr), ct.byref(n), ct.byref(trip)))
        return dict(lcount=lc.value, trash_pix=tr.value, n_map=n.value, triplet=trip.value)

    def lindices(self):
        import torch
        out = torch.empty(self.shape()["lcount"], dtype=torch.int32, device="cuda")
        check(lib().mdp_pointing_lindices(self.ctx.h, self.h, ct.c_void_p(out.data_ptr())))
        return out

    def local_indices(self):
        import torch
        out = torch.empty(self.m * self.nnz, dtype=torch.int32, device="cuda")
        check(lib().mdp_pointing_local_indices(self.ctx.h, self.h, ct.c_void_p(out.data_ptr())))
        return out

    def matvec(self, x, y):
        check(lib().mdp_matvec(self.ctx.h, self.h, ct.c_void_p(_ptr(x)), ct.c_void_p(_ptr(y))), "mdp_matvec")

    def trmatvec(self, y, x):
        check(lib().mdp_trmatvec(self.ctx.h, self.h, ct.c_void_p(_ptr(y)), ct.c_void_p(_ptr(x))), "mdp_trmatvec")

    def close(self):
        if self.h:
            lib().mdp_pointing_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Noise:
    """Device inverse-noise operator (reference Tpltz): blocks of a banded symmetric Toeplitz."""

    def __init__(self, ctx: Context, block_sizes, lam: int, invtt, idv=None):
        self.ctx = ctx
        bs = np.ascontiguousarray(block_sizes, dtype=np.int32)
        if idv is None:
            idv = np.concatenate([[0], np.cumsum(bs.astype(np.int64))[:-1]])
        iv = np.ascontiguousarray(idv, dtype=np.int64)
        tt = np.ascontiguousarray(invtt, dtype=np.float64)
        self.h = ct.c_void_p()
        check(lib().mdp_noise_create(ctx.h, len(bs), iv.ctypes.data_as(ct.POINTER(ct.c_int64)),
                                     bs.ctypes.data_as(c_i32p), lam, tt.ctypes.data_as(c_f64p), ct.byref(self.h)),
              "mdp_noise_create")

    def set_plan(self, plan: str, fp32: bool = False):
        """Replaces the tile plan of one precision (see mdp_noise_set_plan):
        "auto", "model", "fft:N", "log2_ml,cluster,threads", "s,log_m1,log_m2", "c,C"."""
        check(lib().mdp_noise_set_plan(self.ctx.h, self.h, int(fp32), plan.encode()), "mdp_noise_set_plan")
        return self

    def _plan(self, fp32: int):
        lm, c, th, tu, s1, s2 = (ct.c_int() for _ in range(6))
        check(lib().mdp_noise_plan(self.ctx.h, self.h, fp32, ct.byref(lm), ct.byref(c), ct.byref(th), ct.byref(tu),
                                   ct.byref(s1), ct.byref(s2)))
        if s1.value and c.value:
            return dict(cluster_four_step=[1 << s1.value, 1 << s2.value], tuned=bool(tu.value))
        if s1.value:
            return dict(split=[1 << s1.value, 1 << s2.value], tuned=bool(tu.value))
        return dict(cta_points=1 << lm.value, threads=th.value, tuned=bool(tu.value))

    def tile(self):
        n, c, t = ct.c_int(), ct.c_int(), ct.c_int64()
        check(lib().mdp_noise_tile(self.h, ct.byref(n), ct.byref(c), ct.byref(t)))
        out = dict(fft_n=n.value, cluster=c.value, n_tiles=t.value)
        if n.value:
            out.update(self._plan(0))
        return out

    def tile_fp32(self):
        n, c, t = ct.c_int(), ct.c_int(), ct.c_int64()
        check(lib().mdp_noise_tile_fp32(self.ctx.h, self.h, ct.byref(n), ct.byref(c), ct.byref(t)))
        out = dict(fft_n=n.value, cluster=c.value, n_tiles=t.value)
        if n.value:
            out.update(self._plan(1))
        return out

    def apply(self, vin, vout):
        check(lib().mdp_stbmm(self.ctx.h, self.h, ct.c_void_p(_ptr(vin)), ct.c_void_p(_ptr(vout))), "mdp_stbmm")

    def apply_fp32(self, vin, vout):
        check(lib().mdp_stbmm_fp32(self.ctx.h, self.h, ct.c_void_p(_ptr(vin)), ct.c_void_p(_ptr(vout))),
              "mdp_stbmm_fp32")

    def close(self):
        if self.h:
            lib().mdp_noise_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gls_solve(ctx: Context, A: Pointing, N: Noise, signal, noise, tol=1e-8, maxiter=500, verbose=False, precond=0,
              z_2lvl=0):
    """PCG_GLS_true on device tensors.  Returns (x, lstid, cond, hits, res_rel, info) as torch tensors.

    precond 0: block Jacobi; 1: two-level a priori; 2: two-level a posteriori (Lanczos), with z_2lvl
    deflation columns (0: one)."""
    import torch
    n0 = A.shape()["n_map"]
    x = torch.empty(max(n0, 1), dtype=torch.float64, device="cuda")
    lst = torch.empty(max(n0, 1), dtype=torch.int32, device="cuda")
    cond = torch.empty(max(n0 // 3, 1), dtype=torch.float64, device="cuda")
    hits = torch.empty(max(n0 // 3, 1), dtype=torch.int32, device="cuda")
    res = np.zeros(maxiter + 1)
    prm = SolveParams(tol, maxiter, 1 if verbose else 0, precond, z_2lvl)
    info = SolveInfo()
    check(lib().mdp_gls_solve(ctx.h, A.h, N.h, ct.c_void_p(_ptr(signal)), ct.c_void_p(_ptr(noise)), ct.byref(prm),
                              ct.c_void_p(x.data_ptr()), ct.c_void_p(lst.data_ptr()), ct.c_void_p(cond.data_ptr()),
                              ct.c_void_p(hits.data_ptr()), res.ctypes.data_as(c_f64p), ct.byref(info)),
          "mdp_gls_solve")
    n = info.n_map
    return x[:n], lst[:n], cond[:n // 3], hits[:n // 3], res[:info.iterations + 1], info


def prepare_fp32(ctx: Context, A: Pointing, N: Noise):
    """Builds the FP32 operator state of the mixed-precision solves (FP32 weights, FP32 tile plan and
    spectra) ahead of the solve."""
    check(lib().mdp_prepare_fp32(ctx.h, A.h, N.h), "mdp_prepare_fp32")


def gls_solve_mixed(ctx: Context, A: Pointing, N: Noise, signal, noise, tol=1e-8, maxiter=500, inner_tol=1e-4,
                    inner_maxiter=100, verbose=False, precond=0, z_2lvl=0):
    """Mixed-precision solve (FP32 operator inside FP64 iterative refinement); same outputs as gls_solve.

    precond / z_2lvl as gls_solve: the two-level columns precondition the inner PCGs."""
    import torch
    n0 = A.shape()["n_map"]
    x = torch.empty(max(n0, 1), dtype=torch.float64, device="cuda")
    lst = torch.empty(max(n0, 1), dtype=torch.int32, device="cuda")
    cond = torch.empty(max(n0 // 3, 1), dtype=torch.float64, device="cuda")
    hits = torch.empty(max(n0 // 3, 1), dtype=torch.int32, device="cuda")
    res = np.zeros(maxiter + 1)
    prm = SolveParams(tol, maxiter, 1 if verbose else 0, precond, z_2lvl)
    info = SolveInfo()
    check(lib().mdp_gls_solve_mixed(ctx.h, A.h, N.h, ct.c_void_p(_ptr(signal)), ct.c_void_p(_ptr(noise)),
                                    ct.byref(prm), inner_tol, inner_maxiter, ct.c_void_p(x.data_ptr()),
                                    ct.c_void_p(lst.data_ptr()), ct.c_void_p(cond.data_ptr()),
                                    ct.c_void_p(hits.data_ptr()), res.ctypes.data_as(c_f64p), ct.byref(info)),
          "mdp_gls_solve_mixed")
    n = info.n_map
    return x[:n], lst[:n], cond[:n // 3], hits[:n // 3], res[:info.outer_iterations + 1], info


def gls_solve_ecg(ctx: Context, A: Pointing, N: Noise, signal, noise, tol=1e-8, maxiter=500, enl_fac=4,
                  ortho_alg=1, bs_red=0, verbose=False):
    """ECG_GLS on device tensors: enlarged CG with enl_fac search directions (ortho_alg 1: Orthomin,
    0: Orthodir; bs_red 1: adaptive block size).  Returns (x, lstid, cond, hits, res_rel, info)."""
    import torch
    n0 = A.shape()["n_map"]
    x = torch.empty(max(n0, 1), dtype=torch.float64, device="cuda")
    lst = torch.empty(max(n0, 1), dtype=torch.int32, device="cuda")
    cond = torch.empty(max(n0 // 3, 1), dtype=torch.float64, device="cuda")
    hits = torch.empty(max(n0 // 3, 1), dtype=torch.int32, device="cuda")
    res = np.zeros(maxiter + 1)
    prm = ECGParams(tol, maxiter, enl_fac, ortho_alg, bs_red, 1 if verbose else 0)
    info = SolveInfo()
    check(lib().mdp_ecg_solve(ctx.h, A.h, N.h, ct.c_void_p(_ptr(signal)), ct.c_void_p(_ptr(noise)), ct.byref(prm),
                              ct.c_void_p(x.data_ptr()), ct.c_void_p(lst.data_ptr()), ct.c_void_p(cond.data_ptr()),
                              ct.c_void_p(hits.data_ptr()), res.ctypes.data_as(c_f64p), ct.byref(info)),
          "mdp_ecg_solve")
    n = info.n_map
    return x[:n], lst[:n], cond[:n // 3], hits[:n // 3], res[:info.iterations + 1], info


def gls_solve_multi(ctx: Context, A: Pointing, N: Noise, noise, signal=None, signal_col=-1, tol=1e-8, maxiter=500,
                    inner_tol=1e-4, inner_maxiter=100, slots=0, use_graph=True, verbose=False):
    """Multi-RHS mixed-precision solve of the columns noise[r] (+ signal on column signal_col).

    noise: device tensor [nrhs, m] (float32 or float64, rows contiguous).  Returns (x [nrhs, n_map],
    lstid, cond, hits, per-column info list, MultiInfo)."""
    import torch
    if noise.dim() != 2 or noise.stride(1) != 1:
        raise ValueError("noise must be a [nrhs, m] tensor with contiguous rows")
    nrhs = noise.shape[0]
    n0 = A.shape()["n_map"]
    x = torch.empty((nrhs, max(n0, 1)), dtype=torch.float64, device="cuda")
    lst = torch.empty(max(n0, 1), dtype=torch.int32, device="cuda")
    cond = torch.empty(max(n0 // 3, 1), dtype=torch.float64, device="cuda")
    hits = torch.empty(max(n0 // 3, 1), dtype=torch.int32, device="cuda")
    prm = MultiParams(tol, maxiter, inner_tol, inner_maxiter, slots, 1 if use_graph else 0, 1 if verbose else 0)
    ci = (MultiColInfo * nrhs)()
    info = MultiInfo()
    fp32 = 1 if noise.dtype == torch.float32 else 0
    if not fp32 and noise.dtype != torch.float64:
        raise ValueError("noise must be float32 or float64")
    check(lib().mdp_gls_solve_multi(ctx.h, A.h, N.h, nrhs, ct.c_void_p(noise.data_ptr()), fp32,
                                    noise.stride(0), ct.c_void_p(_ptr(signal) if signal is not None else 0),
                                    signal_col, ct.byref(prm), ct.c_void_p(x.data_ptr()),
                                    ct.c_void_p(lst.data_ptr()), ct.c_void_p(cond.data_ptr()),
                                    ct.c_void_p(hits.data_ptr()), ci, ct.byref(info)), "mdp_gls_solve_multi")
    n = info.n_map
    # the solutions are stored with stride n_map (after the cut)
    xs = x.reshape(-1)[: nrhs * n].reshape(nrhs, n)
    return xs, lst[:n], cond[:n // 3], hits[:n // 3], list(ci), info


def mlmap_host(wl_pix, wl_weights, signal, noise, block_sizes, lam, invtt, nside, tol=1e-8, maxiter=500):
    """MLmap_b200: the MLmap solve from host arrays; returns the I, Q, U, Cond, Hits maps."""
    npix = 12 * nside * nside
    out = [np.zeros(npix) for _ in range(4)] + [np.zeros(npix, dtype=np.int32)]
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32)
    it = ct.c_int()
    rr = ct.c_double()
    pix = np.ascontiguousarray(wl_pix, dtype=np.int32)
    w = np.ascontiguousarray(wl_weights, dtype=np.float64)
    s = np.ascontiguousarray(signal, dtype=np.float64)
    nz = np.ascontiguousarray(noise, dtype=np.float64)
    tt = np.ascontiguousarray(invtt, dtype=np.float64)
    check(lib().MLmap_b200(0, 0, tol, maxiter, nside, len(s), len(bs), bs.ctypes.data_as(c_i32p), 3,
                           pix.ctypes.data_as(c_i32p), w.ctypes.data_as(c_f64p), s.ctypes.data_as(c_f64p),
                           nz.ctypes.data_as(c_f64p), lam, tt.ctypes.data_as(c_f64p),
                           *[o.ctypes.data_as(c_f64p) for o in out[:4]], out[4].ctypes.data_as(c_i32p),
                           ct.byref(it), ct.byref(rr)), "MLmap_b200")
    return tuple(out) + (it.value, rr.value)
