"""First rows of the inverse-noise Toeplitz blocks, estimated on the device.

Mirrors MAPPRAISER's TOAST-side helpers ``noise2invtt`` and ``compute_invtt``
(mappraiser/python/TOAST_interface/utils.py:500-602 and 439-481): same names,
arguments, output layout and errors.  Per block of n noise samples:

* periodogram ``scipy.signal.welch(x, fsamp, window='hann', nperseg=n,
  detrend='linear')`` (one segment);
* fit of ``a + log10(1 + ((f + fmin)/fknee)**alpha)`` to ``log10(psd[1:])``
  under the bounds ``[-20, -10, 0, 0] .. [0, 0, 20, 1]`` from
  ``(-7, -1, 0.1, 1e-6)``;
* ``irfft`` of the inverse PSD ``10**-a / (1 + ((f + fmin)/fknee)**alpha)`` on
  the block's rfft grid, times the apodisation window (``chebwin`` at 150 dB or
  ``gaussian``) of ``2*Lambda`` points after ``ifftshift``, first ``Lambda``.

All of it runs in ``libmidapack_b200.so`` (``mdp_noise2invtt``); this module
moves arrays and checks arguments.  The reference's ``curve_fit`` (trust region
reflective, ``ftol = 1e-8``) stops short of the least-squares minimum that the
device fit converges to; the two invtt rows differ by the reference's own fit
tolerance (relative 1e-5 at most on the seeded cases), and agree to 1e-7 with
``curve_fit`` run to ``ftol = xtol = gtol = 1e-15``.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import MDP_ENOCONV, Context, MidapackError, _ptr, c_f64p, c_i32p, check, lib

APOD = {"chebwin": 0, "gaussian": 1}
_default_ctx = None


def _ctx(ctx):
    global _default_ctx
    if ctx is not None:
        return ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _plain_fsamp(fsamp) -> float:
    # remove the unit of an astropy quantity, as utils.py:514-518 does
    try:
        f_unit = fsamp.unit
        fsamp = float(fsamp / (1.0 * f_unit))
    except AttributeError:
        pass
    return float(fsamp)


def _apod_code(apod_window_type: str) -> int:
    if apod_window_type not in APOD:
        raise RuntimeError(f"Apodisation window '{apod_window_type}' is not supported.")
    return APOD[apod_window_type]


def _device_f64(x):
    import torch
    if isinstance(x, torch.Tensor):
        if not x.is_cuda:
            x = x.cuda()
        return x.to(torch.float64).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def invtt_blocks(noise, block_sizes, Lambda: int, fsamp, apod_window_type: str = "chebwin", ctx: Context | None = None,
                 return_fit: bool = False):
    """noise2invtt of consecutive blocks of ``noise`` (host array or CUDA tensor).

    Returns a CUDA float64 tensor of ``len(block_sizes) * Lambda`` values (block b
    at ``b*Lambda``); with ``return_fit`` also the fitted ``(a, alpha, fknee, fmin)``
    per block and the model evaluations each fit used.
    """
    import torch
    fsamp = _plain_fsamp(fsamp)
    code = _apod_code(apod_window_type)
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32).ravel()
    if bs.size == 0:
        raise ValueError("no blocks")
    if Lambda > int(bs.min()) // 2:
        raise RuntimeError("Bandwidth cannot be larger than timestream.")
    need = int(bs.astype(np.int64).sum())
    if len(noise) < need:
        raise ValueError(f"noise has {len(noise)} samples, the blocks need {need}")
    ctx = _ctx(ctx)
    d_noise = _device_f64(noise)
    out = torch.empty(bs.size * Lambda, dtype=torch.float64, device=d_noise.device)
    params = np.zeros((bs.size, 4))
    evals = np.zeros(bs.size, dtype=np.int32)
    rc = lib().mdp_noise2invtt(ctx.h, int(bs.size), bs.ctypes.data_as(c_i32p), ct.c_void_p(_ptr(d_noise)),
                               int(Lambda), fsamp, code, ct.c_void_p(_ptr(out)), params.ctypes.data_as(c_f64p),
                               evals.ctypes.data_as(c_i32p))
    if rc == MDP_ENOCONV:
        # curve_fit's own error when maxfev is reached
        raise RuntimeError("Optimal parameters not found: " + lib().mdp_last_error().decode())
    check(rc, "mdp_noise2invtt")
    if return_fit:
        return out, params, evals
    return out


def periodogram(noise, block_sizes, fsamp, ctx: Context | None = None):
    """One-segment Welch periodogram of every block: a CUDA tensor of
    ``sum(n // 2 + 1)`` values, block after block."""
    import torch
    fsamp = _plain_fsamp(fsamp)
    bs = np.ascontiguousarray(block_sizes, dtype=np.int32).ravel()
    ctx = _ctx(ctx)
    d_noise = _device_f64(noise)
    out = torch.empty(int((bs.astype(np.int64) // 2 + 1).sum()), dtype=torch.float64, device=d_noise.device)
    check(lib().mdp_periodogram(ctx.h, int(bs.size), bs.ctypes.data_as(c_i32p), ct.c_void_p(_ptr(d_noise)), fsamp,
                                ct.c_void_p(_ptr(out))), "mdp_periodogram")
    return out


def apod_window(Lambda: int, apod_window_type: str = "chebwin", ctx: Context | None = None):
    """The apodisation window after ifftshift, first ``Lambda`` points (CUDA tensor)."""
    import torch
    code = _apod_code(apod_window_type)
    ctx = _ctx(ctx)
    out = torch.empty(int(Lambda), dtype=torch.float64, device="cuda")
    check(lib().mdp_apod_window(ctx.h, int(Lambda), code, ct.c_void_p(_ptr(out))), "mdp_apod_window")
    return out


def noise2invtt(nsetod, nn, Lambda, fsamp, idet, invtt_dtype, apod_window_type, verbose=False, save_psd=False,
                save_dir=None, ctx: Context | None = None):
    """utils.py:500-602 for one block: returns the first ``Lambda`` values of the
    block's inverse-noise row as ``invtt_dtype`` (a host array)."""
    if save_psd:
        raise NotImplementedError("save_psd writes diagnostic files; not provided by this library")
    if len(nsetod) != nn:
        raise NotImplementedError("only the one-segment periodogram (len(nsetod) == nn) is provided")
    if Lambda > nn // 2:
        raise RuntimeError("Bandwidth cannot be larger than timestream.")
    out, params, evals = invtt_blocks(nsetod, [nn], Lambda, fsamp, apod_window_type, ctx=ctx, return_fit=True)
    if verbose:
        print("\n[det " + str(idet) + "]: PSD fit log(sigma2) = %1.2f, alpha = %1.2f, fknee = %1.2f, fmin = %1.2e\n"
              % tuple(params[0]), flush=True)
    return out.cpu().numpy().astype(invtt_dtype)


def compute_invtt(nobs, ndet, mappraiser_noise, local_block_sizes, Lambda, fsamp, buffer, invtt_dtype,
                  print_info=False, save_psd=False, save_dir=None, apod_window_type="chebwin",
                  ctx: Context | None = None):
    """utils.py:439-481: the first ``Lambda`` values of every block's inverse-noise
    row written into ``buffer`` at ``(iobs*ndet + idet)*Lambda``; the blocks are
    consecutive in ``mappraiser_noise`` in that order.  Returns None."""
    if save_psd:
        raise NotImplementedError("save_psd writes diagnostic files; not provided by this library")
    nb = nobs * ndet
    bs = np.asarray(local_block_sizes)[:nb]
    out, params, evals = invtt_blocks(mappraiser_noise, bs, Lambda, fsamp, apod_window_type, ctx=ctx, return_fit=True)
    if print_info:
        print("\n[det 0]: PSD fit log(sigma2) = %1.2f, alpha = %1.2f, fknee = %1.2f, fmin = %1.2e\n"
              % tuple(params[0]), flush=True)
    buffer[:nb * Lambda] = out.cpu().numpy().astype(invtt_dtype)
    return None


__all__ = ["APOD", "invtt_blocks", "periodogram", "apod_window", "noise2invtt", "compute_invtt", "MidapackError"]
