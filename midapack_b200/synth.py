"""Seeded synthetic map-making workloads.

No public dataset is involved in this path; every workload is generated here
from a seed, following the staging conventions of MAPPRAISER's TOAST interface:

* pixel index of sample t, Stokes k:  ``3*p + k`` (``mappraiser.py:1214-1216``),
  flagged samples get pixel -1, i.e. indices -3, -2, -1 (``utils.py:150-154``);
* pointing weights ``(1, cos 2psi, sin 2psi)``;
* the first row of each Toeplitz block follows ``noise2invtt``
  (``mappraiser/python/TOAST_interface/utils.py:500-602``): the inverse PSD on
  the block's rfft grid, ``irfft``, a ``chebwin(2*lambda, at=150)`` window,
  ``ifftshift``, keep the first ``lambda`` taps.  The PSD is known (no fit):
  ``sigma^2 * (1 + f_knee / (f + f_min))`` with f_min = 1e-5 Hz (the reference
  model ``psd_model`` with alpha = -1).

Scan: detector d sweeps the rows of a W x H flat grid back and forth in
W-sample runs (even runs left to right, odd runs right to left), starting at a
seeded random row/column offset; psi = detector angle (0/45/90/135 deg by
d mod 4) + 2*pi*f_hwp*t (half-wave plate at 2 Hz).  Sky: Gaussian I, Q, U with
sigma (100, 1, 1).  Noise: white sigma = 1 plus 1/f, made by filtering seeded
white noise with sqrt(PSD) per detector.  d = P m_true + n, returned as
``signal`` (= P m_true) and ``noise`` (= n), the split MLmap takes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

F_MIN = 1e-5
FS = 100.0
F_HWP = 2.0


@dataclass
class Workload:
    """One map-making problem in the reference's MLmap argument layout."""

    name: str
    width: int
    height: int
    n_det: int
    n_samp: int            # samples per detector
    block_len: int         # samples per stationary interval (one Toeplitz block)
    lam: int               # Toeplitz half bandwidth (taps)
    fknee: float
    seed: int
    gap_frac: float = 0.0
    pix: np.ndarray = field(default=None, repr=False)       # int32 [3*Ns]
    weights: np.ndarray = field(default=None, repr=False)   # f64 [3*Ns]
    signal: np.ndarray = field(default=None, repr=False)    # f64 [Ns]
    noise: np.ndarray = field(default=None, repr=False)     # f64 [Ns]
    invtt: np.ndarray = field(default=None, repr=False)     # f64 [n_blocks*lam]
    block_sizes: np.ndarray = field(default=None, repr=False)  # int32 [n_blocks]
    sky: np.ndarray = field(default=None, repr=False)       # f64 [npix, 3]

    @property
    def n_samples(self) -> int:
        return self.n_det * self.n_samp

    @property
    def npix(self) -> int:
        return self.width * self.height

    @property
    def nside(self) -> int:
        """HEALPix nside with 12*nside^2 == W*H (the flat grids are sized so)."""
        ns = int(round((self.npix / 12) ** 0.5))
        return ns if 12 * ns * ns == self.npix else 0


def psd(f: np.ndarray, fknee: float, sigma: float = 1.0) -> np.ndarray:
    return sigma ** 2 * (1.0 + fknee / (f + F_MIN))


def invtt_row(n_block: int, lam: int, fknee: float, sigma: float = 1.0) -> np.ndarray:
    """First row of the inverse-noise Toeplitz block (noise2invtt recipe, known PSD)."""
    from scipy.signal import get_window

    if lam > n_block // 2:
        raise ValueError("Bandwidth cannot be larger than timestream.")
    f = np.fft.rfftfreq(n_block, 1.0 / FS)
    inv_tt = np.fft.irfft(1.0 / psd(f, fknee, sigma), n=n_block)
    win = np.fft.ifftshift(get_window(("chebwin", 150), 2 * lam))[:lam]
    return np.multiply(win, inv_tt[:lam], dtype=np.float64)


def scan_pixels(width: int, height: int, n_det: int, n_samp: int, rng: np.random.Generator) -> np.ndarray:
    """Pixel id per sample, detector-major [n_det, n_samp] (int64)."""
    t = np.arange(n_samp, dtype=np.int64)
    run = t // width
    u = t % width
    out = np.empty((n_det, n_samp), dtype=np.int64)
    for d in range(n_det):
        r0 = int(rng.integers(0, height))
        c0 = int(rng.integers(0, width))
        col = np.where(run % 2 == 0, u, width - 1 - u)
        col = (col + c0) % width
        row = (run + r0) % height
        out[d] = row * width + col
    return out


def psi_angles(n_det: int, n_samp: int) -> np.ndarray:
    t = np.arange(n_samp, dtype=np.float64) / FS
    out = np.empty((n_det, n_samp))
    for d in range(n_det):
        out[d] = np.deg2rad(45.0 * (d % 4)) + 2.0 * np.pi * F_HWP * t
    return out


def noise_tod(n_samp: int, fknee: float, rng: np.random.Generator, sigma: float = 1.0) -> np.ndarray:
    w = rng.standard_normal(n_samp)
    f = np.fft.rfftfreq(n_samp, 1.0 / FS)
    return np.fft.irfft(np.fft.rfft(w) * np.sqrt(psd(f, fknee, sigma)), n=n_samp)


def make_workload(name: str, width: int, height: int, n_det: int, n_samp: int, block_len: int, lam: int,
                  fknee: float = 1.0, seed: int = 20261203, gap_frac: float = 0.0) -> Workload:
    """Builds the arrays MLmap takes (host, numpy). Intended for up to ~1e8 samples."""
    wl = Workload(name, width, height, n_det, n_samp, block_len, lam, fknee, seed, gap_frac)
    rng = np.random.default_rng(seed)
    pixd = scan_pixels(width, height, n_det, n_samp, rng)
    psi = psi_angles(n_det, n_samp)
    sky = np.empty((width * height, 3))
    sky[:, 0] = 100.0 * rng.standard_normal(width * height)
    sky[:, 1] = rng.standard_normal(width * height)
    sky[:, 2] = rng.standard_normal(width * height)
    ns = n_det * n_samp
    p = pixd.reshape(-1)
    w = np.empty((ns, 3))
    w[:, 0] = 1.0
    w[:, 1] = np.cos(2.0 * psi.reshape(-1))
    w[:, 2] = np.sin(2.0 * psi.reshape(-1))
    signal = (w * sky[p]).sum(axis=1)
    noise = np.concatenate([noise_tod(n_samp, fknee, rng) for _ in range(n_det)])
    if gap_frac > 0:
        flagged = rng.random(ns) < gap_frac
        p = np.where(flagged, -1, p)
    idx = (3 * p[:, None] + np.arange(3)[None, :]).astype(np.int32).reshape(-1)
    if n_samp % block_len != 0:
        raise ValueError("block_len must divide n_samp")
    nb = ns // block_len
    row = invtt_row(block_len, lam, fknee)
    wl.pix = idx
    wl.weights = w.reshape(-1)
    wl.signal = signal
    wl.noise = noise
    wl.invtt = np.tile(row, nb)
    wl.block_sizes = np.full(nb, block_len, dtype=np.int32)
    wl.sky = sky
    return wl


def make_pointing(width: int, height: int, n_det: int, n_samp: int, block_len: int, lam: int, fknee: float = 1.0,
                  seed: int = 20261203, gap_frac: float = 0.0, **_unused):
    """Pointing and noise model of the first ``n_det`` detectors of a workload,
    without its TOD: (pix int32 [3Ns], weights f64 [3Ns], block_sizes int32,
    invtt f64 [n_blocks*lam]).  Same scan, angles, flags and Toeplitz rows as
    make_workload, from its own seeded stream (host, numpy; for timing an
    operator on a sample of a large workload)."""
    rng = np.random.default_rng(seed)
    ns = n_det * n_samp
    p = scan_pixels(width, height, n_det, n_samp, rng).reshape(-1)
    if gap_frac > 0:
        p = np.where(rng.random(ns) < gap_frac, -1, p)
    idx = np.empty((ns, 3), dtype=np.int32)
    idx[:] = (3 * p).astype(np.int32)[:, None]
    del p
    idx += np.arange(3, dtype=np.int32)[None, :]
    w = np.empty((ns, 3))
    w[:, 0] = 1.0
    two_psi = 2.0 * psi_angles(n_det, n_samp).reshape(-1)
    w[:, 1] = np.cos(two_psi)
    w[:, 2] = np.sin(two_psi)
    del two_psi
    if n_samp % block_len != 0:
        raise ValueError("block_len must divide n_samp")
    nb = ns // block_len
    return idx.reshape(-1), w.reshape(-1), np.full(nb, block_len, dtype=np.int32), np.tile(
        invtt_row(block_len, lam, fknee), nb)


def mc_noise(n_det: int, n_samp: int, nrhs: int, fknee: float = 1.0, seed: int = 0) -> np.ndarray:
    """Monte-Carlo noise realisations with the workload's PSD: [nrhs, n_det*n_samp]
    float32 (the columns of a multi-RHS solve; FP32 values are exact inputs)."""
    rng = np.random.default_rng(seed)
    out = np.empty((nrhs, n_det * n_samp), dtype=np.float32)
    for r in range(nrhs):
        out[r] = np.concatenate([noise_tod(n_samp, fknee, rng) for _ in range(n_det)]).astype(np.float32)
    return out


def mc_noise_torch(n_det: int, n_samp: int, nrhs: int, fknee: float = 1.0, seed: int = 0, device: str = "cuda"):
    """Device version of mc_noise for large workloads: [nrhs, n_det*n_samp] float32."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((nrhs, n_det * n_samp), dtype=torch.float32, device=device)
    f = torch.fft.rfftfreq(n_samp, 1.0 / FS, dtype=torch.float32, device=device)
    amp = torch.sqrt(1.0 + fknee / (f + F_MIN))
    for r in range(nrhs):
        white = torch.randn((n_det, n_samp), dtype=torch.float32, device=device, generator=g)
        out[r] = torch.fft.irfft(torch.fft.rfft(white, dim=1) * amp, n=n_samp, dim=1).reshape(-1)
    return out


# Configurations of the reference workload family, by sizes.
CONFIGS = {
    # plain FP64 PCG, CPU-runnable: 256x192 grid, 4 det x 2^20, lambda 2^12, one block per det
    "c1_4det_2p20_256x192_lam4096": dict(width=256, height=192, n_det=4, n_samp=1 << 20, block_len=1 << 20,
                                         lam=1 << 12, fknee=1.0, seed=20261204),
    # FP64 at scale: 2048x1536 grid, 64 det x 2^24, 2^20-sample intervals, lambda 2^14, 1% gaps
    "c2_64det_2p24_2048x1536_lam16384": dict(width=2048, height=1536, n_det=64, n_samp=1 << 24,
                                             block_len=1 << 20, lam=1 << 14, fknee=1.0, seed=20261205,
                                             gap_frac=0.01),
    # multi-RHS: 1024x768 grid, 16 det x 2^23, lambda 2^13, 1% flagged samples as at scale (without flags
    # P^T N^-1 P is singular: a constant offset is in its null space, and noise-only columns stall above 1e-8)
    "c4_16det_2p23_1024x768_lam8192": dict(width=1024, height=768, n_det=16, n_samp=1 << 23,
                                           block_len=1 << 23, lam=1 << 13, fknee=1.0, seed=20261207,
                                           gap_frac=0.01),
}


def small(name: str = "small", width: int = 32, height: int = 24, n_det: int = 2, n_samp: int = 4096,
          block_len: int = 2048, lam: int = 64, fknee: float = 1.0, seed: int = 7, gap_frac: float = 0.0
          ) -> Workload:
    return make_workload(name, width, height, n_det, n_samp, block_len, lam, fknee, seed, gap_frac)


def make_workload_torch(name: str, width: int, height: int, n_det: int, n_samp: int, block_len: int, lam: int,
                        fknee: float = 1.0, seed: int = 20261203, gap_frac: float = 0.0, device: str = "cuda"):
    """Same generator as make_workload, run on the GPU with torch for the
    ~1e9-sample workloads (its own seeded streams, so values differ from the
    numpy version).  Returns a Workload whose arrays are device tensors
    (pix int32 [3Ns], weights/signal/noise float64) plus numpy block_sizes/invtt."""
    import torch

    wl = Workload(name, width, height, n_det, n_samp, block_len, lam, fknee, seed, gap_frac)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    ns = n_det * n_samp
    npix = width * height
    sky = torch.empty((npix, 3), dtype=torch.float64, device=device)
    sky.normal_(generator=g)
    sky[:, 0] *= 100.0
    pix = torch.empty(3 * ns, dtype=torch.int32, device=device)
    w = torch.empty(3 * ns, dtype=torch.float64, device=device)
    signal = torch.empty(ns, dtype=torch.float64, device=device)
    noise = torch.empty(ns, dtype=torch.float64, device=device)
    t = torch.arange(n_samp, device=device, dtype=torch.int64)
    run = t // width
    u = t % width
    tsec = t.to(torch.float64) / FS
    f = torch.fft.rfftfreq(n_samp, 1.0 / FS, dtype=torch.float64, device=device)
    amp = torch.sqrt(1.0 + fknee / (f + F_MIN))
    offs = torch.randint(0, 1 << 30, (n_det, 2), generator=g, device=device)
    k3 = torch.arange(3, device=device, dtype=torch.int32)
    for d in range(n_det):
        r0 = int(offs[d, 0]) % height
        c0 = int(offs[d, 1]) % width
        col = torch.where(run % 2 == 0, u, width - 1 - u)
        col = (col + c0) % width
        row = (run + r0) % height
        p = (row * width + col)
        psi = math.radians(45.0 * (d % 4)) + 2.0 * math.pi * F_HWP * tsec
        sl = slice(3 * d * n_samp, 3 * (d + 1) * n_samp)
        wd = w[sl].view(n_samp, 3)
        wd[:, 0] = 1.0
        wd[:, 1] = torch.cos(2.0 * psi)
        wd[:, 2] = torch.sin(2.0 * psi)
        signal[d * n_samp:(d + 1) * n_samp] = (wd * sky[p]).sum(dim=1)
        white = torch.randn(n_samp, dtype=torch.float64, device=device, generator=g)
        noise[d * n_samp:(d + 1) * n_samp] = torch.fft.irfft(torch.fft.rfft(white) * amp, n=n_samp)
        if gap_frac > 0:
            flagged = torch.rand(n_samp, device=device, generator=g, dtype=torch.float64) < gap_frac
            p = torch.where(flagged, torch.full_like(p, -1), p)
        pix[sl].view(n_samp, 3).copy_((3 * p.to(torch.int32))[:, None] + k3[None, :])
        del p, psi, col, row
    if n_samp % block_len != 0:
        raise ValueError("block_len must divide n_samp")
    nb = ns // block_len
    row_t = invtt_row(block_len, lam, fknee)
    wl.pix, wl.weights, wl.signal, wl.noise = pix, w, signal, noise
    wl.invtt = np.tile(row_t, nb)
    wl.block_sizes = np.full(nb, block_len, dtype=np.int32)
    wl.sky = sky
    return wl
