"""Seeded small workloads shared by the parity tests."""
import numpy as np

from midapack_b200 import synth


def with_degenerate_pixels(wl, n_bad=2, hits=3, seed=0):
    """Points a few samples at new pixels with one fixed angle: their 3x3 blocks are
    rank one, so the rcond cut removes them."""
    rng = np.random.default_rng(seed)
    pix = wl.pix.reshape(-1, 3).copy()
    w = wl.weights.reshape(-1, 3).copy()
    valid = np.nonzero(pix[:, 0] >= 0)[0]
    base = int(pix[valid, 0].max()) // 3 + 10
    for b in range(n_bad):
        rows = rng.choice(valid, size=hits, replace=False)
        p = base + 7 * b
        pix[rows] = 3 * p + np.arange(3)
        w[rows] = np.array([1.0, np.cos(0.3 * b), np.sin(0.3 * b)])
        valid = np.setdiff1d(valid, rows)
    wl.pix = pix.reshape(-1).astype(np.int32)
    wl.weights = w.reshape(-1)
    return wl


def solver_cases():
    return {
        "plain": lambda: synth.small(n_det=2, n_samp=4096, block_len=2048, lam=64, seed=21),
        "gaps": lambda: synth.small(n_det=2, n_samp=4096, block_len=1024, lam=32, gap_frac=0.02, seed=22),
        "cut": lambda: with_degenerate_pixels(synth.small(n_det=2, n_samp=4096, block_len=2048, lam=64, seed=23)),
        "cut_gaps": lambda: with_degenerate_pixels(
            synth.small(n_det=2, n_samp=4096, block_len=2048, lam=64, gap_frac=0.02, seed=24), seed=1),
        "white": lambda: synth.small(n_det=2, n_samp=2048, block_len=1024, lam=1, seed=25),
    }
