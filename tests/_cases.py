"""Seeded small workloads shared by the parity tests."""
import numpy as np

from midapack_b200 import synth


def with_degenerate_pixels(wl, n_bad=2, seed=0):
    """Gives a few interior pixels a single polarisation angle on all their
    samples: their 3x3 blocks are rank one, so the rcond cut removes them."""
    rng = np.random.default_rng(seed)
    pix = wl.pix.reshape(-1, 3)
    w = wl.weights.reshape(-1, 3).copy()
    p = pix[:, 0] // 3
    observed = np.unique(p[pix[:, 0] >= 0])
    chosen = rng.choice(observed[len(observed) // 4: 3 * len(observed) // 4], size=n_bad, replace=False)
    for b, q in enumerate(chosen):
        rows = (p == q) & (pix[:, 0] >= 0)
        w[rows] = np.array([1.0, np.cos(0.3 * b), np.sin(0.3 * b)])
    wl.weights = w.reshape(-1)
    return wl


def solver_cases():
    return {
        "plain": lambda: synth.small(n_det=2, n_samp=8192, block_len=4096, lam=128, seed=7),
        "gaps": lambda: synth.small(n_det=2, n_samp=4096, block_len=1024, lam=32, gap_frac=0.02, seed=22),
        "cut": lambda: with_degenerate_pixels(synth.small(n_det=2, n_samp=4096, block_len=2048, lam=64, seed=23)),
        "cut_gaps": lambda: with_degenerate_pixels(
            synth.small(n_det=2, n_samp=4096, block_len=2048, lam=64, gap_frac=0.02, seed=24), seed=1),
        "white": lambda: synth.small(n_det=2, n_samp=2048, block_len=1024, lam=1, seed=25),
    }


def noise_golden():
    """Cases of tests/golden/noise2invtt/noise2invtt_ref.npz with their inputs
    (regenerated from the seed, or the reference's own test noise) and the
    reference noise2invtt output."""
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    d = np.load(os.path.join(here, "noise2invtt", "noise2invtt_ref.npz"))
    cases, at = [], 0
    for i, name in enumerate(d["names"]):
        n, lam, fs, fk, seed = (int(d["n"][i]), int(d["lam"][i]), float(d["fsamp"][i]), float(d["fknee"][i]),
                                int(d["seed"][i]))
        if fk == 0.0:
            x = np.load(os.path.join(here, "ref_fixture_rank1_12000.npz"))["noise"][:n].copy()
        else:
            x = synth.noise_tod(n, fk, np.random.default_rng(seed))
        cases.append(dict(name=str(name), n=n, lam=lam, fsamp=fs, apod=str(d["apod"][i]), noise=x,
                          invtt=d["invtt"][at:at + lam]))
        at += lam
    return cases
