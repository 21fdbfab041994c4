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


def template_case(seed=31, lengths=(4096, 3072), ndet=2, npoly=2, ground=1, n_sss_bins=8, nhwp=2, delta_t=5.0):
    """A small MTmap workload: nces CESs (one per entry of `lengths`) x ndet detectors
    on a 64 x 48 flat grid (12 * 16^2 pixels, nside 16), sweeps of 400-700 samples with
    the boresight going back and forth in azimuth, a HWP at 2 Hz; data = sky + white
    noise + a polynomial drift per sweep, a ground pattern in azimuth and HWP
    harmonics.  Returns (scan, pix, weights, signal, noise, invtt, nside)."""
    from oracle.restate import TemplateScan
    rng = np.random.default_rng(seed)
    fs = synth.FS
    sweeps, az, hwp = [], [], []
    for L in lengths:
        st = [0]
        while st[-1] < L:
            st.append(min(L, st[-1] + int(rng.integers(400, 700))))
        if st[-1] - st[-2] < 100:     # no runt sweep at the end
            st.pop(-2)
        sweeps.append(np.array(st, dtype=np.int32))
        a = np.empty(L)
        for s in range(len(st) - 1):
            u = (np.arange(st[s], st[s + 1]) - st[s]) / max(st[s + 1] - st[s] - 1, 1)
            a[st[s]:st[s + 1]] = 10.0 + 20.0 * (u if s % 2 == 0 else 1.0 - u)
        az.append(a)
        hwp.append(2 * np.pi * 2.0 * np.arange(L) / fs)
    sc = TemplateScan(sweeps, az, np.full(len(lengths), 10.0), np.full(len(lengths), 30.0), hwp, ndet, npoly,
                      ground, n_sss_bins, nhwp, delta_t, fs)
    W, H, nside = 64, 48, 16
    sky = rng.standard_normal((W * H, 3)) * np.array([100.0, 1.0, 1.0])
    pix, wts, sig, noi = [], [], [], []
    for i, L in enumerate(lengths):
        p = synth.scan_pixels(W, H, ndet, L, rng)
        psi = synth.psi_angles(ndet, L)
        for j in range(ndet):
            idx = np.stack([3 * p[j], 3 * p[j] + 1, 3 * p[j] + 2], 1).ravel()
            w = np.stack([np.ones(L), np.cos(2 * psi[j]), np.sin(2 * psi[j])], 1)
            pix.append(idx)
            wts.append(w.ravel())
            sig.append((w * sky[p[j]]).sum(1))
            drift = np.zeros(L)
            for s in range(len(sweeps[i]) - 1):
                r = np.arange(sweeps[i][s], sweeps[i][s + 1])
                drift[r] = rng.normal(0, 3.0) + rng.normal(0, 1.0) * (r - r.mean()) / len(r)
            ground_sig = 2.0 * np.sin(az[i] / 3.0)
            hwpss = 0.5 * np.cos(hwp[i]) + 0.2 * np.sin(2 * hwp[i])
            noi.append(rng.standard_normal(L) + drift + ground_sig + hwpss)
    invtt = 1.0 / (1.0 + 0.1 * np.arange(len(lengths) * ndet))
    return (sc, np.concatenate(pix).astype(np.int32), np.concatenate(wts), np.concatenate(sig),
            np.concatenate(noi), invtt, nside)
