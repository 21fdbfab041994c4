"""Generates the golden fixtures in this directory.

Inputs come from the reference's own test data
(mappraiser/test/data_bin/*_1.bin: int32 pixels 3p+k at HEALPix nside 512,
(1, cos, sin) weights, signal, noise, 8192-tap invtt rows), cut to the first
12000 samples of rank 1 as one stationary block, plus one small seeded
synthetic workload with flagged samples and rank-deficient pixels.  Outputs
come from running the reference's own compiled C operators (oracle/_ref,
built by oracle/build_ref.sh): MatInit's local indices and lindices,
MatVecProd, TrMatVecProd, stbmmProd on seeded vectors, and the single-rank
MLmap solve (PCG_GLS_true, block Jacobi).

    python tests/golden/make_golden.py [/root/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402


def golden_from(name, pix, w, sig, noi, block_sizes, lam, invtt, tol, maxiter, seed):
    m = len(sig)
    rng = np.random.default_rng(seed)
    loc, lind, trash = ref.local_shape(pix, m, 3)
    n = len(lind) - 3 * trash
    x = rng.standard_normal(n)
    y = ref.matvec(pix, w, x, m)
    t = rng.standard_normal(m)
    xt = ref.trmatvec(pix, w, t, m, n)
    v = rng.standard_normal(m)
    nv = ref.stbmm(v, block_sizes, lam, invtt)
    xs, lst, cond, hits, res = ref.pcg(pix, w, sig, noi, block_sizes, lam, invtt, tol=tol, maxiter=maxiter)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), pix=pix, weights=w, signal=sig, noise=noi,
                        block_sizes=np.asarray(block_sizes, np.int32), lam=lam, invtt=invtt, tol=tol,
                        maxiter=maxiter, local=loc, lindices=lind, trash=trash, x_in=x, Px=y, t_in=t, Ptt=xt,
                        v_in=v, Nv=nv, x_sol=xs, lstid=lst, cond=cond, hits=hits, res_rel=res)
    print(name, "m", m, "n", n, "iterations", len(res) - 1)


def main(refroot="/root/reference"):
    d = os.path.join(refroot, "mappraiser", "test", "data_bin")
    ms = 12000
    pix = np.fromfile(os.path.join(d, "pixels_1.bin"), dtype=np.int32)[:3 * ms]
    w = np.fromfile(os.path.join(d, "pixweights_1.bin"), dtype=np.float64)[:3 * ms]
    sig = np.fromfile(os.path.join(d, "signal_1.bin"), dtype=np.float64)[:ms]
    noi = np.fromfile(os.path.join(d, "noise_1.bin"), dtype=np.float64)[:ms]
    lam = 8192
    invtt = np.fromfile(os.path.join(d, "invtt_1.bin"), dtype=np.float64)[:lam]
    golden_from("ref_fixture_rank1_12000", pix, w, sig, noi, [ms], lam, invtt, 1e-10, 500, 1)

    from midapack_b200 import synth
    from tests._cases import with_degenerate_pixels
    wl = with_degenerate_pixels(synth.small(n_det=2, n_samp=2048, block_len=1024, lam=48, seed=41), seed=2)
    golden_from("synthetic_cut_4096", wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt,
                1e-10, 400, 2)
    wl = synth.small(n_det=2, n_samp=2048, block_len=1024, lam=48, gap_frac=0.03, seed=42)
    golden_from("synthetic_gaps_4096", wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt,
                1e-10, 400, 3)


if __name__ == "__main__":
    main(*sys.argv[1:])
