"""Generates noise2invtt_ref.npz: golden outputs of the reference's own noise2invtt.

The reference function (mappraiser/python/TOAST_interface/utils.py:484-602:
psd_model, logpsd_model, inversepsd_model, noise2invtt) is read from the
reference tree and executed unmodified with numpy/scipy; its module imports
toast and astropy, which are not installed, so only those function definitions
are taken from the file.  Inputs: the noise stream of the reference's own test
data (mappraiser/test/data_bin, rank 1, first 12000 samples, as stored in
../ref_fixture_rank1_12000.npz; its sampling rate is not recorded there, 100 Hz
is assumed) and seeded synthetic 1/f noise (midapack_b200.synth.noise_tod,
regenerated by the tests from the seed).

    python tests/golden/noise2invtt/make.py [/root/reference]
"""
import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

from midapack_b200 import synth  # noqa: E402

# name, n, lambda, fsamp, fknee (synthetic; 0 = reference data), seed, window
CASES = [
    ("ref_rank1_noise", 12000, 2048, 100.0, 0.0, 0, "chebwin"),
    ("pow2_4096", 4096, 256, 100.0, 1.0, 11, "chebwin"),
    ("ragged_6000", 6000, 512, 100.0, 0.5, 12, "chebwin"),
    ("pow2_16384_gauss", 16384, 1024, 100.0, 2.0, 13, "gaussian"),
    ("prime_10007", 10007, 128, 37.0, 1.0, 14, "chebwin"),
    ("split_65536", 65536, 4096, 100.0, 0.1, 15, "chebwin"),
    ("short_1000_gauss", 1000, 8, 100.0, 5.0, 16, "gaussian"),
]


def case_noise(n, fknee, seed):
    if fknee == 0.0:
        return np.load(os.path.join(os.path.dirname(HERE), "ref_fixture_rank1_12000.npz"))["noise"][:n].copy()
    return synth.noise_tod(n, fknee, np.random.default_rng(seed))


def reference_functions(ref_root):
    import scipy.signal
    from scipy.optimize import curve_fit
    path = os.path.join(ref_root, "mappraiser", "python", "TOAST_interface", "utils.py")
    tree = ast.parse(open(path).read())
    keep = {"psd_model", "logpsd_model", "inversepsd_model", "noise2invtt"}
    mod = ast.Module(body=[n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in keep],
                     type_ignores=[])
    ns = {"np": np, "scipy": scipy, "curve_fit": curve_fit, "os": os}
    exec(compile(mod, path, "exec"), ns)
    return ns


def main(ref_root):
    ns = reference_functions(ref_root)
    out = {"names": np.array([c[0] for c in CASES])}
    cols = ["n", "lam", "fsamp", "fknee", "seed"]
    for i, c in enumerate(cols):
        out[c] = np.array([case[i + 1] for case in CASES])
    out["apod"] = np.array([case[6] for case in CASES])
    rows = []
    for name, n, lam, fs, fknee, seed, apod in CASES:
        x = case_noise(n, fknee, seed)
        rows.append(ns["noise2invtt"](x, n, lam, fs, 0, np.float64, apod))
    out["invtt"] = np.concatenate(rows)
    np.savez(os.path.join(HERE, "noise2invtt_ref.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
