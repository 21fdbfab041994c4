"""Times the reference's own C operator P^T N^-1 P (oracle/_ref) on host cores.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg runs this as a
separate process (a fresh interpreter that never touched CUDA, since the
oracle forks one process per rank).

    python -m oracle.cpu_baseline SAMPLE.npz RANKS   -> prints seconds per application (JSON)
    python -m oracle.cpu_baseline --mlmap CASE.npz RANKS OUT.npz
        -> runs the reference's whole MLmap (RANKS forked ranks, detectors split
           evenly), prints its wall time and iterations (JSON), saves its maps

operator_sample() and mlmap_workload() do the same in the calling process for a
caller that has not initialised CUDA (the reference arm of bench.py).
"""
import json
import sys

import numpy as np

from oracle import ref


def main(path, ranks):
    d = np.load(path)
    ranks = int(ranks)
    per = int(d["per_det"])
    nbp = int(d["nb_per_det"])
    t = ref.operator_time(ranks, [per] * ranks, [nbp] * ranks, d["block_sizes"][:nbp * ranks], d["pix"], d["weights"],
                          int(d["lam"]), d["invtt"][:nbp * ranks * int(d["lam"])], reps=1)
    print(json.dumps({"seconds_per_application": t, "ranks": ranks}))


def mlmap(path, ranks, out):
    import time
    d = np.load(path)
    ranks = int(ranks)
    m = int(d["signal"].size)
    nb = int(d["block_sizes"].size)
    if m % ranks or nb % ranks:
        raise SystemExit("samples and blocks must split evenly over the ranks")
    t0 = time.perf_counter()
    maps = ref.mlmap(ranks, [m // ranks] * ranks, [nb // ranks] * ranks, d["block_sizes"], d["pix"], d["weights"],
                     d["signal"], d["noise"], int(d["lam"]), d["invtt"], int(d["nside"]), tol=float(d["tol"]),
                     maxiter=int(d["maxiter"]))
    t = time.perf_counter() - t0
    np.savez(out, I=maps[0], Q=maps[1], U=maps[2], Cond=maps[3], Hits=maps[4], res=maps[5])
    print(json.dumps({"seconds": t, "ranks": ranks, "iterations": int(len(maps[5]) - 1)}))


def operator_sample(cfg: dict, ranks: int, reps: int):
    """The reference's P^T N^-1 P on the first `ranks` detectors of the workload
    `cfg` (a synth configuration; one detector per forked rank, pointing and
    Toeplitz rows from synth.make_pointing): seconds of each of `reps`
    applications, max over ranks."""
    from midapack_b200 import synth
    cfg = dict(cfg, n_det=ranks)
    pix, w, bs, invtt = synth.make_pointing(**cfg)
    per = int(cfg["n_samp"])
    nbp = per // int(cfg["block_len"])
    return ref.operator_time(ranks, [per] * ranks, [nbp] * ranks, bs, pix, w, int(cfg["lam"]), invtt, reps=reps,
                             each=True)


def mlmap_workload(wl, ranks: int, tol: float, maxiter: int):
    """The reference's whole MLmap on `ranks` forked ranks for a synth workload
    (detectors and blocks split evenly): (seconds, iterations, maps)."""
    import time
    m = int(wl.signal.size)
    nb = int(wl.block_sizes.size)
    if m % ranks or nb % ranks:
        raise ValueError("samples and blocks must split evenly over the ranks")
    t0 = time.perf_counter()
    maps = ref.mlmap(ranks, [m // ranks] * ranks, [nb // ranks] * ranks, wl.block_sizes, wl.pix, wl.weights,
                     wl.signal, wl.noise, int(wl.lam), wl.invtt, int(wl.nside), tol=tol, maxiter=maxiter)
    return time.perf_counter() - t0, int(len(maps[5]) - 1), maps


if __name__ == "__main__":
    if sys.argv[1] == "--mlmap":
        mlmap(*sys.argv[2:])
    else:
        main(*sys.argv[1:])
