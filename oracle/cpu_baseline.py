"""Times the reference's own C operator P^T N^-1 P (oracle/_ref) on host cores.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg runs this as a
separate process (a fresh interpreter that never touched CUDA, since the
oracle forks one process per rank).

    python -m oracle.cpu_baseline SAMPLE.npz RANKS   -> prints seconds per application (JSON)
    python -m oracle.cpu_baseline --mlmap CASE.npz RANKS OUT.npz
        -> runs the reference's whole MLmap (RANKS forked ranks, detectors split
           evenly), prints its wall time and iterations (JSON), saves its maps
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


if __name__ == "__main__":
    if sys.argv[1] == "--mlmap":
        mlmap(*sys.argv[2:])
    else:
        main(*sys.argv[1:])
