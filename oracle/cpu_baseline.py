"""Times the reference's own C operator P^T N^-1 P (oracle/_ref) on host cores.

TEST/BASELINE INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg runs this as a
separate process (a fresh interpreter that never touched CUDA, since the
oracle forks one process per rank).

    python -m oracle.cpu_baseline SAMPLE.npz RANKS   -> prints seconds per application (JSON)
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


if __name__ == "__main__":
    main(*sys.argv[1:])
