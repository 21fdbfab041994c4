"""Operator benchmark: times P, N^-1 and P^T on a seeded synthetic workload.

    python -m midapack_b200.opbench --dets 8 --samp 8388608 --block 1048576 --lam 16384 --grid 2048x1536

Prints one JSON line with the average milliseconds and the algorithmic GB/s of
each operator (CUDA events on the launching stream, inputs larger than L2).
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dets", type=int, default=8)
    ap.add_argument("--samp", type=int, default=1 << 23)
    ap.add_argument("--block", type=int, default=1 << 20)
    ap.add_argument("--lam", type=int, default=1 << 14)
    ap.add_argument("--grid", default="2048x1536")
    ap.add_argument("--gaps", type=float, default=0.01)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--ops", default="P,Ninv,Pt")
    a = ap.parse_args(argv)
    import torch

    import midapack_b200 as mb
    from midapack_b200 import synth
    w, h = (int(v) for v in a.grid.split("x"))
    wl = synth.make_workload_torch("opbench", w, h, a.dets, a.samp, a.block, a.lam, gap_frac=a.gaps, seed=99)
    ns = wl.n_samples
    ctx = mb.Context(0)
    P = mb.Pointing(ctx, wl.pix, wl.weights, ns, 3)
    N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    n = P.shape()["n_map"]
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty(ns, dtype=torch.float64, device="cuda")
    z = torch.empty(ns, dtype=torch.float64, device="cuda")
    xo = torch.empty(n, dtype=torch.float64, device="cuda")
    P.matvec(x, y)
    tile = N.tile()
    ops = {"P": (lambda: P.matvec(x, y), ns * 36 + n * 8),
           "Ninv": (lambda: N.apply(y, z), ns * 24 + tile["n_tiles"] * (tile["fft_n"] // 2 + 1) * 8),
           "Pt": (lambda: P.trmatvec(z, xo), ns * 36 + n * 8)}
    out = {"samples": ns, "unknowns": n, "tile": tile}
    s = torch.cuda.current_stream()
    for name in a.ops.split(","):
        fn, nbytes = ops[name]
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(a.reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        out[name] = {"ms": round(ms, 4), "algorithmic_GBps": round(nbytes / ms / 1e6, 1)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
