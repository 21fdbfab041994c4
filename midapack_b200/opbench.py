"""Operator benchmark: times P, N^-1 and P^T on a seeded synthetic workload.

    python -m midapack_b200.opbench --dets 8 --samp 8388608 --block 1048576 --lam 16384 --grid 2048x1536

Prints one JSON line with the average milliseconds and the algorithmic GB/s of
each operator (CUDA events on the launching stream, inputs larger than L2).
"""
from __future__ import annotations

import argparse
import json
import os


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
    ap.add_argument("--plans", default="",
                    help="';'-separated tile plans 'log2_cta_points,cluster,threads' to time N^-1 with "
                         "(FP64 for Ninv, FP32 for Ninv32); empty: the plan the library picks")
    a = ap.parse_args(argv)
    import torch

    import midapack_b200 as mb
    from midapack_b200 import synth
    w, h = (int(v) for v in a.grid.split("x"))
    wl = synth.make_workload_torch("opbench", w, h, a.dets, a.samp, a.block, a.lam, gap_frac=a.gaps, seed=99)
    ns = wl.n_samples
    ctx = mb.Context(0)
    P = mb.Pointing(ctx, wl.pix, wl.weights, ns, 3)
    n = P.shape()["n_map"]
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty(ns, dtype=torch.float64, device="cuda")
    z = torch.empty(ns, dtype=torch.float64, device="cuda")
    xo = torch.empty(n, dtype=torch.float64, device="cuda")
    P.matvec(x, y)
    y32, z32 = y.float(), torch.empty(ns, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(a.reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.reps

    out = {"samples": ns, "unknowns": n}
    plans = [p for p in a.plans.split(";") if p] or [None]
    for name in a.ops.split(","):
        if name in ("P", "Pt"):
            fn = (lambda: P.matvec(x, y)) if name == "P" else (lambda: P.trmatvec(z, xo))
            ms = timed(fn)
            out[name] = {"ms": round(ms, 4), "algorithmic_GBps": round((ns * 36 + n * 8) / ms / 1e6, 1)}
            continue
        if name == "Op32":
            # the FP32 operator of the mixed-precision solver: P (FP32 weights and TOD), N^-1 (FP32
            # tiles), P^T (FP64 accumulation), from and to FP64 maps
            N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
            mb.prepare_fp32(ctx, P, N)
            fn = lambda: mb.check(mb.lib().mdp_apply_op(ctx.h, P.h, N.h, x.data_ptr(), xo.data_ptr(), 1),  # noqa: E731
                                  "mdp_apply_op")
            ms = timed(fn)
            out[name] = {"ms": round(ms, 4), "tile": N.tile_fp32(), "plan": N._plan(1)}
            N.close()
            continue
        fp32 = name == "Ninv32"
        var = "MDP_TOEPLITZ_PLAN32" if fp32 else "MDP_TOEPLITZ_PLAN"
        res = []
        for plan in plans:
            if plan:
                os.environ[var] = plan
            try:
                N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
                tile = N.tile_fp32() if fp32 else N.tile()
            finally:
                os.environ.pop(var, None)
            sz = 4 if fp32 else 8
            nbytes = ns * 3 * sz + tile["n_tiles"] * (tile["fft_n"] // 4 + 1) * 2 * sz
            ms = timed((lambda: N.apply_fp32(y32, z32)) if fp32 else (lambda: N.apply(y, z)))
            res.append({"plan": plan, "tile": tile, "ms": round(ms, 4), "algorithmic_GBps": round(nbytes / ms / 1e6, 1)})
            N.close()
        out[name] = res if len(res) > 1 else res[0]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
