"""Time-to-map benchmark of the GLS map-making solve on one B200: mixed
precision vs plain FP64, multi-RHS, and served latency.

Headline (value): the at-scale workload, synthetic and seeded (no public
dataset is involved): 64 detectors x 2^24 samples (1.07e9 samples) on a
2048x1536 flat grid (3.1M pixels, 9.4M I/Q/U unknowns), 2^20-sample stationary
intervals (1024 Toeplitz blocks, lambda = 2^14), 1% flagged samples, int32
pointing, FP64 weights and TOD.  One step = one complete map-making solve from
device-resident inputs: pointing compression (MatInit), inverse-noise spectra
and tile plans, block-Jacobi build with the rcond cut, PCG to relative
residual 1e-8 (the reference's criterion); value = mixed precision,
config.fp64 = the plain FP64 path.  Further keys on the same line: e2e (the
same solve from pinned host inputs through the library's API, copies
included; e2e.mlmap_fp64 the reference's MLmap entry point, FP64, host maps
out), cpu_baseline (the reference's C operator on
the host cores, extrapolated), c1_reference (the CPU-runnable workload: the
reference's whole MLmap on 4 host ranks vs the GPU paths), mixed_fknee_sweep
(CPU-runnable workload, f_knee 0.1/1/5 Hz), solvers_low_fknee (two-level
preconditioners and ECG at f_knee 0.1 Hz), multi_rhs (128 right-hand sides
sharing one pointing), serving (Poisson stream of independent solves, p50/p99
latency).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --impl reference the reference's own C code (oracle/_ref, built from its
sources; no part of this library is loaded) is timed on the host cores on a
bounded sample of the same workload: W + K operator applications P^T N^-1 P
(the last K timed), one detector of the at-scale scan per forked rank, as many
ranks as host cores, extrapolated to all detectors and to the solve's
applications (REFERENCE_ITERATIONS + 1, a fixed count stated on the line);
beside it, measured and not extrapolated, the reference's whole MLmap on the
CPU-runnable workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIG = "c2_64det_2p24_2048x1536_lam16384"
MULTI_CONFIG = "c4_16det_2p23_1024x768_lam8192"
METRIC = "time-to-map at 1e-8 residual, mixed vs FP64 on 1 B200; served p50/p99 latency"
TOL = 1e-8
MAXITER = 500
# multi-RHS part: the relative residual at which the plain FP64 path's own maps
# are within 1e-8 of the converged (1e-12) solution, so that mixed-precision
# maps can be held to 1e-8 of the FP64 oracle
MULTI_TOL = 1e-10
# PCG iterations of the at-scale workload at TOL (PCG_GLS_true's recurrences and
# stop test): fixed here for the reference arm, which cannot run the whole solve
# on the host; the library's FP64 PCG, whose iteration counts equal the
# reference's within one on every case both run, takes 60 on a B200.
REFERENCE_ITERATIONS = 60


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--inner-tol", type=float, default=1e-4)
    ap.add_argument("--no-compare", action="store_true", help="skip timing the other precision")
    ap.add_argument("--no-multi", action="store_true", help="skip the multi-RHS part")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving part")
    ap.add_argument("--no-fknee", action="store_true", help="skip the f_knee sweep part")
    ap.add_argument("--no-c1", action="store_true", help="skip the CPU-runnable reference comparison")
    ap.add_argument("--no-solvers", action="store_true", help="skip the two-level / ECG part")
    ap.add_argument("--no-noise", action="store_true", help="skip the noise2invtt part")
    ap.add_argument("--only", default="", choices=["", "multi", "serve", "fknee", "c1", "solvers", "noise", "operator"],
                    help="run only one part (prints its JSON); 'operator' times P, N^-1 and P^T alone")
    ap.add_argument("--op-dets", type=int, default=8, help="operator part: detectors")
    ap.add_argument("--op-samp", type=int, default=1 << 23, help="operator part: samples per detector")
    ap.add_argument("--op-block", type=int, default=1 << 20, help="operator part: block length")
    ap.add_argument("--op-lam", type=int, default=1 << 14, help="operator part: lambda")
    ap.add_argument("--op-grid", default="2048x1536", help="operator part: grid WxH")
    ap.add_argument("--op-reps", type=int, default=5, help="operator part: timed repetitions")
    ap.add_argument("--op-list", default="P,Ninv,Pt,Ninv32,Op32", help="operator part: operators to time")
    ap.add_argument("--op-plans", default="",
                    help="operator part: ';'-separated N^-1 tile plans (mdp_noise_set_plan names); empty: auto")
    ap.add_argument("--multi-rhs", type=int, default=128, help="right-hand sides of the multi-RHS part")
    ap.add_argument("--multi-fp64-cols", type=int, default=2, help="columns timed with the plain FP64 path")
    ap.add_argument("--multi-inner-tol", type=float, default=1e-4,
                    help="relative residual of the multi-RHS inner (FP32) solves between FP64 refinements")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-rate", type=float, default=50.0, help="mean Poisson arrival rate, solves/s")
    ap.add_argument("--serve-datasets", type=int, default=16)
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--ninv-plan", default="", help="force the FP64 N^-1 tile plan of the headline solves (profiling)")
    ap.add_argument("--ninv-plan32", default="", help="force the FP32 N^-1 tile plan of the headline solves (profiling)")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 ranks: N independent solves instead of one solve sharded over the ranks")
    return ap.parse_args()


_T0 = time.perf_counter()


def log(msg: str):
    """Progress of the run on stderr (the JSON line stays the only stdout)."""
    sys.stderr.write(f"[bench +{time.perf_counter() - _T0:7.1f} s] {msg}\n")
    sys.stderr.flush()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload_config(name: str, world: int) -> dict:
    """The workload a line is measured on (both arms print the same dict)."""
    from midapack_b200 import synth
    c = synth.CONFIGS[name]
    ns = c["n_det"] * c["n_samp"]
    return {"workload": name if world == 1 else f"{name} per rank, {world} ranks",
            "detectors": c["n_det"] * world, "samples_per_detector": c["n_samp"], "samples": ns * world,
            "grid": f"{c['width']}x{c['height']}", "pixels": c["width"] * c["height"], "lambda": c["lam"],
            "block_len": c["block_len"], "blocks": ns // c["block_len"] * world,
            "flagged_fraction": c.get("gap_frac", 0.0), "fknee_hz": c.get("fknee", 1.0), "tol": TOL,
            "l2": "inputs (tens of GB) far larger than L2",
            "parallelism": "one solve per GPU" if world == 1 else f"one solve sharded over {world} ranks"}


def algorithmic_bytes(ns: int, n_map: int, n_tiles: int, fft_m: int):
    """Bytes one application of each operator must move (FP64, triplet pointing)."""
    return {
        "P": ns * (4 + 24 + 8) + n_map * 8,
        "Ninv": ns * (8 + 8 + 8) + n_tiles * (fft_m + 1) * 8,   # mean pass read, tile read, write
        "Pt": ns * (4 + 24 + 8) + n_map * 8,
    }


def algorithmic_bytes32(ns: int, n_map: int, t32):
    """FP32 operator of the mixed solver: FP32 weights and TOD, FP64 map."""
    n_tiles, fft_m = t32
    return {
        "P": ns * (4 + 12 + 4) + n_map * 8,
        "Ninv": ns * (4 + 4) + n_tiles * (fft_m + 1) * 4,   # means fused into P
        "Pt": ns * (4 + 4 + 12 + 4) + n_map * 8,            # bin list, offset, weights, TOD
    }


# DRAM bytes per tile of one N^-1 application, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of the three split kernels,
# lambda 2^14, 2^20-sample blocks), keyed by (precision, M1, M2); scaled to a
# launch by the tile count.  256 x 256: 704 tiles in one application; 256 x 512:
# three applications of 160 tiles, the split_pairs_kernel's 1.3 MB taken out
# (profiles/ninv_split_fp32_256x256_lambda16384.md, operator_p_pt_ninv_dram_2p25.md)
NINV_TRAFFIC_PER_TILE = {("f32", 256, 256): 1857072128 / 704,
                         ("f32", 256, 512): (2370306304 - 1314000) / (3 * 160)}


def ninv_kernel(t: dict, prec: str) -> str:
    if t.get("cluster_four_step"):
        m1, m2 = t["cluster_four_step"]
        return f"ninv4_kernel<{prec}, {t['cluster']}> ({m1}x{m2} cluster four-step tiles)"
    if t.get("split"):
        m1, m2 = t["split"]
        return f"split_cols_kernel + split_rows_kernel + split_cols_kernel<{prec}> ({m1}x{m2} four-step tiles)"
    return f"toeplitz_tile_kernel<{prec}, {int(np.log2(t['cta_points']))}, {t['cluster']}>"


def cpu_reference(wl_host, iterations: int, sample_dets: int, full_samples: int, cores: int):
    """Reference C operator (oracle/_ref) on host cores: one P^T N^-1 P application
    over `sample_dets` detectors (one per forked rank, in a fresh process that
    never initialised CUDA), extrapolated to the full solve."""
    from oracle import ref
    if not ref.available():
        return None
    pix, w, bs, lam, invtt, per_det = wl_host
    # Toeplitz blocks per detector: blocks whose cumulative end falls within one detector's samples
    ends = np.cumsum(np.asarray(bs, dtype=np.int64))
    nb_per_det = int(np.searchsorted(ends, per_det, side="right"))
    if nb_per_det < 1 or ends[nb_per_det - 1] != per_det:
        raise RuntimeError("Toeplitz blocks do not tile the detectors")
    # the sample (several GB) goes through host memory when /dev/shm exists
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as td:
        path = os.path.join(td, "sample.npz")
        np.savez(path, pix=pix, weights=w, block_sizes=bs, lam=lam, invtt=invtt, per_det=per_det,
                 nb_per_det=nb_per_det)
        r = subprocess.run([sys.executable, "-m", "oracle.cpu_baseline", path, str(sample_dets)], cwd=ROOT,
                           capture_output=True, text=True, timeout=900)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not lines:
            sys.stderr.write("reference baseline output (tail):\n" + r.stdout[-4000:] + "\n----- stderr -----\n" +
                             r.stderr[-4000:] + "\n")
            errs = [ln for ln in r.stderr.splitlines() if "shim_mpi" in ln or "Error" in ln]
            raise RuntimeError(f"reference baseline failed: {' | '.join(errs[-3:])}")
        t = json.loads(lines[-1])["seconds_per_application"]
    # sample_dets ranks ran concurrently: per-application time of the full job on `cores` ranks
    per_iter_full = t * (full_samples / (per_det * sample_dets)) * (sample_dets / cores)
    return {"op_seconds_sample": t, "per_iter_full_s": per_iter_full, "time_to_map_s": per_iter_full * (iterations + 1)}


def bench_multi(args, device):
    """Multi-RHS configuration: 16 det x 2^23 samples, 1024x768 px, lambda 2^13,
    1% flagged samples; args.multi_rhs columns = 1 signal+noise + Monte-Carlo
    noise realisations (FP32 values, same PSD), solved by the multi-RHS mixed
    solver; the plain FP64 path times args.multi_fp64_cols columns one by one."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    cfg = synth.CONFIGS[MULTI_CONFIG]
    wl = synth.make_workload_torch(MULTI_CONFIG, **cfg)
    m = wl.n_samples
    noise = synth.mc_noise_torch(wl.n_det, wl.n_samp, args.multi_rhs, wl.fknee, seed=20261211)
    ctx = mb.Context(device)
    # warm-up: plans, tuner and bins on a separate pointing of the same data
    P0 = mb.Pointing(ctx, wl.pix, wl.weights, m, 3)
    N0 = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    mb.gls_solve_multi(ctx, P0, N0, noise[:2], signal=wl.signal, signal_col=0, tol=MULTI_TOL, maxiter=3, slots=0)
    del P0, N0
    torch.cuda.synchronize()
    P = mb.Pointing(ctx, wl.pix, wl.weights, m, 3)
    N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    l0 = ctx.launches
    t0 = time.perf_counter()
    x, lst, cond, hits, ci, info = mb.gls_solve_multi(ctx, P, N, noise, signal=wl.signal, signal_col=0, tol=MULTI_TOL,
                                                      maxiter=MAXITER, inner_tol=args.multi_inner_tol, slots=0,
                                                      use_graph=True)
    torch.cuda.synchronize()
    t_multi = time.perf_counter() - t0
    log(f"multi-RHS solve: {args.multi_rhs} columns in {t_multi:.2f} s")
    launches = ctx.launches - l0
    xs = x[: min(args.multi_fp64_cols, args.multi_rhs)].cpu().numpy()
    del x
    fp64 = []
    errs = {"multi_mixed": {"I": 0.0, "Q": 0.0, "U": 0.0}, "fp64_path": {"I": 0.0, "Q": 0.0, "U": 0.0}}
    for c in range(min(args.multi_fp64_cols, args.multi_rhs)):
        P1 = mb.Pointing(ctx, wl.pix, wl.weights, m, 3)
        N1 = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
        sig = wl.signal if c == 0 else torch.zeros_like(wl.signal)
        nz = noise[c].double()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x1, l1, _, _, _, i1 = mb.gls_solve(ctx, P1, N1, sig, nz, tol=MULTI_TOL, maxiter=4 * MAXITER)
        torch.cuda.synchronize()
        fp64.append((time.perf_counter() - t0, i1.iterations, bool(i1.converged)))
        x1 = x1.cpu().numpy()
        # FP64 oracle of the column: the plain FP64 path at tol 1e-12 (untimed)
        xo = mb.gls_solve(ctx, P1, N1, sig, nz, tol=1e-12, maxiter=4 * MAXITER)[0].cpu().numpy()
        log(f"multi-RHS part: FP64 column {c} and its oracle done")
        for tag, xv in (("multi_mixed", xs[c]), ("fp64_path", x1)):
            for k, name in enumerate("IQU"):
                errs[tag][name] = max(errs[tag][name],
                                      float(np.linalg.norm(xv[k::3] - xo[k::3]) / np.linalg.norm(xo[k::3])))
        del P1, N1, nz, sig
    t64 = float(np.mean([f[0] for f in fp64]))
    out = {"workload": MULTI_CONFIG, "tol": MULTI_TOL, "inner_tol": args.multi_inner_tol, "rhs": args.multi_rhs, "columns": "1 signal+noise + "
           f"{args.multi_rhs - 1} Monte-Carlo noise realisations (FP32 values)",
           "time_s": round(t_multi, 3), "solves_per_s": round(args.multi_rhs / t_multi, 3),
           "fp64_path": {"seconds_per_solve": round(t64, 4), "solves_per_s": round(1.0 / t64, 3),
                         "columns_timed": len(fp64), "iterations": [f[1] for f in fp64],
                         "converged": all(f[2] for f in fp64)},
           "speedup_vs_fp64": round(t64 * args.multi_rhs / t_multi, 3),
           "slots": info.slots, "graph": bool(info.graph), "batched_iterations": info.batched_iterations,
           "inner_iterations_mean": round(info.total_iterations / args.multi_rhs, 1),
           "fp64_applications": info.fp64_applications, "converged": sum(c.converged for c in ci),
           "precond_s": round(info.precond_seconds, 3), "map_rel_err_vs_fp64_oracle": errs,
           "oracle": "plain FP64 path at tol 1e-12 on the timed FP64 columns",
           "fft_tile_fp32": N.tile_fp32(), "gpu_launches": int(launches)}
    del P, N, noise, wl
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def bench_operator(args, device):
    """The operators alone on a seeded workload (--op-* sizes; inputs larger
    than L2): P, N^-1 (FP64 and FP32, each tile plan of --op-plans), P^T and
    the FP32 operator P^T N^-1 P of the mixed solver; CUDA events on the
    launching stream around --op-reps applications after two warm-ups, and each
    operator's algorithmic bytes per second."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    w, h = (int(v) for v in args.op_grid.split("x"))
    wl = synth.make_workload_torch("operator", w, h, args.op_dets, args.op_samp, args.op_block, args.op_lam,
                                   gap_frac=0.01, seed=99)
    ns = wl.n_samples
    ctx = mb.Context(device)
    P = mb.Pointing(ctx, wl.pix, wl.weights, ns, 3)
    n = P.shape()["n_map"]
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty(ns, dtype=torch.float64, device="cuda")
    z = torch.empty(ns, dtype=torch.float64, device="cuda")
    xo = torch.empty(n, dtype=torch.float64, device="cuda")
    P.matvec(x, y)
    y32, z32 = y.float(), torch.empty(ns, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = ctx.launches
        e0.record(stream)
        for _ in range(args.op_reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.op_reps, (ctx.launches - l0) // args.op_reps

    out = {"samples": ns, "unknowns": n, "lambda": args.op_lam, "block": args.op_block}
    plans = [p for p in args.op_plans.split(";") if p] or ["auto"]
    for name in args.op_list.split(","):
        if name in ("P", "Pt"):
            ms, nl = timed((lambda: P.matvec(x, y)) if name == "P" else (lambda: P.trmatvec(z, xo)))
            out[name] = {"ms": round(ms, 4), "launches": nl,
                         "algorithmic_GBps": round(algorithmic_bytes(ns, n, 0, 0)[name] / ms / 1e6, 1)}
            continue
        res = []
        for plan in plans:
            fp32 = name in ("Ninv32", "Op32")
            N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
            if plan != "auto":
                N.set_plan(plan, fp32=fp32)
            tile = N.tile_fp32() if fp32 else N.tile()
            if name == "Op32":
                mb.prepare_fp32(ctx, P, N)
                ms, nl = timed(lambda: mb.check(mb.lib().mdp_apply_op(ctx.h, P.h, N.h, x.data_ptr(), xo.data_ptr(), 1),
                                                "mdp_apply_op"))
                res.append({"plan": plan, "tile": tile, "ms": round(ms, 4), "launches": nl})
            else:
                ab = (algorithmic_bytes32(ns, n, (tile["n_tiles"], tile["fft_n"] // 2)) if fp32
                      else algorithmic_bytes(ns, n, tile["n_tiles"], tile["fft_n"] // 2))["Ninv"]
                ms, nl = timed((lambda: N.apply_fp32(y32, z32)) if fp32 else (lambda: N.apply(y, z)))
                res.append({"plan": plan, "tile": tile, "ms": round(ms, 4), "launches": nl,
                            "algorithmic_GBps": round(ab / ms / 1e6, 1)})
            N.close()
        out[name] = res if len(res) > 1 else res[0]
    ctx.close()
    return out


def bench_fknee(args, device):
    """Mixed-precision configuration on the CPU-runnable workload (4 det x 2^20
    samples, 256x192 px, lambda 2^12) with f_knee in {0.1, 1, 5} Hz: mixed and
    plain FP64 time-to-map at 1e-8 and each map's I/Q/U error against the FP64
    oracle (plain FP64 path at tol 1e-12).  1% flagged samples: without them the
    operator of this workload is singular (constant offset) and neither path
    reaches 1e-8.  Timed per path: the block-Jacobi build and the solve, on
    operators built beforehand (compression and FP64 spectra at creation, the
    FP32 weights and spectra by prepare_fp32 for the mixed path)."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    base = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"])
    ctx = mb.Context(device)
    out = {"workload": "c1_4det_2p20_256x192_lam4096 + 1% flagged samples", "tol": TOL}
    for fk in (0.1, 1.0, 5.0):
        cfg = dict(base, fknee=fk, gap_frac=0.01)
        wl = synth.make_workload_torch("c3", **cfg)
        m = wl.n_samples
        res = {}
        for prec, fn, tol in (("oracle", mb.gls_solve, 1e-12), ("fp64", mb.gls_solve, TOL),
                              ("mixed", mb.gls_solve_mixed, TOL)):
            ts = []
            for rep in range(1 if prec == "oracle" else 3):
                P = mb.Pointing(ctx, wl.pix, wl.weights, m, 3)
                N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)  # FP64 plan and spectra built here
                if prec == "mixed":
                    mb.prepare_fp32(ctx, P, N)  # the FP32 operator state, likewise outside the timed solve
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                o = fn(ctx, P, N, wl.signal, wl.noise, tol=tol, maxiter=4 * MAXITER)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            res[prec] = (o[0].cpu().numpy(), o[5], min(ts))
        xo = res["oracle"][0]
        entry = {}
        for prec in ("fp64", "mixed"):
            x, info, t = res[prec]
            entry[prec] = {"time_to_map_s": round(t, 4), "iterations": info.iterations,
                           "converged": bool(info.converged),
                           "map_rel_err_vs_fp64_oracle": {
                               name: float(np.linalg.norm(x[k::3] - xo[k::3]) / np.linalg.norm(xo[k::3]))
                               for k, name in enumerate("IQU")}}
        entry["oracle_iterations"] = res["oracle"][1].iterations
        out[f"fknee_{fk:g}"] = entry
        del wl, res
    ctx.close()
    torch.cuda.empty_cache()
    return out


def run_part(fn, args, device):
    """One auxiliary part of the bench line; a part that fails is reported on
    the line (its error) instead of ending the run without a line."""
    log(f"{fn.__name__}: start")
    try:
        out = fn(args, device)
        log(f"{fn.__name__}: done")
        return out
    except Exception as ex:  # noqa: BLE001
        import torch
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        sys.stderr.write(f"bench part {fn.__name__} failed: {type(ex).__name__}: {ex}\n")
        return {"error": f"{type(ex).__name__}: {ex}"}


def bench_c1(args, device):
    """The CPU-runnable configuration (4 detectors x 2^20 samples, 256x192 px,
    lambda 2^12, one Toeplitz block per detector) with 1% flagged samples (without
    them the operator is singular and the reference stalls above 1e-8): the
    reference's whole MLmap (oracle/_ref: set-up, block-Jacobi, PCG to 1e-8) on 4
    forked host ranks, wall time, against the plain FP64 and mixed GPU paths
    (time-to-map from device-resident inputs, compression and operator set-up
    included, best of 3 after a warm-up) and each GPU map's I/Q/U error against
    the reference's maps on the observed pixels."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    from oracle import ref
    cfg = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"], gap_frac=0.01)
    wl = synth.make_workload("c1", **cfg)
    m, nside = wl.n_samples, wl.nside
    out = {"workload": "c1_4det_2p20_256x192_lam4096 + 1% flagged samples", "tol": TOL}
    if not ref.available():
        out["reference"] = {"unavailable": "oracle/_ref not built"}
        refmaps = None
    else:
        with tempfile.TemporaryDirectory() as td:
            case, res_path = os.path.join(td, "case.npz"), os.path.join(td, "maps.npz")
            np.savez(case, pix=wl.pix, weights=wl.weights, signal=wl.signal, noise=wl.noise,
                     block_sizes=wl.block_sizes, lam=wl.lam, invtt=wl.invtt, nside=nside, tol=TOL,
                     maxiter=4 * MAXITER)
            r = subprocess.run([sys.executable, "-m", "oracle.cpu_baseline", "--mlmap", case, "4", res_path],
                               cwd=ROOT, capture_output=True, text=True, timeout=1200)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            if r.returncode != 0 or not lines:
                raise RuntimeError("reference MLmap failed: " + r.stderr[-500:])
            rj = json.loads(lines[-1])
            mz = np.load(res_path)
            refmaps = (mz["I"], mz["Q"], mz["U"], mz["Hits"])
        out["reference"] = {"path": "reference MLmap (oracle/_ref, shim FFT/MPI/LAPACK), 4 forked host ranks",
                            "ranks": rj["ranks"], "time_to_map_s": round(rj["seconds"], 3),
                            "iterations": rj["iterations"],
                            "per_iter_ms": round(1e3 * rj["seconds"] / max(rj["iterations"], 1), 3)}
    ctx = mb.Context(device)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    pix, w, sig, noi = d(wl.pix), d(wl.weights), d(wl.signal), d(wl.noise)
    npix = 12 * nside * nside
    for prec, fn in (("fp64", mb.gls_solve), ("mixed", mb.gls_solve_mixed)):
        ts = []
        for rep in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            P = mb.Pointing(ctx, pix, w, m, 3)
            N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
            o = fn(ctx, P, N, sig, noi, tol=TOL, maxiter=4 * MAXITER)
            torch.cuda.synchronize()
            if rep:
                ts.append(time.perf_counter() - t0)
        x, lst, info = o[0].cpu().numpy(), o[1].cpu().numpy(), o[5]
        entry = {"time_to_map_s": round(min(ts), 4), "iterations": info.iterations, "converged": bool(info.converged),
                 "per_iter_ms": round(1e3 * min(ts) / max(info.iterations, 1), 3)}
        if refmaps is not None:
            p = lst[0::3] // 3
            hit = refmaps[3][p] > 0
            errs = {}
            for k, name in enumerate("IQU"):
                mine = np.zeros(npix)
                mine[p] = x[k::3]
                sel = np.zeros(npix, dtype=bool)
                sel[p[hit]] = True
                errs[name] = float(np.linalg.norm(mine[sel] - refmaps[k][sel]) / np.linalg.norm(refmaps[k][sel]))
            entry["map_rel_err_vs_reference"] = errs
            entry["speedup_vs_reference"] = round(out["reference"]["time_to_map_s"] / min(ts), 1)
        out[prec] = entry
    ctx.close()
    torch.cuda.empty_cache()
    return out


def bench_noise2invtt(args, device):
    """noise2invtt (mappraiser/python/TOAST_interface/utils.py:500-602) for every
    stationary interval of the at-scale workload: 1024 intervals x 2^20 samples,
    lambda 2^14, chebwin window.  The device path (periodogram, fit, inverse row of
    each interval; noise resident on the device; CUDA events around the call, best
    of 2 after a warm-up) against the reference's algorithm (the scipy
    restatement with curve_fit's default tolerances, one host core) on a sample of
    2 intervals, extrapolated to all 1024, and the device rows' error against that
    restatement's rows (bounded by curve_fit's ftol = 1e-8)."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import noise as mn
    from midapack_b200 import synth
    from oracle import restate
    nblk, n, lam, distinct = 1024, 1 << 20, 1 << 14, 8
    rng = np.random.default_rng(20261212)
    blocks = [synth.noise_tod(n, fk, rng) for fk in np.linspace(0.1, 5.0, distinct)]
    d_noise = torch.from_numpy(np.concatenate(blocks)).cuda().repeat(nblk // distinct)
    sizes = np.full(nblk, n, dtype=np.int32)
    ctx = mb.Context(device)
    times = []
    for rep in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = ctx.launches
        e0.record()
        out, params, evals = mn.invtt_blocks(d_noise, sizes, lam, 100.0, "chebwin", ctx=ctx, return_fit=True)
        e1.record()
        torch.cuda.synchronize()
        launches = ctx.launches - l0
        if rep:
            times.append(e0.elapsed_time(e1) / 1e3)
    rows = out.view(nblk, lam).cpu().numpy()
    del d_noise, out
    cpu_t, errs = [], []
    for b in range(2):
        t0 = time.perf_counter()
        r, _, _ = restate.noise2invtt(blocks[b], n, lam, 100.0, "chebwin")
        cpu_t.append(time.perf_counter() - t0)
        errs.append(float(np.linalg.norm(rows[b] - r) / np.linalg.norm(r)))
    dev = min(times)
    cpu_all = float(np.mean(cpu_t)) * nblk
    ctx.close()
    torch.cuda.empty_cache()
    return {"workload": f"{nblk} intervals x 2^20 samples, lambda 2^14, chebwin ({distinct} distinct seeded 1/f "
                        f"streams, f_knee 0.1-5 Hz, tiled)",
            "device_s": round(dev, 4), "intervals_per_s": round(nblk / dev, 1),
            "samples_per_s": round(nblk * n / dev, 1), "gpu_launches": int(launches),
            "fit_evaluations_mean": round(float(evals.mean()), 1), "fit_evaluations_max": int(evals.max()),
            "cpu_reference_algorithm": {"kind": "port", "cores": 1, "sample": "2 intervals (scipy welch + "
                                        "curve_fit + irfft), extrapolated x512",
                                        "s_per_interval": round(float(np.mean(cpu_t)), 3),
                                        "extrapolated_s": round(cpu_all, 1)},
            "speedup_vs_cpu": round(cpu_all / dev, 1),
            "row_rel_err_vs_reference_algorithm": max(errs)}


def bench_solvers(args, device):
    """The reference's other solvers and preconditioners on the CPU-runnable
    workload at low f_knee (0.1 Hz, the ill-conditioned end of the sweep), 1%
    flagged samples: block-Jacobi PCG (precond 0), the two-level
    preconditioners (precond 1 a priori, precond 2 a posteriori, z_2lvl
    columns) and ECG (solver 1, Orthomin, enlFac search directions), FP64, and the
    mixed-precision solve with block Jacobi and with the a-priori two-level
    preconditioner, all to relative residual 1e-8; time-to-map from device-resident inputs with the
    set-up (compression, spectra, block-Jacobi, deflation columns) included, best
    of 2 after a warm-up, and each map's I/Q/U error against the FP64 PCG
    solution at 1e-12."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    cfg = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"], gap_frac=0.01, fknee=0.1)
    wl = synth.make_workload_torch("solvers", **cfg)
    m = wl.n_samples
    ctx = mb.Context(device)
    out = {"workload": "c1_4det_2p20_256x192_lam4096 + 1% flagged samples, f_knee 0.1 Hz", "tol": TOL}
    runs = [("pcg_bj", mb.gls_solve, {}),
            ("pcg_2lvl_apriori_z1", mb.gls_solve, {"precond": 1, "z_2lvl": 1}),
            ("pcg_2lvl_apriori_z8", mb.gls_solve, {"precond": 1, "z_2lvl": 8}),
            ("pcg_2lvl_aposteriori_z8", mb.gls_solve, {"precond": 2, "z_2lvl": 8}),
            ("pcg_2lvl_aposteriori_z16", mb.gls_solve, {"precond": 2, "z_2lvl": 16}),
            ("ecg_omin_enl4", mb.gls_solve_ecg, {"enl_fac": 4}),
            ("ecg_omin_enl8", mb.gls_solve_ecg, {"enl_fac": 8}),
            ("mixed_bj", mb.gls_solve_mixed, {}),
            ("mixed_2lvl_apriori_z1", mb.gls_solve_mixed, {"precond": 1, "z_2lvl": 1})]

    def solve(fn, kw, tol):
        P = mb.Pointing(ctx, wl.pix, wl.weights, m, 3)
        N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
        return fn(ctx, P, N, wl.signal, wl.noise, tol=tol, maxiter=4 * MAXITER, **kw)

    xo = solve(mb.gls_solve, {}, 1e-12)[0].cpu().numpy()
    for name, fn, kw in runs:
        ts = []
        try:
            for rep in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                o = solve(fn, kw, TOL)
                torch.cuda.synchronize()
                if rep:
                    ts.append(time.perf_counter() - t0)
        except Exception as ex:  # noqa: BLE001 - reported on the line, the other parts still run
            out[name] = {"error": f"{type(ex).__name__}: {ex}"}
            continue
        x, info = o[0].cpu().numpy(), o[5]
        out[name] = {"time_to_map_s": round(min(ts), 4), "iterations": info.iterations,
                     "converged": bool(info.converged),
                     "map_rel_err_vs_fp64_oracle": {
                         nm: float(np.linalg.norm(x[k::3] - xo[k::3]) / np.linalg.norm(xo[k::3]))
                         for k, nm in enumerate("IQU")}}
    ctx.close()
    torch.cuda.empty_cache()
    return out


def bench_serving(args, device):
    """Serving configuration: Poisson arrivals (args.serve_rate per second) of
    independent solves on args.serve_datasets resident datasets drawn
    log-uniformly (detectors 1-32, samples/det 2^18-2^23, grid side 64-1024 at
    4:3, lambda 2^8-2^14, f_knee uniform 0.1-5 Hz, 1% flagged samples); each
    request is its dataset's signal plus a fresh noise realisation, mixed
    precision to 1e-8; the same stream again with the plain FP64 path."""
    import torch
    from midapack_b200 import serve
    specs = serve.draw_specs(args.serve_datasets, seed=20261208)
    n = args.serve_requests
    offsets = serve.poisson_arrivals(n, args.serve_rate, seed=20261209)
    pick = np.random.default_rng(20261210).integers(0, len(specs), n)
    ex = serve.GpuExecutor(device, keep_maps=lambda rid: rid < 32)
    srv = serve.Server(ex, slots=args.serve_slots, work_budget=48 << 30, dataset_budget=96 << 30)
    t0 = time.perf_counter()
    for s in specs:
        srv.preload(s)
    # untimed warm-up: every slot solves the largest dataset once per precision,
    # so that the slots' work buffers have their final sizes before timing
    big = max(specs, key=lambda s: s.n_samples)
    for prec in ("fp64", "mixed"):
        warm = [srv.submit(serve.Request(-1 - k, big, noise_seed=k, precision=prec, tol=TOL))
                for k in range(args.serve_slots)]
        for tk in warm:
            tk.wait(1800.0)
    t_pre = time.perf_counter() - t0
    log(f"serving: datasets preloaded, slots warm ({t_pre:.1f} s)")
    out = {"requests": n, "rate_per_s": args.serve_rate, "datasets": len(specs), "slots": args.serve_slots,
           "dataset_samples": [s.n_samples for s in specs], "preload_and_warmup_s": round(t_pre, 2)}
    res = {}
    for prec in ("fp64", "mixed"):
        reqs = [serve.Request(i, specs[pick[i]], noise_seed=1000 + i, precision=prec, tol=TOL) for i in range(n)]
        srv.max_running = 0
        r = serve.run_stream(srv, reqs, offsets, timeout=1800.0)
        st = serve.latency_stats(r)
        st["max_concurrent"] = srv.max_running
        st["errors"] = sum(1 for x in r if x.error)
        if st["errors"]:
            st["error_samples"] = sorted({x.error for x in r if x.error})[:4]
        out[prec] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()}
        res[prec] = r
        log(f"serving: {prec} stream done")
    # the same stream offered at half the FP64 path's measured throughput, so that
    # p50/p99 measure service time rather than the growth of a queue
    rate2 = round(0.5 * out["fp64"]["solves_per_s"], 2)
    if rate2 > 0:
        n2 = min(n, 96)
        off2 = serve.poisson_arrivals(n2, rate2, seed=20261213)
        sus = {"rate_per_s": rate2, "requests": n2}
        for prec in ("fp64", "mixed"):
            reqs = [serve.Request(i, specs[pick[i]], noise_seed=3000 + i, precision=prec, tol=TOL) for i in range(n2)]
            srv.max_running = 0
            r2 = serve.run_stream(srv, reqs, off2, timeout=1800.0)
            st2 = serve.latency_stats(r2)
            st2["max_concurrent"] = srv.max_running
            st2["errors"] = sum(1 for x in r2 if x.error)
            sus[prec] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st2.items()}
        out["sustainable_rate"] = sus
    # FP64 oracle (tol 1e-12) for the requests whose maps were kept: the error
    # of each path's map, max over the requests, per I/Q/U
    n_or = min(8, n)
    oracle = [serve.Request(i, specs[pick[i]], noise_seed=1000 + i, precision="fp64", tol=1e-12, maxiter=2000)
              for i in range(n_or)]
    ores = [tk.wait(1800.0) for tk in [srv.submit(r) for r in oracle]]
    srv.close()
    for prec in ("mixed", "fp64"):
        errs = {"I": 0.0, "Q": 0.0, "U": 0.0}
        for a, o in zip(res[prec][:n_or], ores):
            if a.x is None or o.x is None:
                continue
            for k, name in enumerate("IQU"):
                errs[name] = max(errs[name], float(np.linalg.norm(a.x[k::3] - o.x[k::3]) / np.linalg.norm(o.x[k::3])))
        out[prec]["map_rel_err_vs_fp64_oracle"] = errs
    out["oracle"] = f"plain FP64 path at tol 1e-12 on the first {n_or} requests"
    out["speedup_solves_per_s"] = round(out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"], 3)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        # the reference's own code on the host: no CUDA, no part of this library
        return run_reference(args, rank, world)
    import torch
    local = local % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(local)
    if args.only:
        r = {"multi": bench_multi, "serve": bench_serving, "fknee": bench_fknee, "c1": bench_c1,
             "solvers": bench_solvers, "noise": bench_noise2invtt, "operator": bench_operator}[args.only](args, local)
        print(json.dumps({args.only: r}), flush=True)
        return 0
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        # MDP_BENCH_BACKEND=gloo runs the ranks' exchanges through host memory
        # (a functional check of the sharded path with several ranks on one GPU)
        dist.init_process_group(os.environ.get("MDP_BENCH_BACKEND", "nccl"), timeout=timedelta(seconds=600))

    import midapack_b200 as mb
    from midapack_b200 import synth
    cfg = dict(synth.CONFIGS[args.config])
    cfg["seed"] = cfg["seed"] + rank
    log(f"workload {args.config}: generating")
    wl = synth.make_workload_torch(args.config, **cfg)
    torch.cuda.synchronize()
    log("workload ready")
    ns = wl.n_samples
    nb = len(wl.block_sizes)
    idv = np.arange(nb, dtype=np.int64) * wl.block_len
    ctx = mb.Context(local)

    def one_solve(precision=args.precision):
        P = mb.Pointing(ctx, wl.pix, wl.weights, ns, 3)
        N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt, idv=idv)
        if args.ninv_plan:
            N.set_plan(args.ninv_plan, fp32=False)
        if args.ninv_plan32:
            N.set_plan(args.ninv_plan32, fp32=True)
        if precision == "mixed":
            out = mb.gls_solve_mixed(ctx, P, N, wl.signal, wl.noise, tol=TOL, maxiter=MAXITER,
                                     inner_tol=args.inner_tol)
        else:
            out = mb.gls_solve(ctx, P, N, wl.signal, wl.noise, tol=TOL, maxiter=MAXITER)
        return P, N, out

    if world > 1 and not args.replicas:
        return run_sharded(args, wl, ctx, rank, world, local, idv)

    for k in range(args.warmup):
        one_solve()
        torch.cuda.synchronize()
        log(f"warm-up solve {k + 1}/{args.warmup} ({args.precision})")
    if world > 1:
        torch.distributed.barrier()
    launches0 = ctx.launches
    ctx.profile(True)
    clocks = Clocks(local)
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    infos = []
    for _ in range(args.steps):
        P, N, out = one_solve()
        infos.append(out[5])
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    log(f"timed solves done ({args.steps})")
    ms = e0.elapsed_time(e1) / args.steps
    prof = ctx.profile_read()
    ctx.profile(False)
    launches = ctx.launches - launches0
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t)
        torch.distributed.barrier()
    info = infos[-1]
    tile = N.tile()
    # the other precision, same steps, for the mixed-vs-FP64 comparison
    other = None
    if not args.no_compare:
        oprec = "fp64" if args.precision == "mixed" else "mixed"
        for _ in range(1):
            one_solve(oprec)
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        oinfo = None
        for _ in range(args.steps):
            _, _, oout = one_solve(oprec)
            oinfo = oout[5]
        e3.record(stream)
        torch.cuda.synchronize()
        oms = e2.elapsed_time(e3) / args.steps
        log(f"timed solves done ({oprec})")
        if world > 1:
            t = torch.tensor([oms], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            oms = float(t)
        other = {"precision": oprec, "time_to_map_s": round(oms / 1e3, 4), "iterations": oinfo.iterations,
                 "outer_iterations": oinfo.outer_iterations, "fp64_applications": oinfo.fp64_applications,
                 "converged": bool(oinfo.converged)}
    n_map = info.n_map
    ab = algorithmic_bytes(ns, n_map, tile["n_tiles"], tile["fft_n"] // 2)
    per = {k: (prof[k][0] / max(prof[k][1], 1)) for k in ("P", "Ninv", "Pt", "vec")}
    dom = max(("P", "Ninv", "Pt"), key=lambda k: per[k])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = ab[dom] / (per[dom] * 1e-3) / 1e9
    kname = {"P": "matvec_chunk_sums_kernel", "Ninv": ninv_kernel(tile, "double"),
             "Pt": "trmatvec_slices_kernel<double, double> + pt_partial_sum_kernel"}
    ninv_tile, ninv_prec = tile, "f64"
    if args.precision == "mixed":
        t32 = N.tile_fp32()
        ab = algorithmic_bytes32(ns, n_map, (t32["n_tiles"], t32["fft_n"] // 2))
        tile = {"fp64": tile, "fp32": t32}
        kname = {"P": "matvec32_chunk_sums4_kernel", "Ninv": ninv_kernel(t32, "float"),
                 "Pt": "trmatvec_slices_kernel<float, float> + pt_partial_sum_kernel"}
        ninv_tile, ninv_prec = t32, "f32"
        dom = max(("P", "Ninv", "Pt"), key=lambda k: per[k])
        achieved = ab[dom] / (per[dom] * 1e-3) / 1e9
    traffic = None
    if dom == "Ninv" and ninv_tile.get("split"):
        tpt = NINV_TRAFFIC_PER_TILE.get((ninv_prec, *ninv_tile["split"]))
        if tpt:
            traffic = int(tpt * ninv_tile["n_tiles"])
    roofline = {"bound": "hbm", "kernel": kname[dom],
                "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "traffic": traffic, "peak_source": "measured" if peaks else "fallback",
                "per_application_ms": {k: round(v, 4) for k, v in per.items()},
                "algorithmic_bytes": ab}
    if dom == "Ninv" and ninv_tile.get("split"):
        # what the ncu captures show about the split kernels
        roofline["limiter"] = ("not DRAM (1.8-2.7 TB/s of DRAM traffic, ~3x the algorithmic bytes from the "
                               "four-step scratch): instruction issue in the row and inverse-column passes (issue "
                               "slot ~65 % busy, top stall 'not selected') and load latency in the forward-column "
                               "pass (ncu)")

    # the reference's CPU path on a bounded sample (before any large host allocation)
    cpu = None
    if rank == 0 and not args.no_cpu and world == 1:
        log("cpu baseline: start")
        cpu = run_cpu_baseline(wl, cpu_sample(wl), REFERENCE_ITERATIONS, ns)
        log("cpu baseline: done")
    # pinned host inputs for the end-to-end run
    pinned = None
    if not args.no_e2e:
        pinned = {k: torch.empty(getattr(wl, k).numel(), dtype=getattr(wl, k).dtype, pin_memory=True)
                  for k in ("pix", "weights", "signal", "noise")}
        for k, v in pinned.items():
            v.copy_(getattr(wl, k))
    del P, N, infos
    wl.pix = wl.weights = wl.signal = wl.noise = None
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # end to end through the reference-facing API with host buffers
    e2e = None
    if pinned:
        try:
            log("e2e: start")
            e2e = run_e2e_device_api(args, wl, world, pinned)
            log("e2e (device API): done")
            # the reference's own entry point (MLmap: FP64, host maps out) on the same inputs
            e2e["mlmap_fp64"] = run_e2e(args, wl, world, pinned)
            log("e2e (MLmap_b200): done")
        except Exception as ex:  # noqa: BLE001 - reported on the line
            sys.stderr.write(f"e2e failed: {type(ex).__name__}: {ex}\n")
            e2e = dict(e2e or {"value": None, "unit": "s"}, error=f"{type(ex).__name__}: {ex}")
    pinned = None

    # multi-RHS and serving configurations (one GPU: rank 0 of a single-process run)
    multi = serve_out = fknee = None
    ctx.trim()
    c1 = None
    if world == 1 and not args.no_c1:
        c1 = run_part(bench_c1, args, local)
    if world == 1 and not args.no_fknee:
        fknee = run_part(bench_fknee, args, local)
    solvers = None
    if world == 1 and not args.no_solvers:
        solvers = run_part(bench_solvers, args, local)
    noise_part = None
    if world == 1 and not args.no_noise:
        noise_part = run_part(bench_noise2invtt, args, local)
    if world == 1 and not args.no_multi:
        multi = run_part(bench_multi, args, local)
    if world == 1 and not args.no_serve:
        serve_out = run_part(bench_serving, args, local)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms / 1e3 * 1.0, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": workload_config(args.config, 1),
            "solve": {"precision": args.precision, "unknowns": int(n_map), "iterations": info.iterations,
                      "outer_iterations": info.outer_iterations, "fp64_applications": info.fp64_applications,
                      "converged": bool(info.converged), "precond_s": round(info.precond_seconds, 4),
                      "solve_s": round(info.solve_seconds, 4), "fft_tile": tile},
            "roofline": roofline, "clocks": clk, "gpu_launches": int(launches),
        }
        if other:
            line["solve"]["fp64" if other["precision"] == "fp64" else "mixed"] = other
        if args.precision == "mixed":
            line["dtype"] = "f32 operator + f64 refinement"
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if c1:
            line["c1_reference"] = c1
        if fknee:
            line["mixed_fknee_sweep"] = fknee
        if solvers:
            line["solvers_low_fknee"] = solvers
        if noise_part:
            line["noise2invtt"] = noise_part
        if multi:
            line["multi_rhs"] = multi
        if serve_out:
            line["serving"] = serve_out
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_e2e_device_api(args, wl, world, pinned):
    """The headline solve end to end through the library's Python/C device API
    (midapack_b200.Pointing, Noise, gls_solve_mixed or gls_solve by --precision):
    each step copies the inputs from pinned host memory to the device, builds
    the operators, solves and reads the map back; max over ranks."""
    import torch
    import midapack_b200 as mb
    ctx = mb.Context(torch.cuda.current_device())
    nb = len(wl.block_sizes)
    idv = np.arange(nb, dtype=np.int64) * wl.block_len
    times, it = [], 0
    copy_stream = torch.cuda.Stream()
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # the pointing first (the compression needs only it); weights, signal and
        # noise follow on a second stream while the pointing is compressed and
        # the noise operator (spectra, tile plans) is built
        dev = {"pix": pinned["pix"].to("cuda", non_blocking=True)}
        with torch.cuda.stream(copy_stream):
            for k in ("weights", "signal", "noise"):
                dev[k] = pinned[k].to("cuda", non_blocking=True)
            copied = torch.cuda.Event()
            copied.record(copy_stream)
        P = mb.Pointing(ctx, dev["pix"], dev["weights"], wl.n_samples, 3)
        N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt, idv=idv)
        torch.cuda.current_stream().wait_event(copied)
        for k in ("weights", "signal", "noise"):
            dev[k].record_stream(torch.cuda.current_stream())
        if args.precision == "mixed":
            out = mb.gls_solve_mixed(ctx, P, N, dev["signal"], dev["noise"], tol=TOL, maxiter=MAXITER,
                                     inner_tol=args.inner_tol)
        else:
            out = mb.gls_solve(ctx, P, N, dev["signal"], dev["noise"], tol=TOL, maxiter=MAXITER)
        x = out[0].cpu()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        it = out[5].iterations
        P.close()
        N.close()
        del dev, out
    ctx.close()
    t = max(times) if times else 0.0
    if world > 1:
        tt_ = torch.tensor([t], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(tt_, op=torch.distributed.ReduceOp.MAX)
        t = float(tt_)
    h2d = sum(v.numel() * v.element_size() for v in pinned.values())
    return {"value": round(t, 4), "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(x.numel() * 8),
            "api": f"midapack_b200 Pointing + Noise + gls_solve{'_mixed' if args.precision == 'mixed' else ''} "
                   "from pinned host inputs", "iterations": it}


def run_e2e(args, wl, world, pinned):
    """MLmap_b200 (the MLmap solve, host buffers in and maps out) with pinned host inputs."""
    import torch
    import midapack_b200 as mb
    pix, w, s, n = pinned["pix"], pinned["weights"], pinned["signal"], pinned["noise"]
    npix = 12 * wl.nside * wl.nside
    maps = [np.zeros(npix) for _ in range(4)] + [np.zeros(npix, dtype=np.int32)]
    bs = np.ascontiguousarray(wl.block_sizes, dtype=np.int32)
    tt = np.ascontiguousarray(wl.invtt)
    it = mb.ct.c_int()
    rr = mb.ct.c_double()
    L = mb.lib()
    P = lambda t, ty: mb.ct.cast(mb.ct.c_void_p(t.data_ptr()), mb.ct.POINTER(ty))  # noqa: E731
    times = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        mb.check(L.MLmap_b200(0, 0, TOL, MAXITER, wl.nside, wl.n_samples, len(bs), bs.ctypes.data_as(mb.c_i32p), 3,
                              P(pix, mb.ct.c_int32), P(w, mb.ct.c_double), P(s, mb.ct.c_double),
                              P(n, mb.ct.c_double), wl.lam, tt.ctypes.data_as(mb.c_f64p),
                              *[m.ctypes.data_as(mb.c_f64p) for m in maps[:4]], maps[4].ctypes.data_as(mb.c_i32p),
                              mb.ct.byref(it), mb.ct.byref(rr)), "MLmap_b200")
        times.append(time.perf_counter() - t0)
    t = max(times) if times else 0.0
    if world > 1:
        tt_ = torch.tensor([t], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(tt_, op=torch.distributed.ReduceOp.MAX)
        t = float(tt_)
    h2d = pix.numel() * 4 + (w.numel() + s.numel() + n.numel()) * 8 + tt.nbytes + bs.nbytes
    d2h = 4 * npix * 8 + npix * 4
    del pix, w, s, n
    return {"value": round(t, 4), "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": "MLmap_b200 (MLmap solve, host buffers)", "iterations": it.value}


def host_cores() -> int:
    """Host threads this process may use (the reference runs one rank per core)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(wl):
    sample_dets = max(1, min(host_cores(), wl.n_det))
    per_det = wl.n_samp
    return (sample_dets, wl.pix[:3 * per_det * sample_dets].cpu().numpy(),
            wl.weights[:3 * per_det * sample_dets].cpu().numpy())


def run_cpu_baseline(wl, sample, iterations, ns):
    sample_dets, pix, w = sample
    per_det = wl.n_samp
    try:
        r = cpu_reference((pix, w, wl.block_sizes, wl.lam, wl.invtt, per_det), iterations, sample_dets, ns,
                          sample_dets)
    except Exception as ex:  # the baseline is reported, never required
        return {"value": None, "unit": "s", "cores": sample_dets, "kind": "reference", "sample": f"failed: {ex}"}
    if r is None:
        return None
    return {"value": round(r["time_to_map_s"], 2), "unit": "s", "cores": sample_dets, "kind": "reference",
            "sample": (f"reference C (oracle/_ref, shim FFT/MPI) P^T N^-1 P on {sample_dets} detector(s) x 2^24 samples "
                       f"as {sample_dets} forked ranks: {r['op_seconds_sample']:.2f} s per application; "
                       f"extrapolated x{ns // (per_det * sample_dets)} samples x {iterations + 1} applications on "
                       f"{sample_dets} cores")}


def run_sharded(args, wl, ctx, rank, world, local, idv):
    """One solve sharded over the ranks (midapack_b200.dist): each rank holds
    64 detectors x 2^24 samples (its own seeded scan of the same 2048x1536
    sky), one map-sized all-reduce per operator application; weak scaling (the
    job grows with the ranks).  Time per step = max over ranks."""
    import torch
    import torch.distributed as dist
    from midapack_b200.dist import GpuShard, ShardedGLS
    ns = wl.n_samples

    def one(precision):
        shard = GpuShard(ctx, wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, idv=idv)
        out = ShardedGLS(shard).solve(tol=TOL, maxiter=MAXITER, precision=precision, inner_tol=args.inner_tol)
        return shard, out

    def timed(precision, steps):
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream()
        e0.record(stream)
        last = None
        for _ in range(steps):
            shard, out = one(precision)
            shard.close()
            last = out
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1) / steps], dtype=torch.float64,
                         device="cuda" if dist.get_backend() == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t), last

    for _ in range(args.warmup):
        shard, _ = one(args.precision)
        shard.close()
    launches0 = ctx.launches
    clocks = Clocks(local)
    ms, out = timed(args.precision, args.steps)
    clk = clocks.stop()
    launches = ctx.launches - launches0
    info = out[4]
    other = None
    if not args.no_compare:
        oprec = "fp64" if args.precision == "mixed" else "mixed"
        oms, oout = timed(oprec, args.steps)
        other = {"precision": oprec, "time_to_map_s": round(oms / 1e3, 4), "iterations": oout[4].iterations,
                 "outer_iterations": oout[4].outer_iterations, "converged": bool(oout[4].converged)}
    # roofline: this rank's share of one operator application (P, N^-1, P^T), timed alone
    shard = GpuShard(ctx, wl.pix, wl.weights, wl.signal, wl.noise, wl.block_sizes, wl.lam, wl.invtt, idv=idv)
    n_loc = shard.P.shape()["n_map"]
    h = torch.randn(n_loc, dtype=torch.float64, device="cuda")
    fp32 = args.precision == "mixed"
    for _ in range(2):
        shard.apply(h, fp32)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        shard.apply(h, fp32)
    e1.record()
    torch.cuda.synchronize()
    op_ms = e0.elapsed_time(e1) / 3
    t = shard.N.tile_fp32() if fp32 else shard.N.tile()
    ab = (algorithmic_bytes32(ns, n_loc, (t["n_tiles"], t["fft_n"] // 2)) if fp32
          else algorithmic_bytes(ns, n_loc, t["n_tiles"], t["fft_n"] // 2))
    shard.close()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = sum(ab.values()) / (op_ms * 1e-3) / 1e9
    e2e = None if args.no_e2e else run_sharded_e2e(args, wl, ctx, world, idv)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms / 1e3, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 operator + f64 refinement" if fp32 else "f64",
            "data": "synthetic (seeded generator)",
            "config": workload_config(args.config, world),
            "solve": {"precision": args.precision, "unknowns": int(info.n_map), "iterations": info.iterations,
                      "outer_iterations": info.outer_iterations, "converged": bool(info.converged),
                      "exchange": f"one map all-reduce per operator application ({dist.get_backend()})"},
            "roofline": {"bound": "hbm", "kernel": "P^T N^-1 P, one rank's application "
                                                  f"({'FP32' if fp32 else 'FP64'} operator)",
                         "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "traffic": None,
                         "peak_source": "measured" if peaks else "fallback", "per_application_ms": round(op_ms, 4)},
            "clocks": clk, "gpu_launches": int(launches),
        }
        if other:
            line["solve"]["fp64" if other["precision"] == "fp64" else "mixed"] = other
        if e2e:
            line["e2e"] = e2e
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def run_sharded_e2e(args, wl, ctx, world, idv):
    """End to end at N GPUs through the sharded solve's public API: every rank
    copies its shard's inputs from pinned host memory to the device, builds its
    GpuShard and solves (the map comes back to the host), max over ranks.  All
    ranks take the same collective steps; when the node's host memory cannot
    hold every rank's pinned inputs, no rank runs it and the line says why."""
    import psutil
    import torch
    import torch.distributed as dist
    from midapack_b200.dist import GpuShard, ShardedGLS
    keys = ("pix", "weights", "signal", "noise")
    need = sum(getattr(wl, k).numel() * getattr(wl, k).element_size() for k in keys)
    ok = torch.tensor([1.0 if psutil.virtual_memory().available > 1.25 * need * world else 0.0],
                      dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    if float(ok) < 1.0:
        return {"value": None, "unit": "s", "skipped": f"host memory below {world} x {need / 2**30:.0f} GiB pinned"}
    pinned = {k: torch.empty(getattr(wl, k).numel(), dtype=getattr(wl, k).dtype, pin_memory=True) for k in keys}
    for k, v in pinned.items():
        v.copy_(getattr(wl, k))
    for k in keys:  # the device copies of the generator are not needed any more
        setattr(wl, k, None)
    ctx.trim()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    times = []
    for _ in range(args.e2e_steps):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev = {k: v.to("cuda", non_blocking=True) for k, v in pinned.items()}
        shard = GpuShard(ctx, dev["pix"], dev["weights"], dev["signal"], dev["noise"], wl.block_sizes, wl.lam,
                         wl.invtt, idv=idv)
        x = ShardedGLS(shard).solve(tol=TOL, maxiter=MAXITER, precision=args.precision,
                                    inner_tol=args.inner_tol)[0].cpu()
        shard.close()
        del dev
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t = torch.tensor([max(times)], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    del pinned
    return {"value": round(float(t), 4), "unit": "s", "h2d_bytes_per_step": int(need) * world,
            "d2h_bytes_per_step": int(x.numel() * 8) * world,
            "api": "midapack_b200.dist.ShardedGLS(GpuShard(...)).solve, host inputs (all ranks)"}


def run_reference(args, rank, world):
    """The reference arm: the reference's own C operator (oracle/_ref) on the
    host cores, on a bounded sample of the workload (W + K applications of
    P^T N^-1 P on as many detectors as host cores, one forked rank each; the
    last K timed), extrapolated to all detectors and REFERENCE_ITERATIONS + 1
    applications; beside it the reference's whole MLmap on the CPU-runnable
    workload, measured.  Rank 0 alone runs it; nothing here touches CUDA or
    loads this library."""
    if rank != 0:
        return 0
    from midapack_b200 import synth
    from oracle import cpu_baseline as cb
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference compiled from its "
                                                              "sources) is not built"}), flush=True)
        return 0
    cfg = synth.CONFIGS[args.config]
    cores = host_cores()
    sample = max(1, min(cores, cfg["n_det"]))
    times = cb.operator_sample(cfg, sample, max(args.warmup, 0) + max(args.steps, 1))
    timed = times[max(args.warmup, 0):]
    per_app = float(np.mean(timed))
    n_det_total = cfg["n_det"] * world
    # `sample` ranks ran at once on `cores` cores: the full operator is n_det_total/sample such rounds
    per_app_full = per_app * n_det_total / sample * (sample / min(cores, sample))
    v = per_app_full * (REFERENCE_ITERATIONS + 1)
    c1 = None
    try:
        c1cfg = dict(synth.CONFIGS["c1_4det_2p20_256x192_lam4096"], gap_frac=0.01)
        wl1 = synth.make_workload("c1", **c1cfg)
        t1, it1, _ = cb.mlmap_workload(wl1, 4, TOL, 4 * MAXITER)
        c1 = {"workload": "c1_4det_2p20_256x192_lam4096 + 1% flagged samples",
              "path": "reference MLmap (oracle/_ref, shim FFT/MPI/LAPACK), 4 forked host ranks, measured",
              "time_to_map_s": round(t1, 3), "iterations": it1, "ranks": 4}
    except Exception as ex:  # noqa: BLE001 - reported on the line
        c1 = {"error": f"{type(ex).__name__}: {ex}"}
    sample_txt = (f"reference C (oracle/_ref: the reference's sources, shim FFT/MPI) P^T N^-1 P on {sample} "
                  f"detector(s) x {cfg['n_samp']} samples as {sample} forked ranks, {len(timed)} timed applications "
                  f"after {len(times) - len(timed)} untimed: {per_app:.3f} s each; extrapolated x{n_det_total // sample}"
                  f" detectors x {REFERENCE_ITERATIONS + 1} applications")
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": "s", "n_gpus": world,
            "steps": len(timed), "warmup": len(times) - len(timed), "ms_per_step": round(v * 1e3, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)", "config": workload_config(args.config, world),
            "solve": {"precision": "fp64", "iterations": REFERENCE_ITERATIONS,
                      "iterations_source": "fixed: the at-scale FP64 PCG iteration count at tol 1e-8",
                      "seconds_per_application": round(per_app_full, 3),
                      "sample_application_s": [round(t, 4) for t in timed]},
            "cpu_baseline": {"value": round(v, 2), "unit": "s", "cores": min(cores, sample), "kind": "reference",
                             "sample": sample_txt},
            "c1_reference_mlmap": c1,
            "e2e": {"value": round(v, 2), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
