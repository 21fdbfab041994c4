"""Request server on the GPU: requests solved concurrently (several slots,
overlapping on the device) give the same maps as each request solved alone
(one slot, one request at a time), within 1e-8 relative per I/Q/U map, and
the same maps as a direct library call."""
import numpy as np
import pytest

from midapack_b200.serve import DatasetSpec, GpuExecutor, Request, Server

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# grids with width*height not near a multiple of the 25-sample half-wave-plate
# period (a lone detector then sees several angles per pixel)
SPECS = [DatasetSpec("s0", 2, 8192, 32, 24, 64, 1.0, 0.02, 1),
         DatasetSpec("s1", 3, 4096, 48, 36, 128, 2.5, 0.02, 2),
         DatasetSpec("s2", 1, 16384, 40, 31, 300, 0.3, 0.02, 3)]


def _serve(reqs, slots):
    srv = Server(GpuExecutor(), slots=slots, work_budget=8 << 30, dataset_budget=8 << 30)
    for s in SPECS:
        srv.preload(s)
    if slots == 1:
        out = [srv.submit(Request(r.rid, r.spec, r.noise_seed, r.precision, r.tol)).wait(600) for r in reqs]
    else:
        tickets = [srv.submit(Request(r.rid, r.spec, r.noise_seed, r.precision, r.tol)) for r in reqs]
        out = [t.wait(600) for t in tickets]
    peak = srv.max_running
    srv.close()
    return out, peak


def test_results_same_alone_and_in_the_mix():
    reqs = [Request(i, SPECS[i % 3], noise_seed=100 + i, precision="mixed" if i % 4 else "fp64", tol=1e-10)
            for i in range(9)]
    mix, peak = _serve(reqs, slots=4)
    alone, _ = _serve(reqs, slots=1)
    assert peak >= 2
    for a, b in zip(mix, alone):
        assert a.error is None and b.error is None, (a.error, b.error)
        assert a.converged and b.converged
        assert np.array_equal(a.lstid, b.lstid)
        for k in range(3):
            assert _rel(a.x[k::3], b.x[k::3]) < 1e-8, (a.rid, k)


def test_served_map_matches_direct_call():
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    spec = SPECS[1]
    (res,), _ = _serve([Request(0, spec, noise_seed=7, tol=1e-10)], slots=2)
    wl = synth.make_workload_torch(spec.key, spec.width, spec.height, spec.n_det, spec.n_samp, spec.n_samp,
                                   spec.lam, spec.fknee, spec.seed, spec.gap_frac)
    noise = synth.mc_noise_torch(spec.n_det, spec.n_samp, 1, spec.fknee, seed=7)[0].double()
    ctx = mb.Context(0)
    P = mb.Pointing(ctx, wl.pix, wl.weights, wl.n_samples, 3)
    N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
    x, lst, *_ = mb.gls_solve_mixed(ctx, P, N, wl.signal, noise, tol=1e-10)
    x = x.cpu().numpy()
    assert np.array_equal(lst.cpu().numpy(), res.lstid)
    for k in range(3):
        assert _rel(res.x[k::3], x[k::3]) < 1e-8
