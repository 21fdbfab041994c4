"""The allocation-free N^-1 entry point (mdp_stbmm_noalloc), called through
the C ABI, against the regular entry point (mdp_stbmm) on the same inputs.

It exists for callers that cannot allocate device memory while they apply the
noise operator (a memory arena or pool owning all device memory, a solve loop
that must not let cudaMalloc/cudaFree synchronise the device, a plugin that
may only use the buffers its host hands it).  Its scratch is a fixed array
shared by every call, so two calls in a row must each give the regular
result: the second call must not see anything left by the first.  This file
is collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the tolerance of the N^-1 parity tests


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_matches_regular_two_calls(gpu_ctx):
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    L = mb.lib()
    lam = 512
    sizes = [200000, 150001, 70000]  # several 65536-row chunks per block
    invtt = np.concatenate([synth.invtt_row(1 << 16, lam, fk) for fk in (1.0, 0.3, 2.0)])
    N = mb.Noise(gpu_ctx, sizes, lam, invtt)
    rng = np.random.default_rng(17)
    for call in range(2):
        v = torch.from_numpy(rng.standard_normal(sum(sizes)) * (10.0 ** call) + 5.0 * call).cuda()
        ref = torch.empty_like(v)
        out = torch.full_like(v, np.nan)
        N.apply(v, ref)
        rc = L.mdp_stbmm_noalloc(gpu_ctx.h, N.h, ct.c_void_p(v.data_ptr()), ct.c_void_p(out.data_ptr()))
        assert rc == 0, L.mdp_last_error().decode()
        torch.cuda.synchronize()
        assert _rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL


@pytest.mark.parametrize("case", ["gaps_between_blocks", "white"])
def test_noalloc_gapped_and_white_operators(gpu_ctx, case):
    """Blocks that leave rows uncovered (those rows pass through unchanged, a copy
    made before the blocks are applied) and the white-noise operator (lambda 1,
    no mean removal), each twice in a row against mdp_stbmm."""
    import torch
    import midapack_b200 as mb
    from midapack_b200 import synth
    L = mb.lib()
    if case == "white":
        sizes, idv, lam = [5000, 7000], [0, 5000], 1
        invtt = np.array([0.7, 2.5])
    else:
        sizes, idv, lam = [70000, 20000], [1000, 90000], 256
        invtt = np.concatenate([synth.invtt_row(1 << 15, lam, fk) for fk in (1.0, 0.4)])
    nrow = idv[-1] + sizes[-1]
    N = mb.Noise(gpu_ctx, sizes, lam, invtt, idv=np.array(idv, dtype=np.int64))
    rng = np.random.default_rng(23)
    for call in range(2):
        v = torch.from_numpy(rng.standard_normal(nrow) + 3.0 * call).cuda()
        ref = torch.full_like(v, np.nan)
        out = torch.full_like(v, np.nan)
        N.apply(v, ref)
        rc = L.mdp_stbmm_noalloc(gpu_ctx.h, N.h, ct.c_void_p(v.data_ptr()), ct.c_void_p(out.data_ptr()))
        assert rc == 0, L.mdp_last_error().decode()
        torch.cuda.synchronize()
        o, r = out.cpu().numpy(), ref.cpu().numpy()
        covered = np.zeros(nrow, dtype=bool)
        for s0, n in zip(idv, sizes):
            covered[s0:s0 + n] = True
        assert np.isfinite(o[covered]).all() and _rel(o[covered], r[covered]) < TOL
        assert np.array_equal(o[~covered], r[~covered]) and np.array_equal(o[~covered], v.cpu().numpy()[~covered])


def test_noalloc_rejects_in_place_and_oversize(gpu_ctx):
    import torch
    import midapack_b200 as mb
    L = mb.lib()
    N = mb.Noise(gpu_ctx, [1000], 8, np.linspace(1.0, 0.1, 8))
    v = torch.zeros(1000, dtype=torch.float64, device="cuda")
    assert L.mdp_stbmm_noalloc(gpu_ctx.h, N.h, ct.c_void_p(v.data_ptr()), ct.c_void_p(v.data_ptr())) != 0
    nb = 140000  # one double per block plus one per chunk exceeds the 131072-double array
    big = mb.Noise(gpu_ctx, [2] * nb, 2, np.tile([1.0, 0.25], nb))
    a = torch.zeros(2 * nb, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    assert L.mdp_stbmm_noalloc(gpu_ctx.h, big.h, ct.c_void_p(a.data_ptr()), ct.c_void_p(b.data_ptr())) != 0
    assert b"limit" in L.mdp_last_error()
