"""MTmap's solve on the device (mdp_gls_solve_templates: block Jacobi from the
white noise operator, the PCG_GLS_true recurrences with the template weighting
W - W T B T^T W) against the reference's own MTmap (oracle/_ref, one rank):
maps on the observed pixels within 1e-10, same cut, cond and hits, iteration
count +-1."""
import numpy as np
import pytest

from tests._cases import template_case

pytestmark = pytest.mark.gpu

VARIANTS = {
    "poly2_sss8_hwp2": dict(npoly=2, ground=1, n_sss_bins=8, nhwp=2),
    "poly3_only": dict(npoly=3, ground=0, n_sss_bins=0, nhwp=0),
    "poly1_hwp3": dict(npoly=1, ground=0, n_sss_bins=0, nhwp=3, delta_t=2.5),
}


@pytest.mark.parametrize("name", list(VARIANTS))
def test_mtmap_solve_matches_reference(gpu_ctx, ref_lib, name):
    import torch
    import midapack_b200 as mb
    from midapack_b200 import templates
    sc, pix, w, sig, noi, invtt, nside = template_case(**VARIANTS[name])
    I, Q, U, Cond, Hits, res = ref_lib.mtmap(sc, pix, w, sig, noi, invtt, nside, tol=1e-10, maxiter=500)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    wd = d(w)
    P = mb.Pointing(gpu_ctx, d(pix), wd, sig.size, 3)
    N = mb.Noise(gpu_ctx, sc.block_sizes, 1, invtt)
    scan = templates.Scan(sc.sweeps, sc.az, sc.az_min, sc.az_max, sc.hwp, sc.ndet, sc.npoly, sc.ground,
                          sc.n_sss_bins, sc.nhwp, sc.delta_t, sc.fs)
    F = templates.Filter(gpu_ctx, scan, invtt)
    x, lst, cond, hits, rr, info = templates.solve(gpu_ctx, P, N, F, d(sig), d(noi), tol=1e-10, maxiter=500)
    x, lst, cond, hits = x.cpu().numpy(), lst.cpu().numpy(), cond.cpu().numpy(), hits.cpu().numpy()
    assert abs(info.iterations - (len(res) - 1)) <= 1
    p = lst[0::3] // 3
    np.testing.assert_array_equal(hits, Hits[p])
    np.testing.assert_allclose(cond, Cond[p], rtol=1e-12)
    for k, ref_map in enumerate((I, Q, U)):
        mine = x[k::3]
        assert np.linalg.norm(mine - ref_map[p]) <= 1e-10 * np.linalg.norm(ref_map[p])


def test_mtmap_dropin_writes_the_reference_maps(gpu_ctx, ref_lib, tmp_path):
    """MTmap with the reference's C signature (include/mappraiser.h): its FITS maps
    against the reference's MTmap on the observed pixels."""
    import ctypes as ct
    import midapack_b200 as mb
    from midapack_b200 import mappraiser_wrapper as mw
    sc, pix, w, sig, noi, invtt, nside = template_case()
    I, Q, U, Cond, Hits, res = ref_lib.mtmap(sc, pix, w, sig, noi, invtt, nside, tol=1e-10, maxiter=500)
    ip, dp = ct.POINTER(ct.c_int), ct.POINTER(ct.c_double)
    sweeps = [np.ascontiguousarray(s, dtype=np.int32) for s in sc.sweeps]
    az = [np.ascontiguousarray(a, dtype=np.float64) for a in sc.az]
    hwp = [np.ascontiguousarray(h, dtype=np.float64) for h in sc.hwp]
    SW = (ip * sc.nces)(*[s.ctypes.data_as(ip) for s in sweeps])
    AZ = (dp * sc.nces)(*[a.ctypes.data_as(dp) for a in az])
    HW = (dp * sc.nces)(*[h.ctypes.data_as(dp) for h in hwp])
    nsw = np.array([len(s) - 1 for s in sweeps], dtype=np.int32)
    azmin = np.ascontiguousarray(sc.az_min, dtype=np.float64)
    azmax = np.ascontiguousarray(sc.az_max, dtype=np.float64)
    dsp = np.array([sig.size], dtype=np.int32)
    blocks = np.ascontiguousarray(sc.block_sizes, dtype=np.int32)
    px = np.ascontiguousarray(pix, dtype=np.int32)
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (w, sig, noi, invtt)]
    mb.lib().MTmap(0, str(tmp_path).encode(), b"run", 0, 0, 0, 6, sc.npoly, sc.nhwp, ct.c_double(sc.delta_t),
                   sc.ground, sc.n_sss_bins, ct.c_double(1e-10), 500, 0, 0, 0, nside, SW, nsw.ctypes.data_as(ip),
                   AZ, azmin.ctypes.data_as(dp), azmax.ctypes.data_as(dp), HW, sc.nces, dsp.ctypes.data_as(ip),
                   len(blocks), blocks.ctypes.data_as(ip), 3, px.ctypes.data_as(ip), arr[0].ctypes.data_as(dp),
                   arr[1].ctypes.data_as(dp), arr[2].ctypes.data_as(dp), ct.c_double(sc.fs),
                   arr[3].ctypes.data_as(dp))
    maps = [mw.read_fits_map(str(tmp_path / f"{k}_run.fits")) for k in ("mapI", "mapQ", "mapU", "Cond", "Hits")]
    obs = Hits > 0
    np.testing.assert_array_equal(maps[4], Hits)
    for mine, theirs in zip(maps[:3], (I, Q, U)):
        assert np.linalg.norm(mine[obs] - theirs[obs]) <= 1e-10 * np.linalg.norm(theirs[obs])
