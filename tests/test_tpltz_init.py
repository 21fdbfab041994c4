"""The drop-in Toeplitz set-up calls against the reference's own compiled code
(oracle/_ref): define_blocksize (toeplitz.c:168-253) on the host, and, on the
GPU, tpltz_init with its circulant spectrum (toeplitz.c:298-367, circ_init_fftw
441-470), tpltz_cleanup (485-498) and apply_weights (pcg_true.c:578-600)."""
import ctypes as ct

import numpy as np
import pytest

from midapack_b200 import synth

# (n, lambda): powers of two, odd bands, matrices smaller than 4 lambda
SHAPES = [(1 << 20, 4096), (1 << 20, 16384), (1 << 20, 100), (5000, 2000), (300, 100), (1 << 16, 1), (12000, 8192),
          (65536, 3000), (2 ** 24, 16384)]


@pytest.mark.parametrize("flag", [0, 1, 2, 3, 4, 5])
def test_define_blocksize_matches_reference(ref_lib, flag):
    import midapack_b200 as mb
    L = mb.lib()
    for n, lam in SHAPES:
        fixed = 3 * lam + 7
        assert L.define_blocksize(n, lam, flag, fixed) == ref_lib.define_blocksize(n, lam, flag, fixed), (n, lam)


def test_define_blocksize_flag6_minimum():
    """bs_flag 6: the smallest power of two >= 4 lambda, at least 2^14 (the
    reference's comment); its code compares the exponent with 2^14 instead
    (toeplitz.c:229-234), which overflows the power, so its value is not used."""
    import midapack_b200 as mb
    L = mb.lib()
    assert L.define_blocksize(1 << 20, 100, 6, 0) == 1 << 14
    assert L.define_blocksize(1 << 20, 8192, 6, 0) == 1 << 15
    assert L.define_blocksize(1000, 100, 6, 0) == 400


def _our_tpltz_init(n, lam, T, flag_bs=0, fixed_bs=0, flag_nfft=0, fixed_nfft=0):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Flag
    L = mb.lib()
    fl = Flag()
    L.flag_stgy_init_auto(ct.byref(fl))
    fl.flag_bs, fl.fixed_bs, fl.flag_nfft, fl.fixed_nfft = flag_bs, fixed_bs, flag_nfft, fixed_nfft
    tt = np.ascontiguousarray(T, dtype=np.float64).copy()
    nfft, bs = ct.c_int(0), ct.c_int(0)
    tf, vf, vr, pf, pb = (ct.c_void_p() for _ in range(5))
    L.tpltz_init.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                             ct.c_void_p, ct.c_void_p, ct.c_void_p, Flag]
    L.tpltz_cleanup.argtypes = [ct.c_void_p] * 5
    rc = L.tpltz_init(n, lam, ct.byref(nfft), ct.byref(bs), ct.byref(tf), tt.ctypes.data_as(ct.c_void_p),
                      ct.byref(vf), ct.byref(vr), ct.byref(pf), ct.byref(pb), fl)
    assert rc == 0
    h = bs.value // 2 + 1
    F = np.ctypeslib.as_array(ct.cast(tf, ct.POINTER(ct.c_double)), shape=(2 * h,)).copy()
    assert vf.value and vr.value and pf.value and pb.value
    assert L.tpltz_cleanup(ct.byref(tf), ct.byref(vf), ct.byref(vr), ct.byref(pf), ct.byref(pb)) == 0
    assert not (tf.value or vf.value or vr.value or pf.value or pb.value)
    return nfft.value, bs.value, F[0::2] + 1j * F[1::2]


@pytest.mark.gpu
@pytest.mark.parametrize("n,lam,flag_bs,fixed_bs", [(1 << 20, 4096, 0, 0), (1 << 20, 16384, 0, 0), (12000, 8192, 0, 0),
                                                    (1 << 20, 300, 2, 0), (1 << 20, 300, 3, 0), (1 << 20, 300, 5, 0),
                                                    (1 << 20, 300, 1, 4096), (1 << 16, 1, 0, 0)])
def test_tpltz_init_matches_reference(gpu_ctx, ref_lib, n, lam, flag_bs, fixed_bs):
    T = synth.invtt_row(max(n, 2 * lam), lam, 1.0) if lam > 1 else np.array([2.5])
    nf_r, bs_r, F_r = ref_lib.tpltz_init(n, lam, T, flag_bs=flag_bs, fixed_bs=fixed_bs)
    nf, bs, F = _our_tpltz_init(n, lam, T, flag_bs=flag_bs, fixed_bs=fixed_bs)
    assert (nf, bs) == (nf_r, bs_r)
    scale = np.linalg.norm(F_r)
    assert np.linalg.norm(F.real - F_r.real) <= 1e-12 * scale
    # the embedding is even: the spectrum is real (the reference's r2c leaves round-off there)
    assert np.abs(F.imag).max() <= 1e-12 * np.abs(F_r).max()
    assert np.abs(F_r.imag).max() <= 1e-12 * np.abs(F_r).max()


@pytest.mark.gpu
def test_tpltz_init_nfft_and_odd_blocksize(gpu_ctx):
    """fixed nfft, and a block size that is not a power of two (bs = 4 lambda
    when the matrix is shorter than the power of two): the spectrum is the DFT
    of the embedding c[0] = T0, c[i] = c[bs-i] = T[i], checked directly."""
    lam, n = 100, 300
    T = np.exp(-np.arange(lam) / 17.0)
    nf, bs, F = _our_tpltz_init(n, lam, T, flag_nfft=1, fixed_nfft=3)
    assert nf == 3 and bs == 400
    c = np.zeros(bs)
    c[0] = T[0]
    c[1:lam] = T[1:]
    c[bs - np.arange(1, lam)] = T[1:]
    ref = np.fft.rfft(c)
    assert np.abs(F - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("lam", [1, 64, 2048])
def test_apply_weights_matches_reference(gpu_ctx, ref_lib, lam):
    import midapack_b200 as mb
    from midapack_b200.mappraiser_wrapper import Block, Flag, Tpltz
    L = mb.lib()
    bs = np.array([8192, 5000, 12000], dtype=np.int32)
    rows = [synth.invtt_row(8192 * 2, lam, fk) if lam > 1 else np.array([0.5 + fk]) for fk in (0.5, 1.0, 3.0)]
    invtt = np.concatenate(rows)
    tod = np.random.default_rng(lam).standard_normal(int(bs.sum()))
    ref = ref_lib.apply_weights(bs, lam, invtt, tod)
    nb = len(bs)
    blocks = (Block * nb)()
    L.defineBlocks_avg(blocks, invtt.ctypes.data_as(ct.POINTER(ct.c_double)), nb, bs.ctypes.data_as(ct.c_void_p),
                       lam, 0)
    T = Tpltz()
    f = Flag()
    L.flag_stgy_init_auto(ct.byref(f))
    L.defineTpltz_avg.argtypes = [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int,
                                  ct.c_int64, ct.c_int, Flag, ct.c_int]
    L.defineTpltz_avg(ct.byref(T), int(bs.sum()), 1, 1, blocks, nb, nb, 0, int(bs.sum()), f, 0x44000000)
    out = tod.copy()
    assert L.apply_weights(ct.byref(T), out.ctypes.data_as(ct.POINTER(ct.c_double))) == 0
    assert np.linalg.norm(out - ref) <= 1e-12 * np.linalg.norm(ref)
