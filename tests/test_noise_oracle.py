"""noise2invtt (mappraiser/python/TOAST_interface/utils.py:500-602): the
oracle restatement against the golden outputs of the reference's own function
(tests/golden/noise2invtt/make.py), and the argument checks of
midapack_b200.noise that run before any device work.  No GPU."""
import numpy as np
import pytest

from oracle import restate
from tests._cases import noise_golden

CASES = noise_golden()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_restatement_matches_reference_function(case):
    got, _, _ = restate.noise2invtt(case["noise"], case["n"], case["lam"], case["fsamp"], case["apod"])
    assert rel(got, case["invtt"]) <= 1e-12


@pytest.mark.parametrize("case", CASES[:4], ids=[c["name"] for c in CASES[:4]])
def test_tight_fit_within_reference_fit_tolerance(case):
    # the reference's curve_fit stops at ftol = 1e-8; run to the minimum the rows
    # differ by at most that tolerance's effect
    got, _, _ = restate.noise2invtt(case["noise"], case["n"], case["lam"], case["fsamp"], case["apod"], tight=True)
    assert rel(got, case["invtt"]) <= 1e-4


def test_window_restatement():
    from scipy.signal import get_window
    for lam in (8, 100):
        ref = np.fft.ifftshift(get_window(("chebwin", 150), 2 * lam))[:lam]
        assert np.array_equal(restate.apod_window(lam, "chebwin"), ref)


def test_host_argument_checks():
    from midapack_b200 import noise
    x = np.zeros(64)
    with pytest.raises(RuntimeError, match="Bandwidth cannot be larger than timestream"):
        noise.noise2invtt(x, 64, 33, 100.0, 0, np.float64, "chebwin")
    with pytest.raises(RuntimeError, match="not supported"):
        noise.noise2invtt(x, 64, 8, 100.0, 0, np.float64, "hamming")
    with pytest.raises(NotImplementedError):
        noise.noise2invtt(x, 64, 8, 100.0, 0, np.float64, "chebwin", save_psd=True)
    with pytest.raises(RuntimeError, match="Bandwidth"):
        noise.compute_invtt(1, 2, np.zeros(96), [64, 32], 17, 100.0, np.zeros(34), np.float64)
    with pytest.raises(ValueError, match="the blocks need 96"):
        noise.invtt_blocks(np.zeros(90), [64, 32], 8, 100.0)
    with pytest.raises(NotImplementedError):
        noise.noise2invtt(np.zeros(128), 64, 8, 100.0, 0, np.float64, "chebwin")   # several Welch segments
