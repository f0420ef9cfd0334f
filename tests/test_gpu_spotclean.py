"""MorphSpotClean on the GPU against the oracle (gpu). Reconstructions and threshold
replacement are min/max/compare only: bit-exact. The sigmoid blend uses expf (CUDA vs
glibc may differ by an ulp), so it is compared within a few ulp of the image scale."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))
DET = {"holes": 0, "peaks": 1, "both": 2}


def gpu_clean(img, detect, conn8, th, sigma, edge=9, clamp=False, lo=-0.1, hi=7.0, infnan=False):
    t = torch.from_numpy(np.ascontiguousarray(img, np.float32)).cuda()
    M.morph_spot_clean(t, DET[detect], conn8, th, sigma, edge, clamp, lo, hi, infnan)
    out = t.cpu().numpy()
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    assert st.value == 0
    return out


def close(a, b, sigma):
    if sigma == (0.0, 0.0):
        return np.array_equal(a, b)
    scale = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(a.astype(np.float64) - b).max()) <= 8 * np.spacing(np.float32(scale))


@pytest.mark.parametrize("detect", ["holes", "peaks", "both"])
@pytest.mark.parametrize("conn8", [True, False])
@pytest.mark.parametrize("sigma", [(0.0, 0.0), (0.05, 0.02)])
def test_random_images(cuda, detect, conn8, sigma):
    rng = np.random.default_rng(80)
    for t in range(4):
        h, w = rng.integers(5, 60, 2)
        stack = rng.standard_normal((3, h, w)).astype(np.float32)
        if t % 2:
            stack = np.round(stack * 3).astype(np.float32)
        e = int(rng.choice([3, 5, 9]))
        got = gpu_clean(stack, detect, conn8, (0.5, 0.4), sigma, edge=e)
        exp = O.morphspotclean(stack, detect, conn8, (0.5, 0.4), sigma, edge=e)
        assert close(got, exp, sigma), (h, w, e)


def test_spot_projection_golden(cuda):
    got = gpu_clean(G["spot_input"], "holes", True, (0.3, 0.3), (0.01, 0.01))
    assert close(got, G["spot_holes_03_001"], (0.01, 0.01))
    assert np.isclose(got.mean(), 5.89322, rtol=1e-4) and np.isclose(got.std(), 22.368868, rtol=1e-4)
    got = gpu_clean(G["spot_input"], "peaks", False, (0.1, 0.1), (0.0, 0.0))
    assert np.array_equal(got, G["spot_peaks_conn4_thr"])
    got = gpu_clean(G["spot_input"], "both", True, (1.0, 1.0), (0.05, 0.05))
    assert close(got, G["spot_both_conn8_sig"], (0.05, 0.05))


def test_kat_fixture(cuda):
    for d in ("holes", "peaks", "both"):
        got = gpu_clean(G["kat_input"], d, True, (1.0, 1.0), (0.05, 0.05))
        assert close(got, G[f"kat_{d}"], (0.05, 0.05))


def test_wide_and_tall_images(cuda):
    """Rows longer than the 1024-thread CTA (several pixels per thread) and tall images."""
    rng = np.random.default_rng(81)
    img = (np.cumsum(rng.standard_normal((2, 40, 2600)), axis=2) * 0.05).astype(np.float32)
    img[0, 10, 100] += 50
    img[1, 20, 2000] -= 50
    for d in ("holes", "peaks", "both"):
        got = gpu_clean(img, d, True, (0.5, 0.5), (0.0, 0.0))
        assert np.array_equal(got, O.morphspotclean(img, d, True, (0.5, 0.5), (0.0, 0.0)))
    tall = rng.standard_normal((1, 700, 20)).astype(np.float32)
    got = gpu_clean(tall, "peaks", False, (0.5, 0.5), (0.0, 0.0))
    assert np.array_equal(got, O.morphspotclean(tall, "peaks", False, (0.5, 0.5), (0.0, 0.0)))


@pytest.mark.parametrize("conn8", [True, False])
def test_noisy_profile_worklist_completion(cuda, conn8):
    """A smooth attenuation profile with noise and spots: the row sweeps alone would need many
    rounds (paths wind up and down through the noise), so most of the reconstruction is done by
    the worklist completion, whose list overflows into dense passes at first."""
    rng = np.random.default_rng(84)
    h, w = 96, 700
    yy, xx = np.mgrid[:h, :w]
    base = 1.5 * np.exp(-((xx - 350) / 200.0) ** 2 - ((yy - 48) / 60.0) ** 2)
    img = (base + rng.normal(0, 0.03, (2, h, w))).astype(np.float32)
    img[0, 30, 100] += 1.0
    img[1, 60, 500] -= 1.0
    for d in ("holes", "peaks", "both"):
        got = gpu_clean(img, d, conn8, (0.1, 0.1), (0.0, 0.0), edge=5)
        assert np.array_equal(got, O.morphspotclean(img, d, conn8, (0.1, 0.1), (0.0, 0.0), edge=5)), d


@pytest.mark.parametrize("edge", [1, 2, 3, 4, 5, 6, 7, 8, 9, 11])
def test_edge_smoothing_lengths(cuda, edge):
    """The sliding in-place median along the first and last padded rows at every length (3, 5, 7
    and 9 run in registers with a sorting network, the others the reference's insertion sort),
    on values with many ties and zeros of both signs."""
    rng = np.random.default_rng(85 + edge)
    img = (np.round(rng.standard_normal((2, 24, 90)) * 2) / 2).astype(np.float32)
    img[img == 0] = np.where(rng.random(int((img == 0).sum())) < 0.5, -0.0, 0.0).astype(np.float32)
    for d in ("holes", "both"):
        got = gpu_clean(img, d, True, (0.3, 0.3), (0.0, 0.0), edge=edge)
        assert np.array_equal(got, O.morphspotclean(img, d, True, (0.3, 0.3), (0.0, 0.0), edge=edge)), d


def test_clamp_and_infnan(cuda):
    rng = np.random.default_rng(82)
    img = (rng.standard_normal((2, 12, 20)) * 5).astype(np.float32)
    img[0, 3, 4] = np.inf
    img[1, 7, 9] = np.nan
    got = gpu_clean(img, "peaks", True, (0.5, 0.5), (0.0, 0.0), clamp=True, lo=-2, hi=3, infnan=True)
    exp = O.morphspotclean(img, "peaks", True, (0.5, 0.5), (0.0, 0.0), clamp=True, minlevel=-2, maxlevel=3,
                           removeinfnan=True)
    assert np.array_equal(got, exp)


def test_module_interface(cuda):
    rng = np.random.default_rng(83)
    proj = (rng.standard_normal((5, 16, 24)) * 0.2 + 1).astype(np.float32)
    proj[:, 5, 7] = 5.0
    mod = M.MorphSpotCleanModule()
    assert mod.Configure(M.ReconConfig(), {"connectivity": "conn4", "cleanmethod": "morphcleanreplace",
                                           "detectionmethod": "morphdetectpeaks", "threshold": "0.1 0.1",
                                           "sigma": "0 0", "edgesmooth": "5", "maxarea": "30",
                                           "removeinfnan": "false", "clampdata": "false", "minlevel": "-0.1",
                                           "maxlevel": "7", "threading": "false"}) == 0
    got = mod.Process(torch.from_numpy(proj).cuda()).cpu().numpy()
    assert np.array_equal(got, O.morphspotclean(proj, "peaks", False, (0.1, 0.1), (0.0, 0.0), edge=9))
    assert mod.Configure(M.ReconConfig(), {"connectivity": "conn5"}) == -1


def test_rejects_short_images(cuda):
    t = torch.zeros((1, 4, 10), device=cuda)
    with pytest.raises(L.MrError):
        M.morph_spot_clean(t)
