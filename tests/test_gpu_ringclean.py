"""Wavelet-FFT ring cleaning on the GPU against the oracle (gpu). The DWT/IDWT arithmetic is
the reference's operation for operation; the FFT of the stripe damping is float on the GPU
and FP64 in the oracle, so results agree within 1e-5 relative RMS (measured far below)."""
import os

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))


def relrms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def gpu_stripe(s, name, levels, sigma):
    t = torch.from_numpy(np.ascontiguousarray(s, np.float32)).cuda()
    M.stripe_filter(t, name, levels, sigma)
    return t.cpu().numpy()


def test_woodsino_mse(cuda):
    wood = G["wood_input"]
    out = gpu_stripe(wood, "daub7", 2, 0.1)
    exp = O.stripefilter(wood, "daub7", 2, 0.1)
    assert relrms(out - wood, exp - wood) < 1e-4  # the removed stripe component itself
    assert relrms(out, exp) < 1e-6
    mse = float(((wood - out) ** 2).mean())
    assert np.isclose(mse, 1.8129678e-05, rtol=1e-4)


@pytest.mark.parametrize("name,levels,sigma", [("daub2", 1, 0.05), ("daub3", 3, 0.02), ("daub7", 2, 0.1),
                                               ("daub15", 2, 0.05), ("daub5", 3, 0.2), ("daub20", 2, 0.05)])
def test_random_sinograms(cuda, name, levels, sigma):
    rng = np.random.default_rng(95)
    h, w = 97, 131
    s = rng.standard_normal((3, h, w)).astype(np.float32)
    s += np.linspace(0, 1, w, dtype=np.float32)[None, None, :] * 0.3  # stripes
    out = gpu_stripe(s, name, levels, sigma)
    exp = np.stack([O.stripefilter(x, name, levels, sigma) for x in s])
    assert relrms(out, exp) < 1e-5


def test_golden_crops(cuda):
    crop = G["wood_input"][100:260, 50:250]
    assert relrms(gpu_stripe(crop, "daub15", 2, 0.05), G["wood_crop_daub15_2_005"]) < 1e-5
    assert relrms(gpu_stripe(crop, "daub3", 3, 0.02), G["wood_crop_daub3_3_002"]) < 1e-5


def test_module_on_projections(cuda):
    rng = np.random.default_rng(96)
    proj = rng.standard_normal((90, 5, 64)).astype(np.float32)
    proj += (rng.uniform(-0.05, 0.05, 64).astype(np.float32))[None, None, :]  # ring-producing column offsets
    mod = M.WaveletRingClean()
    mod.Configure(M.ReconConfig(), {"wname": "daub7", "sigma": "0.1", "decnum": "2", "parallel": "false",
                                    "method": "verticalfft"})
    out = mod.Process(torch.from_numpy(proj).cuda()).cpu().numpy()
    assert relrms(out, O.waveletringclean(proj, "daub7", 2, 0.1)) < 1e-5


def test_rejects_small_images(cuda):
    t = torch.zeros((1, 8, 8), device=cuda)
    with pytest.raises(Exception):
        M.stripe_filter(t, "daub15", 2, 0.05)
