"""SpotClean2 on the GPU (gpu): mr_spotclean2 against the oracle's restatement of
ImagingAlgorithms::SpotClean (pinned against the compiled reference module on the CPU), bit
for bit: every detection method, region exclusion on and off, iterations, the smallest and
ragged sizes, a block filtered in two batches, the single-image path, and an image that is all
spots."""
import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M

from test_ringalt_pins import spot_phantom

pytestmark = pytest.mark.gpu

METHODS = ["ring", "median", "minmax", "stddev", "trikernel"]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _module(method, gamma, sigma, it, maxarea, minlevel=-0.1, maxlevel=5.0):
    mod = M.SpotClean2()
    mod.Configure(M.ReconConfig(), {"gamma": str(gamma), "sigma": str(sigma), "iterations": str(it),
                                    "maxlevel": str(maxlevel), "minlevel": str(minlevel), "maxarea": str(maxarea),
                                    "detectionmethod": method})
    return mod


@pytest.mark.parametrize("method", METHODS)
def test_spotclean2_matches_oracle(cuda, method):
    rng = np.random.default_rng(3 + len(method))
    for n, h, w in ((3, 16, 16), (4, 23, 37), (3, 96, 130), (2, 256, 300)):
        p = spot_phantom(rng, n, h, w)
        for gamma, sigma, maxarea, it in ((0.1, 0.001, 20, 1), (0.05, 0.01, 0, 2), (0.2, 0.005, 5, 1)):
            t = torch.from_numpy(p).cuda()
            _module(method, gamma, sigma, it, maxarea).Process(t)
            exp = O.spotclean2(p, method, gamma, sigma, it, -0.1, 5.0, maxarea)
            assert np.array_equal(_bits(t.cpu().numpy()), _bits(exp)), (method, n, h, w, gamma, sigma, maxarea, it)


def test_spotclean2_large_regions_and_background_rule(cuda):
    """Dense detections (noisy background): components far larger than maxarea, many small
    ones, and the flood from the last background pixel."""
    rng = np.random.default_rng(17)
    p = (0.3 + rng.normal(0, 0.05, (3, 64, 80))).astype(np.float32)
    p[0, 63, 79] = 2.0
    for maxarea in (3, 20, 200):
        t = torch.from_numpy(p).cuda()
        _module("ring", 0.1, 0.01, 1, maxarea).Process(t)
        assert np.array_equal(_bits(t.cpu().numpy()), _bits(O.spotclean2(p, "ring", 0.1, 0.01, 1, -0.1, 5.0, maxarea)))


def test_spotclean2_two_batches(cuda):
    """60 projections of 1024 x 1024: 53 per batch at five scratch images per projection, so the
    last 7 go through a second batch. Projections are independent, so the oracle checks four."""
    rng = np.random.default_rng(23)
    p = spot_phantom(rng, 60, 1024, 1024, density=0.0005)
    t = torch.from_numpy(p).cuda()
    _module("ring", 0.1, 0.001, 1, 20).Process(t)
    got = t.cpu().numpy()
    for i in (0, 52, 53, 59):
        exp = O.spotclean2(p[i:i + 1], "ring", 0.1, 0.001, 1, -0.1, 5.0, 20)
        assert np.array_equal(_bits(got[i]), _bits(exp[0])), i


def test_spotclean2_single_image_cleans_once(cuda):
    rng = np.random.default_rng(5)
    p = spot_phantom(rng, 1, 40, 50)
    t = torch.from_numpy(p[0].copy()).cuda()
    _module("median", 0.05, 0.01, 3, 0).Process(t)
    assert np.array_equal(_bits(t.cpu().numpy()), _bits(O.spotclean2(p, "median", 0.05, 0.01, 1, -0.1, 5.0, 0)[0]))


def test_spotclean2_every_pixel_a_spot(cuda):
    """Every pixel above maxlevel: all are spots. The last pixel's right neighbour is the value
    past the image end (0, unmarked), so the fill starts there and reaches every pixel; the
    second image also starts from its one unmarked pixel."""
    p = np.full((2, 20, 24), 9.0, np.float32)
    p[1, 3, 5] = 0.5
    t = torch.from_numpy(p).cuda()
    _module("ring", 0.1, 0.001, 1, 20).Process(t)
    assert np.array_equal(_bits(t.cpu().numpy()), _bits(O.spotclean2(p, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20)))
