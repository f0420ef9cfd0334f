"""Alternative ring cleaners on the GPU (gpu): mr_median_filter, mr_basicringclean and
mr_medianmixringclean against the oracle's restatements (pinned against the reference's own
modules on the CPU), bit for bit: every kernel size, the minimal image sizes, ragged sizes
that miss the vectorised paths, NaN / signed zeros / infinities (the heap-sort fallback), and a
block large enough to be filtered in two batches."""
import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu

KERNELS = [(1, 1), (3, 1), (1, 3), (3, 3), (5, 1), (1, 5), (5, 3), (3, 5), (5, 5)]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _special(rng, shape):
    img = rng.integers(-2, 3, shape).astype(np.float32)
    z = rng.random(shape) < 0.3
    img[z] = np.where(rng.random(z.sum()) < 0.5, np.float32(0.0), np.float32(-0.0))
    flat = img.reshape(-1)
    k = max(1, flat.size // 97)
    flat[rng.integers(0, flat.size, k)] = np.nan
    flat[rng.integers(0, flat.size, k)] = np.inf
    flat[rng.integers(0, flat.size, k)] = -np.inf
    return img


@pytest.mark.parametrize("kx,ky", KERNELS)
def test_median_filter_matches_oracle(cuda, kx, ky):
    rng = np.random.default_rng(kx * 7 + ky)
    for h, w in ((max(1, 2 * (ky // 2)), max(1, 2 * (kx // 2))), (5, 7), (19, 33), (64, 130), (8, 257)):
        stack = rng.standard_normal((3, h, w)).astype(np.float32)
        stack[1] = _special(rng, (h, w))
        got = M.median_filter(torch.from_numpy(stack).cuda(), kx, ky).cpu().numpy()
        for i in range(3):
            assert np.array_equal(_bits(got[i]), _bits(O.median_filter(stack[i], kx, ky))), (h, w, i)


@pytest.mark.parametrize("kx,ky", [(3, 3), (5, 5)])
def test_median_filter_zero_and_nan_windows(cuda, kx, ky):
    """Mostly zeros of both signs: most middles are a zero, so the sign rule and the heap sort
    decide nearly every pixel."""
    rng = np.random.default_rng(11 + kx)
    img = np.where(rng.random((48, 70)) < 0.5, np.float32(0.0), np.float32(-0.0)).astype(np.float32)
    img[rng.random(img.shape) < 0.1] = 1.0
    img[rng.random(img.shape) < 0.02] = np.nan
    got = M.median_filter(torch.from_numpy(img).cuda(), kx, ky).cpu().numpy()
    assert np.array_equal(_bits(got), _bits(O.median_filter(img, kx, ky)))


@pytest.mark.parametrize("shape", [(5, 2, 2), (9, 33, 41), (30, 64, 130), (16, 128, 256)])
def test_basicringclean_matches_oracle(cuda, shape):
    rng = np.random.default_rng(sum(shape))
    p = (rng.random(shape) * 2).astype(np.float32)
    p[:, :, shape[2] // 2] += 0.05
    p[0, 0, 0] = -0.0
    t = torch.from_numpy(p).cuda()
    M.BasicRingClean().Process(t)
    assert np.array_equal(_bits(t.cpu().numpy()), _bits(O.basicringclean(p)))


@pytest.mark.parametrize("shape", [(3, 1, 4), (3, 2, 6), (4, 4, 8), (6, 5, 5), (8, 33, 70), (10, 64, 128)])
def test_medianmixringclean_matches_oracle(cuda, shape):
    rng = np.random.default_rng(3 + sum(shape))
    p = (rng.random(shape) * 0.2).astype(np.float32)
    p[:, :, 3] += 0.03
    for thr, wid in ((0.025, 0.0025), (0.01, 0.005)):
        mod = M.MedianMixRingClean()
        mod.Configure(M.ReconConfig(), {"threshold": str(thr), "width": str(wid)})
        t = torch.from_numpy(p).cuda()
        mod.Process(t)
        assert np.array_equal(_bits(t.cpu().numpy()), _bits(O.medianmixringclean(p, thr, wid))), (thr, wid)


def _mix_expected(p, picks, thr, wid):
    """MedianMixRingClean for the projections in picks, built from the oracle's pieces (the mean
    over all projections in float32 order, the profile median, the sigmoid table and the 5x5
    median of each picked projection)."""
    n, h, w = p.shape
    acc = np.zeros((h, w), np.float32)
    for i in range(n):
        acc += p[i]
    mean = acc * (np.float32(1.0) / np.float32(n))
    prof = O.median_filter(mean, 3, 3)
    v = np.abs(mean - prof)
    lut, par = O.sigmoid_lut(1024, thr, wid)
    f = v * par[2] + par[3]
    with np.errstate(invalid="ignore"):
        idx = np.where(f >= 0, np.minimum(np.trunc(np.nan_to_num(f, nan=0.0, posinf=1023.0)), 1023), 0).astype(int)
    wt = np.where(v < par[0], lut[0], np.where(par[1] < v, lut[-1], lut[idx])).astype(np.float32)
    return {i: (np.float32(1.0) - wt) * p[i] + wt * O.median_filter(p[i], 5, 5) for i in picks}


def test_medianmix_expected_helper_matches_oracle():
    rng = np.random.default_rng(2)
    p = (rng.random((6, 12, 16)) * 0.2).astype(np.float32)
    p[:, :, 5] += 0.03
    full = O.medianmixringclean(p)
    for i, v in _mix_expected(p, [0, 5], 0.025, 0.0025).items():
        assert np.array_equal(_bits(v), _bits(full[i]))


def test_medianmixringclean_two_batches(cuda):
    """70 projections of 1024 x 2048: the module filters 64 per batch, so the last 6 go through
    a second batch."""
    rng = np.random.default_rng(9)
    p = (rng.random((70, 1024, 2048)) * 0.2).astype(np.float32)
    p[:, :, 700] += 0.03
    t = torch.from_numpy(p).cuda()
    L.check(L.lib().mr_medianmixringclean(t.data_ptr(), 2048, 1024, 70, 0.025, 0.0025,
                                          torch.cuda.current_stream().cuda_stream))
    got = t.cpu().numpy()
    for i, v in _mix_expected(p, [0, 63, 64, 69], 0.025, 0.0025).items():
        assert np.array_equal(_bits(got[i]), _bits(v)), i


def test_gammaspotclean_passes_through(cuda):
    p = torch.rand(4, 16, 20, device="cuda")
    q = p.clone()
    mod = M.GammaSpotClean()
    mod.Configure(M.ReconConfig(), {"threshold3": "25", "threshold5": "100", "threshold7": "400", "sigma": "0.8",
                                    "mediansize": "3"})
    assert mod.Process(p) is p and torch.equal(p, q)


def test_ringalt_module_errors(cuda):
    with pytest.raises(M.ReconException):
        M.BasicRingClean().Process(torch.zeros(2, 8, 8, dtype=torch.float64, device="cuda"))
    with pytest.raises(M.ReconException):
        M.MedianMixRingClean().Process(torch.zeros(2, 8, 3, device="cuda"))
    with pytest.raises(M.ReconException):
        M.median_filter(torch.zeros(8, 8, device="cuda"), 7, 7)
