"""Alternative ring cleaners on the CPU: the C restatement against the reference's own
BasicRingClean, MedianMixRingClean, GammaSpotCleanModule, kipl TMedianFilter and SigmoidLUT
(compiled from source), the selection networks of the CUDA median proven on every 0-1 input,
the library's host-side sigmoid table, and the entry points' argument checks."""
import importlib.util
import os

import numpy as np
import pytest

import oracle as O
from imagingsuite_b200 import _lib as L

_HERE = os.path.dirname(os.path.abspath(__file__))


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


KERNELS = [(1, 1), (3, 1), (1, 3), (3, 3), (5, 1), (1, 5), (5, 3), (3, 5), (5, 5)]


@pytest.mark.parametrize("kx,ky", KERNELS)
def test_median_filter_matches_reference(ref_lib, kx, ky):
    """All sizes down to the smallest the reference handles (2*(k/2) per axis), so every edge
    code, the window reaching past the row at the right edge and past the image end at the
    bottom-right corner (read as 0 on both sides) are covered."""
    rng = np.random.default_rng(kx * 10 + ky)
    for h in (max(1, 2 * (ky // 2)), 3, 5, 6, 9, 17):
        for w in (max(1, 2 * (kx // 2)), 4, 5, 7, 16, 23):
            if h < 2 * (ky // 2) or w < 2 * (kx // 2):
                continue
            img = rng.standard_normal((h, w)).astype(np.float32)
            assert np.array_equal(_bits(O.median_filter(img, kx, ky)),
                                  _bits(O.median_filter(img, kx, ky, use_ref=True))), (h, w)


@pytest.mark.parametrize("kx,ky", [(3, 3), (5, 5), (5, 1)])
def test_median_filter_special_values(ref_lib, kx, ky):
    """Ties, zeros of both signs, NaN and infinities: the heap sort's placement decides which
    bits end in the middle, and the restatement follows it."""
    rng = np.random.default_rng(7 + kx + ky)
    for t in range(40):
        img = rng.integers(-2, 3, (9, 11)).astype(np.float32)
        z = rng.random(img.shape) < 0.35
        img[z] = np.where(rng.random(z.sum()) < 0.5, np.float32(0.0), np.float32(-0.0))
        if t % 2:
            img[rng.integers(0, 9), rng.integers(0, 11)] = np.nan
        if t % 3 == 0:
            img[rng.integers(0, 9), rng.integers(0, 11)] = np.inf if t % 2 else -np.inf
        assert np.array_equal(_bits(O.median_filter(img, kx, ky)), _bits(O.median_filter(img, kx, ky, use_ref=True)))


def test_median_filter_reads_zero_past_the_image(ref_lib):
    """The reference's bottom-right 3x3 window is {img[2,2], img[2,3], img[3,0] (the row wrap),
    img[3,2] x2, img[3,3] x2, and the value past the image end x2}. With the first three at -3
    and the rest at 5, the corner's median is that past-the-end value: 0 in both oracles
    (edge replication would give 5)."""
    img = np.full((4, 4), 5.0, np.float32)
    img[2, 2] = img[2, 3] = img[3, 0] = -3.0
    out = O.median_filter(img, 3, 3)
    assert np.array_equal(_bits(out), _bits(O.median_filter(img, 3, 3, use_ref=True)))
    assert out[3, 3] == 0.0


@pytest.mark.parametrize("shape", [(1, 2, 2), (3, 5, 6), (7, 16, 20), (20, 33, 40)])
def test_basicringclean_matches_reference(ref_lib, shape):
    rng = np.random.default_rng(sum(shape))
    p = (rng.random(shape) * 2).astype(np.float32)
    p[:, :, shape[2] // 2] += 0.05  # a ring
    p[0, 0, 0] = -0.0
    assert np.array_equal(_bits(O.basicringclean(p)), _bits(O.basicringclean(p, use_ref=True)))


@pytest.mark.parametrize("lam,sigma", [(0.025, 0.0025), (0.1, 0.0075), (0.5, 0.05), (1.0, 0.001), (0.0, 0.1),
                                       (-0.2, 0.03)])
def test_sigmoid_lut_matches_reference(ref_lib, lam, sigma):
    a, pa = O.sigmoid_lut(1024, lam, sigma)
    b, pb = O.sigmoid_lut(1024, lam, sigma, use_ref=True)
    assert np.array_equal(_bits(a), _bits(b)) and np.array_equal(_bits(pa), _bits(pb))


@pytest.mark.parametrize("lam,sigma", [(0.025, 0.0025), (0.1, 0.0075), (1.0, 0.001), (-0.2, 0.03)])
def test_library_sigmoid_lut_matches_reference(ref_lib, lam, sigma):
    """The host table the CUDA MedianMixRingClean uses (mr_sigmoid_lut, no GPU needed)."""
    lut = np.empty(1024, np.float32)
    par = np.empty(4, np.float32)
    L.check(L.lib().mr_sigmoid_lut(1024, lam, sigma, lut.ctypes.data_as(L.P_float), par.ctypes.data_as(L.P_float)))
    b, pb = O.sigmoid_lut(1024, lam, sigma, use_ref=True)
    assert np.array_equal(_bits(lut), _bits(b)) and np.array_equal(_bits(par), _bits(pb))


@pytest.mark.parametrize("shape", [(1, 1, 4), (3, 2, 6), (4, 4, 8), (5, 5, 5), (7, 16, 20), (20, 33, 40)])
def test_medianmixringclean_matches_reference(ref_lib, shape):
    """Profile filter 5x1 below 3 rows, mixing filter 5x1 below 5 rows, 5x5 from 5 rows."""
    rng = np.random.default_rng(3 + sum(shape))
    p = (rng.random(shape) * 0.2).astype(np.float32)
    p[:, :, 3] += 0.03  # a ring the sigmoid weights pick up
    for thr, wid in ((0.025, 0.0025), (0.01, 0.005)):
        assert np.array_equal(_bits(O.medianmixringclean(p, thr, wid)),
                              _bits(O.medianmixringclean(p, thr, wid, use_ref=True)))


def test_gammaspotclean_reference_is_identity(ref_lib):
    """The reference GammaSpotCleanModule returns the projections unchanged (its cleaning
    calls are commented out), which is what the module here does."""
    p = np.random.default_rng(5).random((3, 8, 9)).astype(np.float32)
    assert np.array_equal(_bits(O.ref_gammaspotclean(p)), _bits(p))


def _selector():
    path = os.path.join(_HERE, "..", "imagingsuite_b200", "csrc", "gen_median_net.py")
    spec = importlib.util.spec_from_file_location("gen_median_net", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.selector


@pytest.mark.parametrize("n,outs", [(3, None), (5, None), (9, None), (11, None), (15, None), (25, None),
                                    (20, range(7, 13))])
def test_median_networks_on_all_binary_inputs(n, outs):
    """0-1 principle: a min/max network returns the k-th order statistic of every input on wire
    k iff it does so for every 0-1 input, all 2^n of which are run here (the middle output, or
    ranks 7..12 of 20 for the selector of window pairs)."""
    ops, out = _selector()(n, outs)
    wires = [out] if outs is None else list(outs)
    total, chunk = 1 << n, 1 << 20
    for s in range(0, total, chunk):
        idx = np.arange(s, min(total, s + chunk), dtype=np.uint32)
        v = [((idx >> i) & 1).astype(np.uint8) for i in range(n)]
        ones = np.sum(v, axis=0, dtype=np.int32)
        for op, a, b, _, _ in ops:
            if op == "mov":
                v[a] = v[b]
            else:
                v[a], v[b] = np.minimum(v[a], v[b]), np.maximum(v[a], v[b])
        for k in wires:  # the k-th smallest is 1 iff at most k zeros
            assert np.array_equal(v[k], (ones >= n - k).astype(np.uint8))


def test_median_network_header_is_current():
    """The committed mr_median_net.cuh is what the generator writes."""
    import io
    import contextlib

    path = os.path.join(_HERE, "..", "imagingsuite_b200", "csrc")
    spec = importlib.util.spec_from_file_location("gen_median_net", os.path.join(path, "gen_median_net.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        mod.main()
    with open(os.path.join(path, "mr_median_net.cuh")) as f:
        assert f.read() == buf.getvalue()


def test_ringalt_argument_errors_need_no_gpu():
    lib = L.lib()
    fake = 256
    assert lib.mr_median_filter(None, 8, 8, 1, 3, 3, fake, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_median_filter(fake, 8, 8, 1, 4, 3, fake + 4096, None) == L.MR_ERR_UNSUPPORTED
    assert lib.mr_median_filter(fake, 8, 8, 1, 7, 7, fake + 4096, None) == L.MR_ERR_UNSUPPORTED
    assert lib.mr_median_filter(fake, 3, 8, 1, 5, 5, fake + 4096, None) == L.MR_ERR_ARGUMENT  # reference throws
    assert lib.mr_median_filter(fake, 8, 8, 1, 3, 3, fake, None) == L.MR_ERR_ARGUMENT  # in place
    assert lib.mr_basicringclean(fake, 1, 8, 4, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_medianmixringclean(fake, 3, 8, 4, 0.025, 0.0025, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_medianmixringclean(fake, 8, 8, 4, 0.025, 0.0, None) == L.MR_ERR_ARGUMENT
    assert b"width" in lib.mr_last_error()
    lut = np.empty(4, np.float32)
    assert lib.mr_sigmoid_lut(4, 0.1, -1.0, lut.ctypes.data_as(L.P_float), lut.ctypes.data_as(L.P_float)) == \
        L.MR_ERR_ARGUMENT


def spot_phantom(rng, n, h, w, density=0.004):
    """Smooth projections with spots: single pixels, small blobs, a few outside the level range."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.3 + 0.2 * np.sin(xx / 7.0) * np.cos(yy / 11.0)
    p = np.empty((n, h, w), np.float32)
    for i in range(n):
        q = base + rng.normal(0, 0.004, (h, w))
        k = max(1, int(h * w * density))
        idx = rng.integers(0, h * w, k)
        q.reshape(-1)[idx] += rng.choice([0.3, 1.0, 6.0, -0.9], k)
        y0, x0 = rng.integers(2, h - 6), rng.integers(2, w - 6)
        q[y0:y0 + 3, x0:x0 + 4] += 1.5  # a blob of 12 pixels
        p[i] = q
    return p


@pytest.mark.parametrize("method", ["ring", "median", "minmax", "stddev", "trikernel"])
def test_spotclean2_matches_reference(ref_lib, method):
    """The restatement of ImagingAlgorithms::SpotClean against the compiled SpotClean2 module:
    every detection method, region exclusion on and off, two iterations, ragged sizes."""
    rng = np.random.default_rng(len(method))
    for n, h, w in ((2, 16, 16), (2, 23, 37), (1, 48, 64)):
        p = spot_phantom(rng, n, h, w)
        for gamma, sigma, maxarea, it in ((0.1, 0.001, 20, 1), (0.05, 0.01, 0, 2), (0.2, 0.005, 5, 1)):
            a = O.spotclean2(p, method, gamma, sigma, it, -0.1, 5.0, maxarea)
            b = O.spotclean2(p, method, gamma, sigma, it, -0.1, 5.0, maxarea, use_ref=True)
            assert np.array_equal(_bits(a), _bits(b)), (method, n, h, w, gamma, sigma, maxarea, it)


def test_spotclean2_background_neighbour_rule(ref_lib):
    """RemoveConnectedRegion also floods from the background label's last pixel: a small spot
    next to the last background pixel loses its weight although it is below maxarea, so it is
    not cleaned (it stays in the level range)."""
    p = np.full((1, 16, 16), 0.3, np.float32)
    p[0, 15, 15] = 2.0  # the last pixel is a spot; the last background pixel is (15, 14)
    p[0, 4, 4] = 2.0  # an isolated spot elsewhere
    a = O.spotclean2(p, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20)
    assert np.array_equal(_bits(a), _bits(O.spotclean2(p, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20, use_ref=True)))
    assert a[0, 15, 15] == np.float32(2.0) and a[0, 4, 4] < 1.0


def test_spotclean2_every_pixel_a_spot(ref_lib):
    """All pixels above maxlevel: the reference still ends, because the last pixel's right
    neighbour is the value past the image end (0 in both oracles)."""
    p = np.full((2, 20, 24), 9.0, np.float32)
    p[1, 3, 5] = 0.5
    a = O.spotclean2(p, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20)
    assert np.array_equal(_bits(a), _bits(O.spotclean2(p, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20, use_ref=True)))
    assert not np.any(a == np.float32(9.0))


def test_spotclean2_argument_errors_need_no_gpu():
    lib = L.lib()
    fake = 256
    assert lib.mr_spotclean2(None, 32, 32, 1, 1, 0.1, 0.001, 1, -0.1, 5.0, 20, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_spotclean2(fake, 15, 32, 1, 1, 0.1, 0.001, 1, -0.1, 5.0, 20, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_spotclean2(fake, 32, 32, 1, 7, 0.1, 0.001, 1, -0.1, 5.0, 20, None) == L.MR_ERR_ARGUMENT
    assert lib.mr_spotclean2(fake, 32, 32, 1, 1, 0.1, 0.0, 1, -0.1, 5.0, 20, None) == L.MR_ERR_ARGUMENT
