"""The FP64 restatement of the Joseph projector pair (oracle) against the reference's
LinearForwardProjector and against itself: adjointness and the centre derivative."""
import os

import numpy as np

import oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))


def _relrms(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64) - b) ** 2) / np.mean(np.asarray(b, np.float64) ** 2)))


def test_forward_matches_reference_golden():
    """centre = n/2, no tilt is the reference geometry; the reference accumulates the sample
    position (nfloat += alpha) in float, which bounds the agreement."""
    sl, ang = G["joseph_slices"], G["joseph_angles"]
    for s_, ref in zip(sl, G["joseph_ref"]):
        ours = O.joseph_forward64(s_[None], ang, 64, 32)[:, 0, :]
        assert _relrms(ours, ref) < 1e-4


def test_forward_matches_compiled_reference(ref_lib):
    rng = np.random.default_rng(81)
    for n in (48, 65):
        sl = rng.standard_normal((n, n)).astype(np.float32)
        ang = np.sort(rng.uniform(0, 360, 31)).astype(np.float32)
        ref = O.ref_joseph_project(sl, ang)
        assert _relrms(O.joseph_forward64(sl[None], ang, n, n // 2)[:, 0, :], ref) < 1e-4


def _support_volume(rng, nz, n):
    """Random volume inside the inscribed circle (no samples at the image border)."""
    v = rng.standard_normal((nz, n, n)).astype(np.float32)
    yy, xx = np.mgrid[:n, :n]
    v[:, (xx - (n - 1) / 2) ** 2 + (yy - (n - 1) / 2) ** 2 > (n / 2 - 3) ** 2] = 0
    return v


def test_adjoint_is_exact_transpose():
    rng = np.random.default_rng(82)
    n, nz, nu = 40, 3, 46
    ang = np.sort(rng.uniform(0, 180, 29)).astype(np.float32)
    x = rng.standard_normal((nz, n, n)).astype(np.float32)
    y = rng.standard_normal((ang.size, nz, nu))
    ax = O.joseph_forward64(x, ang, nu, 23.4, 0.02, 1.0)
    aty = O.joseph_adjoint64(y, ang, n, 23.4, 0.02, 1.0)
    lhs, rhs = float((ax * y).sum()), float((x.astype(np.float64) * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_centre_derivative_matches_finite_differences():
    rng = np.random.default_rng(83)
    n, nz, nu = 40, 3, 46
    ang = np.sort(rng.uniform(0, 180, 29)).astype(np.float32)
    x = _support_volume(rng, nz, n)
    _, d = O.joseph_forward64(x, ang, nu, 23.4, 0.02, 1.0, derivative=True)
    h = 1e-6
    fd = (O.joseph_forward64(x, ang, nu, 23.4 + h, 0.02, 1.0) - O.joseph_forward64(x, ang, nu, 23.4 - h, 0.02, 1.0)) / (2 * h)
    assert _relrms(d, fd) < 1e-3
