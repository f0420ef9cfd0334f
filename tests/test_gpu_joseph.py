"""Differentiation form on the GPU (gpu): the Joseph pair against the FP64 oracle and the
reference's golden output, the adjoint dot-product test, gradients of
1/2 |A(x; centre, tilt) x - p|^2 against FP64 finite differences, the autograd wrapper, and
CGLS with joint centre/tilt refinement."""
import math
import os

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import joseph as J
from imagingsuite_b200 import phantom

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))


def _relrms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def _support(rng, nz, n):
    v = rng.standard_normal((nz, n, n)).astype(np.float32)
    yy, xx = np.mgrid[:n, :n]
    v[:, (xx - (n - 1) / 2) ** 2 + (yy - (n - 1) / 2) ** 2 > (n / 2 - 3) ** 2] = 0
    return v


def test_forward_matches_reference_golden(cuda):
    ang = G["joseph_angles"]
    op = J.JosephOperator(64, 2, ang, 64, pivot=0.0)
    vol = torch.from_numpy(np.ascontiguousarray(G["joseph_slices"])).cuda()
    proj = op.forward(vol, 32.0).cpu().numpy()
    for z in range(2):
        assert _relrms(proj[:, z, :], G["joseph_ref"][z]) < 1e-4


@pytest.mark.parametrize("n,nu,centre,tilt", [(64, 70, 35.3, 0.0), (63, 64, 31.27, 1.5), (96, 110, 56.8, -0.7)])
def test_forward_and_derivative_match_oracle(cuda, n, nu, centre, tilt):
    """Values on random volumes; the centre derivative on a phantom (the derivative of a
    piecewise-linear interpolation jumps where a sample crosses a pixel boundary, and FP32 and
    FP64 positions may fall on either side of one)."""
    rng = np.random.default_rng(n)
    nz = 5
    ang = np.sort(rng.uniform(0, 360, 41)).astype(np.float32)
    x = _support(rng, nz, n)
    op = J.JosephOperator(n, nz, ang, nu, pivot=2.0)
    p = op.forward(torch.from_numpy(x).cuda(), centre, tilt)
    ep = O.joseph_forward64(x, ang, nu, centre, math.tan(math.radians(tilt)), 2.0)
    assert _relrms(p.cpu().numpy(), ep) < 2e-5
    ph = phantom.voxelize_torch(phantom.ellipsoids(1000 + n), n, nz, "cuda", supersample=2)
    _, d = op.forward(ph, centre, tilt, derivative=True)
    _, ed = O.joseph_forward64(ph.cpu().numpy(), ang, nu, centre, math.tan(math.radians(tilt)), 2.0, derivative=True)
    assert _relrms(d.cpu().numpy(), ed) < 5e-3


def test_adjoint_matches_oracle(cuda):
    rng = np.random.default_rng(7)
    n, nz, nu = 72, 4, 80
    ang = np.sort(rng.uniform(0, 180, 37)).astype(np.float32)
    y = rng.standard_normal((ang.size, nz, nu)).astype(np.float32)
    op = J.JosephOperator(n, nz, ang, nu, pivot=1.5)
    got = op.adjoint(torch.from_numpy(y).cuda(), 40.2, 0.8).cpu().numpy()
    exp = O.joseph_adjoint64(y, ang, n, 40.2, math.tan(math.radians(0.8)), 1.5)
    assert _relrms(got, exp) < 2e-5


@pytest.mark.parametrize("n,nz,nproj,nu", [(96, 4, 180, 100), (512, 8, 360, 512)])
def test_dot_product(cuda, n, nz, nproj, nu):
    """<A x, y> = <x, A^T y> to FP32 summation rounding (the weights are bit-identical)."""
    g = torch.Generator(device="cuda").manual_seed(n)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    op = J.JosephOperator(n, nz, ang, nu)
    x = torch.randn((nz, n, n), device="cuda", generator=g)
    y = torch.randn((nproj, nz, nu), device="cuda", generator=g)
    ax = op.forward(x, nu / 2 + 3.7, 0.4)
    aty = op.adjoint(y, nu / 2 + 3.7, 0.4)
    lhs = float(torch.dot(ax.reshape(-1).double(), y.reshape(-1).double()))
    rhs = float(torch.dot(x.reshape(-1).double(), aty.reshape(-1).double()))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def _loss64(x, ang, nu, centre, tilt, pivot, p):
    r = O.joseph_forward64(x, ang, nu, centre, math.tan(math.radians(tilt)), pivot) - p
    return 0.5 * float((r * r).sum())


def test_gradients_against_fp64_finite_differences(cuda):
    rng = np.random.default_rng(11)
    n, nz, nu = 64, 6, 72
    ang = np.sort(rng.uniform(0, 180, 60)).astype(np.float32)
    pivot = 2.5
    ph = phantom.voxelize_torch(phantom.ellipsoids(1007), n, nz, "cuda", supersample=2).cpu().numpy()
    p = O.joseph_forward64(ph, ang, nu, 36.0 + 1.3, math.tan(math.radians(1.0)), pivot)
    x = (ph + 0.002 * _support(rng, nz, n)).astype(np.float32)
    c, t = 36.0, 0.3
    op = J.JosephOperator(n, nz, ang, nu, pivot=pivot)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    ct = torch.tensor(c, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(t, dtype=torch.float64, requires_grad=True)
    pt = torch.from_numpy(p.astype(np.float32)).cuda()
    loss = 0.5 * ((J.project(xt, ct, tt, op) - pt) ** 2).sum()
    loss.backward()
    h = 1e-5
    fd_c = (_loss64(x, ang, nu, c + h, t, pivot, p) - _loss64(x, ang, nu, c - h, t, pivot, p)) / (2 * h)
    fd_t = (_loss64(x, ang, nu, c, t + h, pivot, p) - _loss64(x, ang, nu, c, t - h, pivot, p)) / (2 * h)
    assert abs(float(ct.grad) - fd_c) <= 1e-3 * abs(fd_c)
    assert abs(float(tt.grad) - fd_t) <= 1e-3 * abs(fd_t)
    v = _support(rng, nz, n) * 0.01
    eps = 1e-3
    fd_v = (_loss64(x + eps * v, ang, nu, c, t, pivot, p) - _loss64(x - eps * v, ang, nu, c, t, pivot, p)) / (2 * eps)
    an_v = float((xt.grad.double().cpu().numpy() * v).sum())
    assert abs(an_v - fd_v) <= 1e-3 * abs(fd_v)


def test_autograd_matches_operators(cuda):
    rng = np.random.default_rng(12)
    n, nz, nu = 48, 3, 52
    ang = np.sort(rng.uniform(0, 180, 30)).astype(np.float32)
    op = J.JosephOperator(n, nz, ang, nu)
    x = torch.from_numpy(_support(rng, nz, n)).cuda()
    g = torch.from_numpy(rng.standard_normal((30, nz, nu)).astype(np.float32)).cuda()
    xt = x.clone().requires_grad_(True)
    ct = torch.tensor(27.1, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(0.5, dtype=torch.float64, requires_grad=True)
    (J.project(xt, ct, tt, op) * g).sum().backward()
    assert torch.equal(xt.grad, op.adjoint(g, 27.1, 0.5))
    _, d = op.forward(x, 27.1, 0.5, derivative=True)
    dc, dt = op.geometry_grad(d, g, 0.5)
    assert float(ct.grad) == pytest.approx(float(dc), rel=1e-12)
    assert float(tt.grad) == pytest.approx(float(dt), rel=1e-12)


def test_cgls_recovers_centre_and_tilt(cuda):
    n, nz, nu, nproj = 128, 64, 136, 180
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    op = J.JosephOperator(n, nz, ang, nu)
    truth = phantom.voxelize_torch(phantom.ellipsoids(1009), n, nz, "cuda", supersample=2, fov_margin=6)
    c_true, t_true = nu / 2 + 3.7, 2.5
    p = op.forward(truth, c_true, t_true)
    c0, t0 = J.estimate_geometry(op, p)
    print(f"coarse estimate centre {c0:.3f} tilt {t0:.3f}")
    assert abs(c0 - c_true) < 0.5 and abs(t0 - t_true) < 0.5
    x0 = J.fbp(op, p, c0, t0)
    x, c, t, hist = J.cgls(op, p, x0, c0, t0, iterations=50, refine_every=5)
    print(f"centre {c:.4f} (true {c_true}), tilt {t:.4f} (true {t_true}), loss {hist[0]:.4g} -> {hist[-1]:.4g}")
    assert abs(c - c_true) < 0.1
    assert abs(t - t_true) < 0.1
    assert hist[-1] < 0.05 * hist[0]
    # the volume moved towards the truth
    e0 = float(torch.linalg.vector_norm(x0 - truth)) / float(torch.linalg.vector_norm(truth))
    e1 = float(torch.linalg.vector_norm(x - truth)) / float(torch.linalg.vector_norm(truth))
    assert e1 < e0
