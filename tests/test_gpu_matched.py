"""The differentiation form matched to the parallel-beam backprojector (gpu): A^T is
MultiProjectionBPparallel's backprojection (bit for bit against the oracle and the production
kernels), A its exact transpose (dot-product test), gradients in the volume, the centre and
the tilt against FP64 finite differences of the oracle's restatement, CGLS refinement."""
import math

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import joseph as J
from imagingsuite_b200 import phantom

pytestmark = pytest.mark.gpu


def _phantom(n, nz, seed=1011):
    """Ellipsoid phantom inside the field of view, in the backprojector's (y, x, z) layout."""
    v = phantom.voxelize_torch(phantom.ellipsoids(seed), n, nz, "cuda", supersample=2, fov_margin=6)
    return v.permute(1, 2, 0).contiguous()


@pytest.mark.parametrize("tilt", [0.0, 0.6])
@pytest.mark.parametrize("direction", [0, 1])
def test_adjoint_is_the_backprojector(cuda, tilt, direction):
    rng = np.random.default_rng(3)
    n, nz, nproj = 64, 12, 45
    ang = (np.arange(nproj) * 4.0 + 0.3).astype(np.float32)
    op = J.MatchedOperator(n, nz, ang, pivot=4.5, direction=direction)
    p = torch.from_numpy(rng.standard_normal((nproj, nz, n)).astype(np.float32)).cuda()
    got = op.adjoint(p, 31.2, tilt).cpu().numpy()
    exp = O.mbp_adjoint(p.cpu().numpy(), ang, 31.2, math.tan(math.radians(tilt)), 4.5, direction)
    assert np.array_equal(got, exp)
    if tilt == 0.0:
        # the production backprojector (staged) and the per-slice kernel agree bit for bit, and
        # both equal MultiProjectionBPparallel without the buffer-drop rule
        assert np.array_equal(op.adjoint(p, 31.2, 0.0, staged=False).cpu().numpy(), got)
        ref = O.bp_parallel(p.cpu().numpy(), ang, np.ones(nproj, np.float32), 31.2, direction=direction,
                            buffersize=1024)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("tilt", [0.0, 0.4])
def test_forward_matches_oracle_transpose(cuda, tilt):
    rng = np.random.default_rng(4)
    n, nz, nproj = 64, 8, 37
    ang = np.sort(rng.uniform(0, 180, nproj)).astype(np.float32)
    op = J.MatchedOperator(n, nz, ang, pivot=3.5)
    x = torch.from_numpy(rng.standard_normal((n, n, nz)).astype(np.float32)).cuda()
    got, d = op.forward(x, 32.4, tilt, derivative=True)
    exp, dexp = O.mbp_forward64(x.cpu().numpy(), ang, 32.4, math.tan(math.radians(tilt)), 3.5, derivative=True)
    rel = np.sqrt(np.sum((got.cpu().numpy() - exp) ** 2) / np.sum(exp ** 2))
    assert rel < 1e-6
    assert np.abs(d.cpu().numpy() - dexp).max() < 1e-3 * np.abs(dexp).max()


def test_forward_both_kernels_at_1024(cuda):
    """1024 bins: the value-only projection keeps its bins in shared memory (voxel-driven), the
    one with the derivative needs twice that and takes the ray-driven kernel; both against the
    oracle's transpose, and the two values against each other."""
    rng = np.random.default_rng(5)
    n, nz, nproj = 1024, 4, 5
    ang = np.array([0.0, 17.3, 45.0, 101.9, 150.2], np.float32)
    op = J.MatchedOperator(n, nz, ang, pivot=1.5)
    x = torch.from_numpy(rng.standard_normal((n, n, nz)).astype(np.float32)).cuda()
    v_only = op.forward(x, 511.3, 0.3).cpu().numpy()
    v, d = op.forward(x, 511.3, 0.3, derivative=True)
    exp, dexp = O.mbp_forward64(x.cpu().numpy(), ang, 511.3, math.tan(math.radians(0.3)), 1.5, derivative=True)
    for got in (v_only, v.cpu().numpy()):
        assert np.sqrt(np.sum((got - exp) ** 2) / np.sum(exp ** 2)) < 1e-6
    assert np.abs(d.cpu().numpy() - dexp).max() < 1e-3 * np.abs(dexp).max()


@pytest.mark.parametrize("n,nz,nproj,tilt", [(128, 32, 90, 0.0), (96, 16, 61, 0.7), (512, 8, 24, 0.4)])
def test_dot_product(cuda, n, nz, nproj, tilt):
    g = torch.Generator(device="cuda").manual_seed(n + nz)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    op = J.MatchedOperator(n, nz, ang)
    x = torch.randn((n, n, nz), device="cuda", generator=g)
    y = torch.randn((nproj, nz, n), device="cuda", generator=g)
    lhs = float(torch.dot(op.forward(x, n / 2 + 0.37, tilt).reshape(-1).double(), y.reshape(-1).double()))
    rhs = float(torch.dot(x.reshape(-1).double(), op.adjoint(y, n / 2 + 0.37, tilt).reshape(-1).double()))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def _loss64(x, ang, centre, tilt, pivot, p):
    r = O.mbp_forward64(x, ang, centre, math.tan(math.radians(tilt)), pivot, float_u=False) - p
    return 0.5 * float((r * r).sum())


def test_gradients_against_fp64_finite_differences(cuda):
    rng = np.random.default_rng(13)
    n, nz, nproj = 64, 8, 60
    ang = np.sort(rng.uniform(0, 180, nproj)).astype(np.float32)
    pivot = 3.5
    ph = _phantom(n, nz).cpu().numpy()
    p = O.mbp_forward64(ph, ang, 32.0 + 1.3, math.tan(math.radians(1.0)), pivot, float_u=False)
    x = (ph * (1 + 0.01 * rng.standard_normal(ph.shape))).astype(np.float32)
    c, t = 32.0, 0.3
    op = J.MatchedOperator(n, nz, ang, pivot=pivot)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    ct = torch.tensor(c, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(t, dtype=torch.float64, requires_grad=True)
    pt = torch.from_numpy(p.astype(np.float32)).cuda()
    loss = 0.5 * ((J.project(xt, ct, tt, op) - pt) ** 2).sum()
    loss.backward()
    h = 1e-5
    fd_c = (_loss64(x, ang, c + h, t, pivot, p) - _loss64(x, ang, c - h, t, pivot, p)) / (2 * h)
    fd_t = (_loss64(x, ang, c, t + h, pivot, p) - _loss64(x, ang, c, t - h, pivot, p)) / (2 * h)
    assert abs(float(ct.grad) - fd_c) <= 1e-3 * abs(fd_c)
    assert abs(float(tt.grad) - fd_t) <= 1e-3 * abs(fd_t)
    v = (rng.standard_normal(x.shape) * (ph > 0)).astype(np.float32) * 0.01
    eps = 1e-3
    fd_v = (_loss64(x + eps * v, ang, c, t, pivot, p) - _loss64(x - eps * v, ang, c, t, pivot, p)) / (2 * eps)
    an_v = float((xt.grad.double().cpu().numpy() * v).sum())
    assert abs(an_v - fd_v) <= 1e-3 * abs(fd_v)


def test_cgls_recovers_centre_and_tilt(cuda):
    n, nz, nproj = 128, 64, 180
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    op = J.MatchedOperator(n, nz, ang)
    truth = _phantom(n, nz, 1009)
    c_true, t_true = n / 2 + 3.7, 2.5
    p = op.forward(truth, c_true, t_true)
    c0, t0 = J.estimate_geometry(op, p)
    assert abs(c0 - c_true) < 0.5 and abs(t0 - t_true) < 0.5
    x0 = J.fbp(op, p, c0, t0)
    x, c, t, hist = J.cgls(op, p, x0, c0, t0, iterations=50, refine_every=5)
    assert abs(c - c_true) < 0.1
    assert abs(t - t_true) < 0.1
    assert hist[-1] < 0.05 * hist[0]
    e0 = float(torch.linalg.vector_norm(x0 - truth)) / float(torch.linalg.vector_norm(truth))
    e1 = float(torch.linalg.vector_norm(x - truth)) / float(torch.linalg.vector_norm(truth))
    assert e1 < e0
