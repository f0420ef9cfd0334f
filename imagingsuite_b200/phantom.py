"""Seeded synthetic tomography data: ellipsoid phantoms, analytic projections, counts.

The workloads the hot path is measured on are defined by size and statistics, not by a
public dataset, so inputs are generated:

* 10 ellipsoids, centres uniform in the inner 80 % of the box, semi-axes U(0.05, 0.4) of the
  box, attenuation U(0.1, 1.0) per box length, random ZYZ Euler angles;
* line integrals are exact chord lengths through each ellipsoid (parallel beam: rays along
  the projection direction; cone beam: source to detector-pixel centre);
* counts = clip(Poisson(I0 * exp(-integral)) + N(100, 3^2), 0, 65535) as uint16;
  flats = Poisson(I0) + dark; darks = round(N(100, 3^2)).

Two back ends produce the same numbers up to floating-point rounding: numpy (FP64, for
small parity cases) and torch on a CUDA device (FP32, for full-size benchmark inputs).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Ellipsoid:
    center: np.ndarray  # (3,) in box units, box = [-0.5, 0.5]^3
    axes: np.ndarray    # (3,) semi-axes in box units
    rot: np.ndarray     # (3, 3) rotation, columns = ellipsoid axes in world frame
    mu: float           # attenuation per box length


def _euler_zyz(a: float, b: float, c: float) -> np.ndarray:
    def rz(t):
        return np.array([[math.cos(t), -math.sin(t), 0], [math.sin(t), math.cos(t), 0], [0, 0, 1]])

    def ry(t):
        return np.array([[math.cos(t), 0, math.sin(t)], [0, 1, 0], [-math.sin(t), 0, math.cos(t)]])

    return rz(a) @ ry(b) @ rz(c)


def ellipsoids(seed: int, n: int = 10) -> list[Ellipsoid]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        center = rng.uniform(-0.4, 0.4, 3)
        axes = rng.uniform(0.05, 0.4, 3)
        a, c = rng.uniform(0, 2 * math.pi, 2)
        b = math.acos(rng.uniform(-1, 1))
        out.append(Ellipsoid(center, axes, _euler_zyz(a, b, c), float(rng.uniform(0.1, 1.0))))
    return out


def _chords_np(p: np.ndarray, d: np.ndarray, ells: list[Ellipsoid]) -> np.ndarray:
    """Sum over ellipsoids of mu * chord length for rays p + t d (|d| = 1), FP64."""
    total = np.zeros(p.shape[:-1])
    for e in ells:
        q = ((p - e.center) @ e.rot) / e.axes
        w = (d @ e.rot) / e.axes
        a = np.sum(w * w, axis=-1)
        b = 2 * np.sum(q * w, axis=-1)
        c = np.sum(q * q, axis=-1) - 1
        disc = b * b - 4 * a * c
        ok = disc > 0
        chord = np.where(ok, np.sqrt(np.where(ok, disc, 0)) / a, 0.0)
        total += e.mu * chord
    return total


def parallel_integrals(ells, nproj: int, nu: int, nv: int, arc: float = 180.0, box: float | None = None) -> np.ndarray:
    """Parallel-beam line integrals (nproj, nv, nu), FP64, attenuation per box length (so the
    integrals are O(1)). The box spans `box` pixels (default nu) laterally and is centred on
    column (nu-1)/2 and row (nv-1)/2."""
    box = float(nu) if box is None else box
    ang = np.deg2rad(np.arange(nproj) * arc / nproj)
    u = (np.arange(nu) - (nu - 1) / 2) / box
    v = (np.arange(nv) - (nv - 1) / 2) / box
    out = np.empty((nproj, nv, nu))
    for k, t in enumerate(ang):
        d = np.array([math.cos(t), math.sin(t), 0.0])
        lat = np.array([-math.sin(t), math.cos(t), 0.0])
        p = u[None, :, None] * lat + v[:, None, None] * np.array([0, 0, 1.0]) - 2.0 * d
        out[k] = _chords_np(p, np.broadcast_to(d, p.shape), ells)
    return out


def cone_integrals(ells, nproj: int, nu: int, nv: int, sod: float, sdd: float, pitch: float, fov: float,
                   arc: float = 360.0) -> np.ndarray:
    """Cone-beam line integrals (nproj, nv, nu), FP64, flat detector, circular orbit. The
    phantom box has side `fov` (same length unit as sod/sdd/pitch); attenuation per box."""
    ang = np.deg2rad(np.arange(nproj) * arc / nproj)
    u = (np.arange(nu) - (nu - 1) / 2) * pitch
    v = (np.arange(nv) - (nv - 1) / 2) * pitch
    out = np.empty((nproj, nv, nu))
    for k, t in enumerate(ang):
        src = np.array([sod * math.cos(t), sod * math.sin(t), 0.0])
        axis = -src / sod
        lat = np.array([-math.sin(t), math.cos(t), 0.0])
        det = src + sdd * axis
        pix = det + u[None, :, None] * lat + v[:, None, None] * np.array([0, 0, 1.0])
        d = pix - src
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        p = np.broadcast_to(src / fov, d.shape)
        out[k] = _chords_np(p, d, ells)  # chord in box units times mu per box
    return out


def counts(integrals: np.ndarray, i0: float, seed: int, nflat: int, ndark: int):
    """uint16 projections, flats and darks from line integrals (numpy)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = integrals.shape[1:]
    darks = np.round(rng.normal(100.0, 3.0, (ndark,) + shape))
    flats = rng.poisson(i0, (nflat,) + shape) + np.round(rng.normal(100.0, 3.0, (nflat,) + shape))
    proj = rng.poisson(i0 * np.exp(-integrals)) + rng.normal(100.0, 3.0, integrals.shape)
    c = lambda a: np.clip(np.round(a), 0, 65535).astype(np.uint16)
    return c(proj), c(flats), c(darks)


# ----------------------------------------------------------------- torch (device) back end


def counts_torch(integrals, i0: float, seed: int, nflat: int, ndark: int):
    """Device version of :func:`counts` for benchmark-size inputs (torch tensors on CUDA)."""
    import torch

    g = torch.Generator(device=integrals.device)
    g.manual_seed(seed)
    shape = integrals.shape[1:]
    dev = integrals.device

    def normal(sz):
        return torch.randn(sz, generator=g, device=dev) * 3.0 + 100.0

    darks = torch.round(normal((ndark,) + tuple(shape)))
    flats = torch.poisson(torch.full((nflat,) + tuple(shape), float(i0), device=dev), generator=g) + torch.round(
        normal((nflat,) + tuple(shape)))
    proj = torch.poisson(i0 * torch.exp(-integrals), generator=g) + normal(tuple(integrals.shape))
    c = lambda a: torch.clamp(torch.round(a), 0, 65535).to(torch.int32).to(torch.uint16)
    return c(proj), c(flats), c(darks)


def cone_integrals_torch(ells, nproj: int, nu: int, nv: int, sod: float, sdd: float, pitch: float, fov: float,
                         device, arc: float = 360.0, chunk: int = 16):
    """Device (FP32) version of :func:`cone_integrals`."""
    import torch

    out = torch.empty((nproj, nv, nu), dtype=torch.float32, device=device)
    u = (torch.arange(nu, device=device, dtype=torch.float32) - (nu - 1) / 2) * pitch
    v = (torch.arange(nv, device=device, dtype=torch.float32) - (nv - 1) / 2) * pitch
    E = [(torch.tensor(e.center, dtype=torch.float32, device=device),
          torch.tensor(e.rot, dtype=torch.float32, device=device),
          torch.tensor(e.axes, dtype=torch.float32, device=device), e.mu) for e in ells]
    for k0 in range(0, nproj, chunk):
        ks = torch.arange(k0, min(nproj, k0 + chunk), device=device, dtype=torch.float32)
        t = torch.deg2rad(ks * arc / nproj)
        ct, st = torch.cos(t), torch.sin(t)
        zero = torch.zeros_like(ct)
        src = torch.stack([sod * ct, sod * st, zero], -1)  # (c,3)
        axis = -src / sod
        lat = torch.stack([-st, ct, zero], -1)
        det = src + sdd * axis
        pix = (det[:, None, None, :] + u[None, None, :, None] * lat[:, None, None, :]
               + v[None, :, None, None] * torch.tensor([0.0, 0.0, 1.0], device=device))
        d = pix - src[:, None, None, :]
        d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
        p = (src / fov)[:, None, None, :].expand_as(d)
        tot = torch.zeros(d.shape[:-1], device=device)
        for c, rot, axes, mu in E:
            q = ((p - c) @ rot) / axes
            w = (d @ rot) / axes
            a = (w * w).sum(-1)
            b = 2 * (q * w).sum(-1)
            cc = (q * q).sum(-1) - 1
            disc = b * b - 4 * a * cc
            tot += mu * torch.where(disc > 0, torch.sqrt(torch.clamp(disc, min=0)) / a, torch.zeros_like(a))
        out[k0:k0 + len(ks)] = tot
    return out


def voxelize_torch(ells, n: int, nz: int, device, supersample: int = 1, fov_margin: float | None = None):
    """Attenuation volume (nz, n, n), x fastest, of the ellipsoids on an n x n x nz voxel grid
    whose x/y extent is the unit box and whose voxels are cubes (z covers nz/n of the box,
    centred). Values are mu per voxel length (mu per box / n); supersample^3 points per voxel.
    With fov_margin, voxels farther than n/2 - fov_margin from the slice centre are zero (the
    object stays inside the circular field of view)."""
    import torch

    s = supersample
    off = (torch.arange(s, dtype=torch.float64, device=device) + 0.5) / s - 0.5
    xs = ((torch.arange(n, dtype=torch.float64, device=device)[:, None] + off[None, :]).reshape(-1) - (n - 1) / 2) / n
    zs = ((torch.arange(nz, dtype=torch.float64, device=device)[:, None] + off[None, :]).reshape(-1) - (nz - 1) / 2) / n
    out = torch.zeros((nz, n, n), dtype=torch.float32, device=device)
    for zi in range(nz):
        z = zs[zi * s:(zi + 1) * s]
        acc = torch.zeros((s, n * s, n * s), dtype=torch.float64, device=device)
        pz, py, px = torch.meshgrid(z, xs, xs, indexing="ij")
        p = torch.stack([px, py, pz], dim=-1)
        for e in ells:
            rot = torch.as_tensor(e.rot, dtype=torch.float64, device=device)
            q = ((p - torch.as_tensor(e.center, device=device)) @ rot) / torch.as_tensor(e.axes, device=device)
            acc += e.mu * ((q * q).sum(-1) <= 1.0)
        out[zi] = (acc.reshape(s, n, s, n, s).mean(dim=(0, 2, 4)) / n).float()
    if fov_margin is not None:
        c = torch.arange(n, device=device, dtype=torch.float64) - (n - 1) / 2
        out[:, (c[:, None] ** 2 + c[None, :] ** 2) > (n / 2 - fov_margin) ** 2] = 0
    return out


def parallel_integrals_torch(ells, nproj: int, nu: int, nv: int, device, arc: float = 180.0, box: float | None = None,
                             v0: int = 0, chunk: int = 8):
    """Device (FP32) version of :func:`parallel_integrals` for detector rows v0 .. v0+nv-1 of a
    detector whose full height is `box` pixels (default nu): the rows of one slice block."""
    import torch

    box = float(nu) if box is None else box
    out = torch.empty((nproj, nv, nu), dtype=torch.float32, device=device)
    u = (torch.arange(nu, device=device, dtype=torch.float32) - (nu - 1) / 2) / box
    v = (torch.arange(v0, v0 + nv, device=device, dtype=torch.float32) - (box - 1) / 2) / box
    E = [(torch.tensor(e.center, dtype=torch.float32, device=device),
          torch.tensor(e.rot, dtype=torch.float32, device=device),
          torch.tensor(e.axes, dtype=torch.float32, device=device), e.mu) for e in ells]
    for k0 in range(0, nproj, chunk):
        ks = torch.arange(k0, min(nproj, k0 + chunk), device=device, dtype=torch.float32)
        t = torch.deg2rad(ks * arc / nproj)
        ct, st = torch.cos(t), torch.sin(t)
        zero = torch.zeros_like(ct)
        d = torch.stack([ct, st, zero], -1)                      # (c,3)
        lat = torch.stack([-st, ct, zero], -1)
        p = (u[None, None, :, None] * lat[:, None, None, :] + v[None, :, None, None] *
             torch.tensor([0.0, 0.0, 1.0], device=device) - 2.0 * d[:, None, None, :])
        dd = d[:, None, None, :].expand_as(p)
        tot = torch.zeros(p.shape[:-1], device=device)
        for c, rot, axes, mu in E:
            q = ((p - c) @ rot) / axes
            w = (dd @ rot) / axes
            a = (w * w).sum(-1)
            b = 2 * (q * w).sum(-1)
            cc = (q * q).sum(-1) - 1
            disc = b * b - 4 * a * cc
            tot += mu * torch.where(disc > 0, torch.sqrt(torch.clamp(disc, min=0)) / a, torch.zeros_like(a))
        out[k0:k0 + len(ks)] = tot
    return out


def inject_defects_torch(counts, flats, seed: int, spot_fraction: float = 5e-4, ncols: int = 20,
                         gain=(1.005, 1.03)):
    """Production-case defects, in place on uint16 tensors: a fraction of pixels of every
    projection set to 65535 or tripled (half each), and ncols detector columns with a fixed
    gain error in the projections but not in the flats (ring-producing)."""
    import torch

    g = torch.Generator(device=counts.device)
    g.manual_seed(seed)
    nproj, nv, nu = counts.shape
    cols = torch.randperm(nu, generator=g, device=counts.device)[:ncols]
    gains = torch.rand(ncols, generator=g, device=counts.device) * (gain[1] - gain[0]) + gain[0]
    for k in range(nproj):
        c = counts[k].to(torch.float32)
        c[:, cols] *= gains
        sel = torch.rand((nv, nu), generator=g, device=counts.device) < spot_fraction
        hot = torch.rand((nv, nu), generator=g, device=counts.device) < 0.5
        c = torch.where(sel & hot, torch.full_like(c, 65535.0), torch.where(sel, c * 3.0, c))
        counts[k] = torch.clamp(torch.round(c), 0, 65535).to(torch.int32).to(torch.uint16)
    return cols, gains
