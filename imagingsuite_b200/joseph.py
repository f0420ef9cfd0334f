"""Differentiable parallel-beam projection: two projector pairs of mrcuda as a
torch.autograd.Function, gradients with respect to the volume, the centre of rotation and the
tilt, and CGLS with joint centre/tilt refinement.

* MatchedOperator: the backprojector itself (MultiProjectionBPparallel's interpolation, the
  production kernels) as A^T and its exact transpose as A (mr_mbp_*);
* JosephOperator: the Joseph projector of the reference's LinearForwardProjector as A and its
  exact transpose as A^T (mr_joseph_forward / mr_joseph_adjoint), the anchor to that module.

Geometry. Volume (nz, n, n), x fastest; projections (nproj, nz, nu); angles in degrees. The
detector centre of slice z is c_z = centre + tan(tilt) * (z - pivot) in detector bins
(MuhRec's tilt correction moves the centre of rotation linearly with the detector row);
centre = nu // 2, tilt = 0 is the geometry of the reference's LinearForwardProjector
(ReconAlgorithms/linearforwardprojector.cpp:15-144).

Loss of the refinement: 1/2 |A(x; centre, tilt) x - p|^2. Its gradient with respect to x is
A^T (A x - p); with respect to the centre, sum over rays of (dA x / d centre) (A x - p), and
with respect to the tilt (degrees) the same per slice weighted by (z - pivot) * d tan / d tilt.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib as L
from ._lib import check


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class JosephOperator:
    """A(centre, tilt) and A^T for a fixed volume size, detector width and angle set."""

    def __init__(self, n: int, nz: int, angles_deg, nu: int, pivot: float | None = None, device=None):
        self.n, self.nz, self.nu = int(n), int(nz), int(nu)
        a = np.ascontiguousarray(angles_deg, np.float32)
        self.nproj = a.size
        self.angles = a
        self.pivot = float((nz - 1) / 2.0 if pivot is None else pivot)
        params = np.zeros((self.nproj, 8), np.float32)
        check(L.lib().mr_joseph_geometry(a.ctypes.data_as(L.P_float), self.nproj, self.n,
                                         params.ctypes.data_as(L.P_float)))
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.params = torch.from_numpy(params).to(self.device)
        self._volt = torch.empty((self.nz, self.n, self.n), dtype=torch.float32, device=self.device)

    # ---- raw operators (float32 device tensors, contiguous)
    def forward(self, vol: torch.Tensor, centre: float, tilt_deg: float = 0.0, derivative: bool = False):
        self._check_vol(vol)
        proj = torch.empty((self.nproj, self.nz, self.nu), dtype=torch.float32, device=vol.device)
        dproj = torch.empty_like(proj) if derivative else None
        check(L.lib().mr_joseph_forward(vol.data_ptr(), self._volt.data_ptr(), self.n, self.nz, self.params.data_ptr(),
                                        self.nproj, self.nu, float(centre), math.tan(math.radians(tilt_deg)),
                                        self.pivot, proj.data_ptr(), 0 if dproj is None else dproj.data_ptr(),
                                        _stream()))
        return (proj, dproj) if derivative else proj

    def adjoint(self, proj: torch.Tensor, centre: float, tilt_deg: float = 0.0, out: torch.Tensor | None = None,
                accumulate: bool = False) -> torch.Tensor:
        self._check_proj(proj)
        if out is None:
            out = torch.empty((self.nz, self.n, self.n), dtype=torch.float32, device=proj.device)
        check(L.lib().mr_joseph_adjoint(proj.data_ptr(), self.n, self.nz, self.params.data_ptr(), self.nproj, self.nu,
                                        float(centre), math.tan(math.radians(tilt_deg)), self.pivot, int(accumulate),
                                        out.data_ptr(), _stream()))
        return out

    def slice_dot(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        """Per-slice sums of a * b over projections and bins (float64, shape (nz,))."""
        self._check_proj(a)
        self._check_proj(b)
        out = torch.empty(self.nz, dtype=torch.float64, device=a.device)
        check(L.lib().mr_slice_dot(a.data_ptr(), b.data_ptr(), self.nproj, self.nz, self.nu, out.data_ptr(),
                                   _stream()))
        return out

    def geometry_grad(self, dproj: torch.Tensor, g: torch.Tensor, tilt_deg: float):
        """(d/d centre, d/d tilt in degrees) of sum(proj * g), from d proj / d centre."""
        gz = self.slice_dot(dproj, g)
        zw = torch.arange(self.nz, dtype=torch.float64, device=gz.device) - self.pivot
        dtan = math.radians(1.0) / math.cos(math.radians(tilt_deg)) ** 2
        return gz.sum(), (zw * gz).sum() * dtan

    def _check_vol(self, v):
        if v.dtype != torch.float32 or not v.is_cuda or not v.is_contiguous() or tuple(v.shape) != (self.nz, self.n, self.n):
            raise ValueError(f"volume must be a contiguous float32 CUDA tensor of shape {(self.nz, self.n, self.n)}")

    def _check_proj(self, p):
        if p.dtype != torch.float32 or not p.is_cuda or not p.is_contiguous() or \
                tuple(p.shape) != (self.nproj, self.nz, self.nu):
            raise ValueError(f"projections must be a contiguous float32 CUDA tensor of shape "
                             f"{(self.nproj, self.nz, self.nu)}")


class MatchedOperator:
    """The pair matched to the parallel-beam backprojector (mr_mbp_*, include/mrcuda.h): A^T is
    MultiProjectionBPparallel's linear-interpolation backprojection (MultiProjBPparallel.cpp:
    39-170; every projection, weight 1) with the detector centre of slice z at
    c_z = centre + tan(tilt) (z - pivot), and A is its exact transpose. With no tilt, A^T runs the
    production backprojector itself (mr_bp_parallel_staged, TMA-staged); with tilt, the
    per-slice form (mr_mbp_adjoint), which equals it bit for bit at tilt 0.

    Layouts: volume (n, n, nz) = the backprojector's MatrixZXY [y][x][z]; projections
    (nproj, nz, n): the detector is n bins wide, as the reference backprojector takes it; nz a
    multiple of 4 (the backprojector updates slices in groups of 4). Angles in degrees, rotation
    direction as ReconConfig's eDirection (0 = clockwise). Same interface as JosephOperator, so
    project(), cgls(), fbp() and estimate_geometry() take either operator."""

    def __init__(self, n: int, nz: int, angles_deg, pivot: float | None = None, direction: int = 0, device=None):
        if nz % 4:
            raise ValueError("MatchedOperator: nz must be a multiple of 4")
        self.n, self.nz, self.nu = int(n), int(nz), int(n)
        self.angles = np.ascontiguousarray(angles_deg, np.float32)
        self.nproj = self.angles.size
        self.pivot = float((nz - 1) / 2.0 if pivot is None else pivot)
        self.direction = int(direction)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        mask = np.zeros(2 * self.n, np.uint32)
        check(L.lib().mr_bp_circle_mask(self.n, self.n, 0, 0.0, self.nz, mask.ctypes.data_as(L.P_u32)))
        self._mask = torch.from_numpy(mask.view(np.int32)).to(self.device)
        self._geo = {}

    def geometry(self, centre: float, tilt_deg: float):
        """(sincos (nproj, 2), startu (nproj, nz)) on the device for this centre and tilt."""
        key = (float(centre), float(tilt_deg))
        if key not in self._geo:
            sc = np.empty((self.nproj, 2), np.float32)
            su = np.empty((self.nproj, self.nz), np.float32)
            check(L.lib().mr_mbp_geometry(self.angles.ctypes.data_as(L.P_float), self.nproj, self.n, self.nz,
                                          float(centre), math.tan(math.radians(tilt_deg)), self.pivot,
                                          self.direction, sc.ctypes.data_as(L.P_float), su.ctypes.data_as(L.P_float)))
            if len(self._geo) >= 8:
                self._geo.pop(next(iter(self._geo)))
            self._geo[key] = tuple(torch.from_numpy(a).to(self.device) for a in (sc, su, np.ascontiguousarray(sc[:, 0]),
                                                                              np.ascontiguousarray(sc[:, 1]),
                                                                              np.ascontiguousarray(su[:, 0])))
        return self._geo[key]

    def forward(self, vol: torch.Tensor, centre: float, tilt_deg: float = 0.0, derivative: bool = False):
        self._check_vol(vol)
        sc, su, *_ = self.geometry(centre, tilt_deg)
        proj = torch.empty((self.nproj, self.nz, self.n), dtype=torch.float32, device=vol.device)
        dproj = torch.empty_like(proj) if derivative else None
        check(L.lib().mr_mbp_forward(vol.data_ptr(), self.n, self.nz, sc.data_ptr(), su.data_ptr(), self.nproj,
                                     self._mask.data_ptr(), proj.data_ptr(),
                                     None if dproj is None else dproj.data_ptr(), _stream()))
        return (proj, dproj) if derivative else proj

    def adjoint(self, proj: torch.Tensor, centre: float, tilt_deg: float = 0.0, out: torch.Tensor | None = None,
                accumulate: bool = False, staged: bool = True) -> torch.Tensor:
        self._check_proj(proj)
        sc, su, sn, cs, su0 = self.geometry(centre, tilt_deg)
        if out is None:
            out = torch.empty((self.n, self.n, self.nz), dtype=torch.float32, device=proj.device)
        if tilt_deg == 0.0 and staged:
            # the production backprojector: adds into the volume, so start from zero
            if not accumulate:
                out.zero_()
            check(L.lib().mr_bp_parallel_staged(proj.data_ptr(), self.nproj, L.MR_F32, None, None, None, sn.data_ptr(),
                                                cs.data_ptr(), su0.data_ptr(), self.nproj, self.n, self.nz,
                                                self._mask.data_ptr(), 0, 0.0, 0.0, out.data_ptr(), _stream()))
        else:
            check(L.lib().mr_mbp_adjoint(proj.data_ptr(), self.n, self.nz, sc.data_ptr(), su.data_ptr(), self.nproj,
                                         self._mask.data_ptr(), int(accumulate), out.data_ptr(), _stream()))
        return out

    slice_dot = JosephOperator.slice_dot
    geometry_grad = JosephOperator.geometry_grad

    def _check_vol(self, v):
        if v.dtype != torch.float32 or not v.is_cuda or not v.is_contiguous() or tuple(v.shape) != (self.n, self.n, self.nz):
            raise ValueError(f"volume must be a contiguous float32 CUDA tensor of shape {(self.n, self.n, self.nz)}")

    def _check_proj(self, p):
        if p.dtype != torch.float32 or not p.is_cuda or not p.is_contiguous() or \
                tuple(p.shape) != (self.nproj, self.nz, self.n):
            raise ValueError(f"projections must be a contiguous float32 CUDA tensor of shape "
                             f"{(self.nproj, self.nz, self.n)}")


class JosephProjection(torch.autograd.Function):
    """proj = A(centre, tilt) vol, differentiable in vol, centre and tilt (degrees)."""

    @staticmethod
    def forward(ctx, vol, centre, tilt_deg, op: JosephOperator):
        c, t = float(centre), float(tilt_deg)
        need_geo = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        res = op.forward(vol.detach().contiguous(), c, t, derivative=need_geo)
        proj, dproj = res if need_geo else (res, None)
        ctx.op, ctx.c, ctx.t = op, c, t
        ctx.save_for_backward(dproj if dproj is not None else torch.empty(0, device=vol.device))
        ctx.geo = [(v.dtype, v.device) if isinstance(v, torch.Tensor) else (torch.float64, torch.device("cpu"))
                   for v in (centre, tilt_deg)]
        return proj

    @staticmethod
    def backward(ctx, g):
        (dproj,) = ctx.saved_tensors
        g = g.contiguous()
        gv = ctx.op.adjoint(g, ctx.c, ctx.t) if ctx.needs_input_grad[0] else None
        gc = gt = None
        if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
            dc, dt = ctx.op.geometry_grad(dproj, g, ctx.t)
            gc = dc.to(dtype=ctx.geo[0][0], device=ctx.geo[0][1]) if ctx.needs_input_grad[1] else None
            gt = dt.to(dtype=ctx.geo[1][0], device=ctx.geo[1][1]) if ctx.needs_input_grad[2] else None
        return gv, gc, gt, None


def project(vol: torch.Tensor, centre, tilt_deg, op: JosephOperator) -> torch.Tensor:
    """Differentiable forward projection (see JosephProjection)."""
    return JosephProjection.apply(vol, centre, tilt_deg, op)


def _dot(a: torch.Tensor, b: torch.Tensor) -> float:
    return float(torch.dot(a.reshape(-1).double(), b.reshape(-1).double()).item())


def cgls(op: JosephOperator, p: torch.Tensor, x0: torch.Tensor, centre: float, tilt_deg: float = 0.0,
         iterations: int = 50, refine_every: int = 0, max_centre_step: float = 2.0):
    """CGLS on min 1/2 |A(centre, tilt) x - p|^2 from x0, `iterations` iterations in all.

    With refine_every > 0 the centre and the tilt are unknowns too (joint Gauss-Newton): every
    refine_every iterations the projection is linearised at the current (x, centre, tilt),
        A(c + dc, u + du) x ~ A x + dc D + du (z - pivot) D,   D = dA x / d centre, u = tan tilt,
    and CGLS runs on the augmented operator [A, D, (z - pivot) D] with unknowns (x, dc, du)
    (the two extra columns scaled to the operator's norm); the geometry increments are then
    applied (the centre step clipped to max_centre_step bins, the reach of the linearisation
    of an interpolation that is linear within one pixel) and the next block is linearised
    anew. Returns x, centre, tilt (degrees) and the history of 1/2 |residual|^2."""
    x = x0.clone()
    history = []
    zw = (torch.arange(op.nz, dtype=torch.float32, device=x.device) - op.pivot).view(1, op.nz, 1)
    it = 0
    while it < iterations:
        block = iterations - it if not refine_every else min(refine_every, iterations - it)
        if refine_every:
            ax, d = op.forward(x, centre, tilt_deg, derivative=True)
            sigma = math.sqrt(max(_dot(ax, ax), 1e-300) / max(_dot(x, x), 1e-300))
            dd = op.slice_dot(d, d)
            nc = math.sqrt(float(dd.sum()))
            nu_ = math.sqrt(float((zw.view(-1).double() ** 2 * dd).sum()))
            sc = nc / sigma if nc > 0 else 1.0
            su = nu_ / sigma if nu_ > 0 else 1.0
        else:
            ax, d, sc, su = op.forward(x, centre, tilt_deg), None, 1.0, 1.0
        r = p - ax
        a = [0.0, 0.0]  # scaled geometry increments

        def adj(res):
            sx = op.adjoint(res, centre, tilt_deg)
            if d is None:
                return sx, [0.0, 0.0]
            gz = op.slice_dot(d, res)
            return sx, [float(gz.sum()) / sc, float((zw.view(-1).double() * gz).sum()) / su]

        def fwd(vx, va):
            out = op.forward(vx, centre, tilt_deg)
            if d is not None:
                out.add_(d * (va[0] / sc + zw * (va[1] / su)))
            return out

        s_x, s_a = adj(r)
        q_x, q_a = s_x.clone(), list(s_a)
        gamma = _dot(s_x, s_x) + s_a[0] ** 2 + s_a[1] ** 2
        for _ in range(block):
            t = fwd(q_x, q_a)
            tt = _dot(t, t)
            if tt == 0.0 or gamma == 0.0:
                it = iterations
                break
            alpha = gamma / tt
            x.add_(q_x, alpha=alpha)
            a = [a[0] + alpha * q_a[0], a[1] + alpha * q_a[1]]
            r.sub_(t, alpha=alpha)
            s_x, s_a = adj(r)
            gnew = _dot(s_x, s_x) + s_a[0] ** 2 + s_a[1] ** 2
            q_x.mul_(gnew / gamma).add_(s_x)
            q_a = [s_a[0] + (gnew / gamma) * q_a[0], s_a[1] + (gnew / gamma) * q_a[1]]
            gamma = gnew
            history.append(0.5 * _dot(r, r))
            it += 1
        if d is not None:
            dc = max(-max_centre_step, min(max_centre_step, a[0] / sc))
            du = a[1] / su
            lim = max_centre_step / max(1.0, op.nz / 2.0)
            du = max(-lim, min(lim, du))
            centre += dc
            tilt_deg = math.degrees(math.atan(math.tan(math.radians(tilt_deg)) + du))
    return x, centre, tilt_deg, history


def fbp(op: JosephOperator, p: torch.Tensor, centre: float, tilt_deg: float = 0.0, filtertype: str = "hanning",
        cutoff: float = 0.5) -> torch.Tensor:
    """Filtered backprojection through the pair: detector rows ramp-filtered by the
    ProjectionFilterSingle kernels (mr_projfilter_*), backprojected with A^T, and scaled by
    the least-squares factor s minimising |A (s b) - p| (the starting volume of CGLS)."""
    plan = ctypes.c_void_p()
    check(L.lib().mr_projfilter_create(op.nu, filtertype.encode(), float(cutoff), 1.0, 1, 0.1, 2, ctypes.byref(plan)))
    try:
        f = torch.empty_like(p)
        check(L.lib().mr_projfilter_apply(plan, p.data_ptr(), f.data_ptr(), op.nproj * op.nz, None, 1, _stream()))
    finally:
        L.lib().mr_projfilter_destroy(plan)
    b = op.adjoint(f, centre, tilt_deg)
    ab = op.forward(b, centre, tilt_deg)
    s = _dot(ab, p) / max(_dot(ab, ab), 1e-300)
    return b.mul_(s)


def estimate_geometry(op: JosephOperator, p: torch.Tensor):
    """Centre of rotation and tilt from the sinogram centroids (Radon consistency of the
    first moment). For every slice z and angle t the centroid of the projection row,
    u(t) = sum_r r p / sum_r p, must follow c_z + a cos(theta_t) + b sin(theta_t) for an object
    inside the field of view; a least-squares fit of (c_z, a, b) per slice (weighted by the
    row masses) gives the slice's centre, and a line through the centres, weighted by the
    slices' masses, gives the centre at the pivot and the tilt. Returns (centre, tilt_deg);
    the per-slice centres of the last call are in estimate_geometry.last."""
    pd = p.double()
    r = torch.arange(op.nu, dtype=torch.float64, device=p.device)
    m0 = pd.sum(dim=2)                                   # (nproj, nz)
    m1 = (pd * r).sum(dim=2)
    th = torch.from_numpy(np.deg2rad(op.angles.astype(np.float64))).to(p.device)
    basis = torch.stack([torch.ones_like(th), torch.cos(th), torch.sin(th)], dim=1)  # (nproj, 3)
    cz, wz = [], []
    for z in range(op.nz):
        w = m0[:, z].clamp_min(0.0)
        if float(w.sum()) <= 0.0:
            cz.append(float("nan"))
            wz.append(0.0)
            continue
        u = m1[:, z] / torch.where(w > 0, w, torch.ones_like(w))
        sw = torch.sqrt(w)
        sol = torch.linalg.lstsq(basis * sw[:, None], (u * sw)[:, None]).solution[:, 0]
        cz.append(float(sol[0]))
        wz.append(float(w.sum()))
    cz, wz = np.asarray(cz), np.asarray(wz)
    keep = np.isfinite(cz) & (wz > 1e-3 * wz.max())
    estimate_geometry.last = {"slice_centres": np.where(np.isfinite(cz), cz, 0.0).tolist(), "slice_weights": wz.tolist()}
    z = np.arange(op.nz, dtype=np.float64)[keep] - op.pivot
    if keep.sum() > 1:
        slope, icpt = np.polyfit(z, cz[keep], 1, w=np.sqrt(wz[keep]))
    elif keep.sum() == 1:
        slope, icpt = 0.0, float(cz[keep][0])
    else:
        slope, icpt = 0.0, float(op.nu // 2)
    return float(icpt), math.degrees(math.atan(slope))
