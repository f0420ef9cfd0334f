"""FDK precision form on the GPU (gpu): the FP64 error oracle kernel against the CPU FP64
restatement (bit for bit), and the 16-bit backprojection through FP64-derived maps against
the FP64 oracle, with the FP32 reference-exact path measured beside it."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M
from imagingsuite_b200 import phantom

pytestmark = pytest.mark.gpu


def _geom(nu, nv, pp, center, pitch, voxel, tilt=0.0, pivot=0.0):
    og = O.fdk_geom(300.0, 600.0, pp, center, (pitch, pitch), (voxel,) * 3, correcttilt=bool(tilt), tiltangle=tilt,
                    tiltpivot=pivot)
    g = L.FdkGeom()
    ctypes.memmove(ctypes.byref(g), ctypes.byref(og), ctypes.sizeof(g))
    return og, g


def _maps(g, nu, nv, ang):
    m = np.zeros((ang.size, 12), np.float64)
    L.check(L.lib().mr_fdk_maps64(ctypes.byref(g), nu, nv, ang.ctypes.data_as(L.P_float), ang.size,
                                  m.ctypes.data_as(L.P_double)))
    return m


def _mask(nu):
    m = np.zeros(2 * nu, np.uint32)
    L.check(L.lib().mr_bp_circle_mask(nu, nu, 0, 0.0, 0, m.ctypes.data_as(L.P_u32)))
    return torch.from_numpy(m.view(np.int32)).cuda()


def _f64(filt, maps, slices, nu, nv, mask):
    n = filt.shape[0]
    out = torch.empty((len(slices), nu, nu), dtype=torch.float64, device="cuda")
    sl = torch.tensor(slices, dtype=torch.int32, device="cuda")
    m = torch.from_numpy(maps).cuda()
    L.check(L.lib().mr_fdk_backproject_f64(filt.data_ptr(), nu, nv, n, m.data_ptr(), mask.data_ptr(), sl.data_ptr(),
                                           len(slices), out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return out.cpu().numpy()


@pytest.mark.parametrize("tilt", [0.0, 0.4])
def test_f64_kernel_matches_oracle(cuda, tilt):
    rng = np.random.default_rng(40)
    nu, nv, n = 48, 40, 24
    proj = rng.standard_normal((n, nv, nu)).astype(np.float32)
    ang = np.sort(rng.uniform(0, 360, n)).astype(np.float32)
    og, g = _geom(nu, nv, (23.37, 19.61), 23.71, 0.2, 0.1, tilt=tilt, pivot=4.0)
    maps = _maps(g, nu, nv, ang)
    assert np.array_equal(maps, O.fdk_maps64(og, nu, nv, ang))
    sl = [0, 3, 17, 39]
    got = _f64(torch.from_numpy(proj).cuda(), maps, sl, nu, nv, _mask(nu))
    exp = O.fdk_bp64(proj, maps, sl)
    assert np.array_equal(got, exp)


def _phantom_filtered(nu, nv, n, pitch, voxel, pp, center):
    ells = phantom.ellipsoids(1004)
    integ = phantom.cone_integrals_torch(ells, n, nu, nv, 300.0, 600.0, pitch, nu * voxel, torch.device("cuda"))
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint = pp
    pi.fCenter = center
    pi.fResolution = (pitch, pitch)
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, n)
    cfg.MatrixInfo.fVoxelSize = (voxel,) * 3
    cfg.MatrixInfo.nDims = (nu, nu, nv)
    fdk = M.FDKbp_single()
    fdk.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1", "precision": "fp32"})
    fdk.SetROI((0, 0, nu, nv))
    ang = (np.arange(n) * 360.0 / n).astype(np.float32)
    w = np.full(n, np.float32(1.0 / n))
    xip, yip, zip_, s2, sc, uni = fdk.partials(ang)
    filt = torch.empty_like(integ)
    wd = torch.from_numpy(w).cuda()
    L.check(L.lib().mr_fdk_filter(integ.data_ptr(), nu, nv, n, wd.data_ptr(), s2, sc, L.MR_F32, filt.data_ptr(), None,
                                  torch.cuda.current_stream().cuda_stream))
    return fdk, filt, ang, (xip, yip, zip_, uni)


def _relrms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


@pytest.mark.parametrize("nu", [128, 256])
def test_fast_paths_against_fp64(cuda, nu):
    nv = n = nu
    pitch, voxel = 0.2 * 1024 / nu, 0.1 * 1024 / nu
    pp, center = ((nu - 1) / 2 + 0.13, (nv - 1) / 2 - 0.21), (nu - 1) / 2 + 0.07
    fdk, filt, ang, (xip, yip, zip_, uni) = _phantom_filtered(nu, nv, n, pitch, voxel, pp, center)
    g = fdk.geometry()
    maps = fdk.maps64(ang)
    mask = fdk._mask
    st = torch.cuda.current_stream().cuda_stream
    sl = sorted(np.random.default_rng(16).choice(nv, 16, replace=False).tolist())
    ref = _f64(filt, maps, sl, nu, nv, mask)
    # FP32 reference-exact path
    X, Y, Z = (torch.from_numpy(a).cuda() for a in (xip, yip, zip_))
    bw, bh = ctypes.c_int(), ctypes.c_int()
    L.check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                               zip_.ctypes.data_as(L.P_float), nu, nv, n, L.MR_F32, ctypes.byref(bw), ctypes.byref(bh)))
    vol = torch.empty((nv, nu, nu), device="cuda")
    L.check(L.lib().mr_fdk_backproject(filt.data_ptr(), L.MR_F32, None, nu, nv, n, X.data_ptr(), Y.data_ptr(),
                                       Z.data_ptr(), uni, mask.data_ptr(), bw.value, bh.value, 0, vol.data_ptr(), st))
    v32 = vol.cpu().numpy()[sl]
    e32 = _relrms(v32, ref)
    b16w, b16h = ctypes.c_int(), ctypes.c_int()
    L.check(L.lib().mr_fdk_box_maps(maps.ctypes.data_as(L.P_double), nu, nv, n, L.MR_BF16, ctypes.byref(b16w),
                                    ctypes.byref(b16h)))
    mf = torch.from_numpy(maps).cuda()
    errs = {}
    for name, dt in (("bf16", L.MR_BF16), ("fp16", L.MR_F16)):
        q, s = M.quantize(filt, name)
        out = torch.empty((nv, nu, nu), device="cuda")
        L.check(L.lib().mr_fdk_backproject_fast(q.data_ptr(), dt, s.data_ptr(), nu, nv, n, mf.data_ptr(), mask.data_ptr(),
                                                b16w.value, b16h.value, 0, out.data_ptr(), st))
        errs[name] = _relrms(out.cpu().numpy()[sl], ref)
    status = ctypes.c_int()
    L.check(L.lib().mr_device_status(ctypes.byref(status)))
    assert status.value == 0
    print(f"nu={nu}: rel RMS vs FP64 fp32 {e32:.3e} bf16 {errs['bf16']:.3e} fp16 {errs['fp16']:.3e}")
    assert e32 < 1e-3
    assert errs["bf16"] < 1e-3
    assert errs["fp16"] < 1e-3


def test_fast_accumulate_in_batches(cuda):
    nu = nv = n = 128
    pitch, voxel = 0.2 * 8, 0.1 * 8
    fdk, filt, ang, _ = _phantom_filtered(nu, nv, n, pitch, voxel, (63.63, 63.29), 63.57)
    maps = fdk.maps64(ang)
    bw, bh = ctypes.c_int(), ctypes.c_int()
    L.check(L.lib().mr_fdk_box_maps(maps.ctypes.data_as(L.P_double), nu, nv, n, L.MR_BF16, ctypes.byref(bw),
                                    ctypes.byref(bh)))
    mf = torch.from_numpy(maps).cuda()
    st = torch.cuda.current_stream().cuda_stream
    q, s = M.quantize(filt, "fp16")
    whole = torch.empty((nv, nu, nu), device="cuda")
    L.check(L.lib().mr_fdk_backproject_fast(q.data_ptr(), L.MR_F16, s.data_ptr(), nu, nv, n, mf.data_ptr(),
                                            fdk._mask.data_ptr(), bw.value, bh.value, 0, whole.data_ptr(), st))
    parts = torch.empty_like(whole)
    h = n // 2
    for k, (a, b) in enumerate(((0, h), (h, n))):
        L.check(L.lib().mr_fdk_backproject_fast(q[a:b].data_ptr(), L.MR_F16, s[a:b].data_ptr(), nu, nv, b - a,
                                                mf[a:b].data_ptr(), fdk._mask.data_ptr(), bw.value, bh.value, k,
                                                parts.data_ptr(), st))
    assert _relrms(parts.cpu().numpy(), whole.cpu().numpy()) < 1e-6


def test_fast_rejects_f32_and_bad_layout(cuda):
    z = torch.zeros(16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert L.lib().mr_fdk_backproject_fast(z.data_ptr(), L.MR_F32, z.data_ptr(), 8, 8, 1, z.data_ptr(), z.data_ptr(),
                                           8, 8, 0, z.data_ptr(), st) == L.MR_ERR_ARGUMENT
    # row pitch 6 x 2 bytes is not a multiple of 16 bytes
    assert L.lib().mr_fdk_backproject_fast(z.data_ptr(), L.MR_BF16, z.data_ptr(), 6, 6, 1, z.data_ptr(), z.data_ptr(),
                                           8, 8, 0, z.data_ptr(), st) == L.MR_ERR_UNSUPPORTED
