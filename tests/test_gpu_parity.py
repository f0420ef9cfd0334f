"""CUDA path against the oracle, through the C ABI (gpu).

Bars: bit-exact for the integer dark/flat arithmetic, reference averaging, doses and the
backprojection geometry/accumulation (given identical filtered projections); the log in
FullLogNorm within 1 ulp (CUDA logf vs glibc logf); FFT-based filters within 1e-5
relative RMS (float FFT vs the oracle's FP64 FFT); full FP32 volumes within 1e-5
relative RMS of the oracle.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu


def relrms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / max(np.mean(b ** 2), 1e-300)))


def ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def dev(x, cuda):
    return torch.from_numpy(np.ascontiguousarray(x)).to(cuda)


def stream():
    return torch.cuda.current_stream().cuda_stream


# ------------------------------------------------------------------ FullLogNorm


def _counts(seed, nproj, nv, nu):
    rng = np.random.default_rng(seed)
    darks = np.round(rng.normal(100, 3, (5, nv, nu))).astype(np.uint16)
    flats = (rng.poisson(30000, (5, nv, nu)) + 100).astype(np.uint16)
    proj = (rng.poisson(15000, (nproj, nv, nu)) + 100).astype(np.uint16)
    proj[0, 0, :7] = 60  # I - D <= 0
    return proj, flats, darks


@pytest.mark.parametrize("usenorm", [False, True])
@pytest.mark.parametrize("method", ["ImageAverage", "ImageSum", "ImageMedian", "ImageMax", "ImageWeightedAverage"])
def test_fulllognorm_module(cuda, usenorm, method):
    proj, flats, darks = _counts(1, 13, 20, 36)
    roi = (3, 2, 30, 17)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.dose_roi = roi
    cfg.ProjectionInfo.nOBCount, cfg.ProjectionInfo.nDCCount = 5, 5
    mod = M.FullLogNorm()
    mod.Configure(cfg, {"usenormregion": str(usenorm).lower(), "uselut": "false", "referenceaverage": method})
    mod.SetReferenceImages(dev(darks, cuda), dev(flats, cuda))
    out = mod.Process(dev(proj, cuda), {}).cpu().numpy()

    refs = O.lognorm_refs(darks.astype(np.float32), flats.astype(np.float32), method, usenorm, roi)
    assert np.array_equal(mod.mDark.cpu().numpy(), refs.dark)            # averaging: exact
    assert (mod.fDarkDose, mod.fFlatDose) == (refs.darkdose, refs.flatdose)  # doses: exact
    assert ulps(mod.mFlatField.cpu().numpy(), refs.logflat).max() <= 1
    if usenorm:
        doses = np.array([O.frame_dose(proj[i].astype(np.float32), roi) for i in range(proj.shape[0])], np.float32)
        dl = O.lognorm_doselog(doses, refs.darkdose)
    else:
        dl = np.zeros(1, np.float32)
    exp = O.lognorm_apply(proj.astype(np.float32), refs.dark, refs.logflat, dl)
    # CUDA logf and glibc logf may differ by 1 ulp of log(I - D); the difference of two logs
    # carries that absolute error, so the bar is 2 ulp of the log terms' magnitude
    tol = 2 * np.spacing(np.float32(np.abs(refs.logflat).max() + np.abs(dl).max()))
    assert np.abs(out.astype(np.float64) - exp).max() <= tol
    assert np.mean(out == exp) > 0.9
    assert np.array_equal(out == 0, exp == 0)  # the (I - D <= 0) mask is exact


@pytest.mark.parametrize("ndark,nflat", [(5, 0), (0, 5), (0, 0)])
@pytest.mark.parametrize("usenorm", [False, True])
@pytest.mark.parametrize("uselut", [False, True])
def test_fulllognorm_module_missing_references(cuda, ndark, nflat, usenorm, uselut):
    """FullLogNorm without flat fields (-log(I - D) + dose, NormPlugins.cpp:498-540 and the LUT
    path's dose shift), without darks (I alone), or with neither, through the module, against
    the oracle (pinned to the compiled module on these branches)."""
    proj, flats, darks = _counts(3, 11, 20, 36)
    darks, flats = darks[:ndark], flats[:nflat]
    roi = (3, 2, 30, 17)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.dose_roi = roi
    cfg.ProjectionInfo.nOBCount, cfg.ProjectionInfo.nDCCount = nflat, ndark
    mod = M.FullLogNorm()
    mod.Configure(cfg, {"usenormregion": str(usenorm).lower(), "uselut": str(uselut).lower(),
                        "referenceaverage": "ImageAverage"})
    mod.SetReferenceImages(dev(darks.reshape(ndark, 20, 36), cuda), dev(flats.reshape(nflat, 20, 36), cuda))
    out = mod.Process(dev(proj, cuda), {}).cpu().numpy()
    refs = O.lognorm_refs(darks.reshape(ndark, 20, 36).astype(np.float32),
                          flats.reshape(nflat, 20, 36).astype(np.float32), "ImageAverage", usenorm, roi)
    if usenorm:
        doses = np.array([O.frame_dose(proj[i].astype(np.float32), roi) for i in range(proj.shape[0])], np.float32)
        dl = O.lognorm_doselog(doses, refs.darkdose)
    else:
        dl = np.zeros(1, np.float32)
    exp = O.lognorm_apply(proj.astype(np.float32), refs.dark, refs.logflat, dl, ndc=ndark > 0, nob=nflat > 0,
                          uselut=uselut)
    if uselut and nflat == 0:
        assert np.array_equal(out, exp)  # the table is built with the reference's double log
    else:
        # log(flat) (and, on the exact path, log(I - D)) through CUDA's logf: within 1 ulp of glibc's
        tol = 2 * np.spacing(np.float32(np.abs(refs.logflat).max() + np.abs(dl).max() + np.log(65536.0)))
        assert np.abs(out.astype(np.float64) - exp).max() <= tol
        if not uselut:
            assert np.array_equal(out == 0, exp == 0)


def test_lognorm_f32_inplace_and_unaligned(cuda):
    proj, flats, darks = _counts(2, 3, 7, 13)  # npix = 91: scalar path
    refs = O.lognorm_refs(darks.astype(np.float32), flats.astype(np.float32))
    p = dev(proj.astype(np.float32), cuda)
    d, lf = dev(refs.dark, cuda), dev(refs.logflat, cuda)
    dl = torch.zeros(1, device=cuda)
    L.check(L.lib().mr_lognorm_apply(p.data_ptr(), L.MR_F32, 91, 3, d.data_ptr(), lf.data_ptr(), dl.data_ptr(), 1, 1, 1,
                                     p.data_ptr(), stream()))
    exp = O.lognorm_apply(proj.astype(np.float32), refs.dark, refs.logflat, np.zeros(1, np.float32))
    assert np.abs(p.cpu().numpy().astype(np.float64) - exp).max() <= 2 * np.spacing(np.float32(np.abs(refs.logflat).max()))


def test_lognorm_rejects_bad_arguments(cuda):
    x = torch.zeros(10, device=cuda)
    st = L.lib().mr_lognorm_apply(x.data_ptr(), L.MR_F32, 10, 2, x.data_ptr(), x.data_ptr(), x.data_ptr(), 3, 1, 1,
                                  x.data_ptr(), stream())
    assert st == L.MR_ERR_ARGUMENT
    with pytest.raises(M.ReconException):
        mod = M.FullLogNorm()
        mod.Configure(M.ReconConfig(), {"usenormregion": "false", "referenceaverage": "ImageAverage"})
        mod.Process(torch.zeros((1, 4, 4), device=cuda), {})


@pytest.mark.parametrize("dtype", ["u16", "f32"])
@pytest.mark.parametrize("ndc,nob", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_lognorm_lut_bit_exact(cuda, dtype, ndc, nob):
    """The uselut path through the C ABI with the oracle's reference images: the LogLUT is
    built on the host with the reference's double log, so the GPU equals the oracle bit for bit
    (values at or below 0, above 65535, and per-projection doses included)."""
    proj, flats, darks = _counts(3, 13, 20, 36)
    proj[0, 1, :3] = 65000
    refs = O.lognorm_refs(darks.astype(np.float32), flats.astype(np.float32))
    dl = np.linspace(-0.1, 0.2, proj.shape[0]).astype(np.float32)
    exp = O.lognorm_apply(proj.astype(np.float32), refs.dark, refs.logflat, dl, ndc=bool(ndc), nob=bool(nob),
                          uselut=True)
    src = dev(proj, cuda) if dtype == "u16" else dev(proj.astype(np.float32), cuda)
    out = torch.empty(proj.shape, dtype=torch.float32, device=cuda)
    d, lf, dd = dev(refs.dark, cuda), dev(refs.logflat, cuda), dev(dl, cuda)
    L.check(L.lib().mr_lognorm_apply_lut(src.data_ptr(), L.MR_U16 if dtype == "u16" else L.MR_F32, 20 * 36,
                                         proj.shape[0], d.data_ptr(), lf.data_ptr(), dd.data_ptr(), dl.size, ndc, nob,
                                         out.data_ptr(), stream()))
    assert np.array_equal(out.cpu().numpy().view(np.uint32), exp.view(np.uint32))


def test_fulllognorm_lut_module(cuda):
    """The module with uselut=true: the LUT path after the module's own reference images (whose
    log(flat) is CUDA logf, within 1 ulp of glibc)."""
    proj, flats, darks = _counts(4, 13, 20, 36)
    mod = M.FullLogNorm()
    mod.Configure(M.ReconConfig(), {"usenormregion": "false", "uselut": "true", "referenceaverage": "ImageAverage"})
    assert mod.GetParameters()["uselut"] == "true"
    mod.SetReferenceImages(dev(darks, cuda), dev(flats, cuda))
    out = mod.Process(dev(proj, cuda), {}).cpu().numpy()
    refs = O.lognorm_refs(darks.astype(np.float32), flats.astype(np.float32))
    exp = O.lognorm_apply(proj.astype(np.float32), refs.dark, refs.logflat, np.zeros(1, np.float32), uselut=True)
    tol = 2 * np.spacing(np.float32(np.abs(refs.logflat).max() + 12.0))
    assert np.abs(out.astype(np.float64) - exp).max() <= tol


@pytest.mark.parametrize("shape", [(1, 5, 5), (3, 6, 7), (10, 33, 41), (20, 256, 300)])
def test_weighted_average_matches_oracle(cuda, shape):
    """ImageWeightedAverage on the GPU: per-frame 5x5 standard deviation (EdgeMirror) and the
    1/sigma weights, bit for bit."""
    rng = np.random.default_rng(sum(shape))
    st = rng.poisson(1000, shape).astype(np.float32)
    st[:, 2:5, 1:4] = 700.0
    st[0, 0, :] = 1e4
    out = torch.empty(shape[1:], device=cuda)
    x = dev(st, cuda)
    L.check(L.lib().mr_reference_average(x.data_ptr(), shape[2], shape[1], shape[0], 3, out.data_ptr(), stream()))
    exp = O.average(st, "ImageWeightedAverage")
    assert np.array_equal(out.cpu().numpy().view(np.uint32), exp.view(np.uint32))


# ------------------------------------------------------------ ProjectionFilterSingle


@pytest.mark.parametrize("ftype", ["ram-lak", "shepp-logan", "hanning", "hamming", "butterworth"])
@pytest.mark.parametrize("nu,pd,cutoff", [(256, 2, 0.5), (100, 1, 0.3), (2048, 2, 0.5), (37, 0, 0.25)])
def test_projfilter(cuda, ftype, nu, pd, cutoff):
    rng = np.random.default_rng(nu)
    proj = rng.standard_normal((3, 5, nu)).astype(np.float32) + 2.0
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.roi = (0, 0, nu, 5)
    mod = M.ProjectionFilterSingle()
    mod.Configure(cfg, {"filtertype": ftype, "cutoff": str(cutoff), "order": "2", "usebias": "true",
                        "biasweight": "0.1", "paddingdoubler": str(pd)})
    out = mod.Process(dev(proj, cuda)).cpu().numpy()
    exp = O.projfilter(proj, O.projfilter_plan(nu, ftype, cutoff, 2.0, True, 0.1, pd))
    assert relrms(out, exp) < 1e-5


def test_projfilter_fused_weights(cuda):
    rng = np.random.default_rng(5)
    proj = rng.standard_normal((4, 6, 128)).astype(np.float32)
    w = rng.uniform(0.5, 2, 4).astype(np.float32)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.roi = (0, 0, 128, 6)
    mod = M.ProjectionFilterSingle()
    mod.Configure(cfg, {"filtertype": "hanning", "cutoff": "0.5", "order": "1", "usebias": "true",
                        "biasweight": "0.1", "paddingdoubler": "2"})
    a = mod.Process(dev(proj, cuda), weights=dev(w, cuda)).cpu().numpy()
    b = mod.Process(dev(proj, cuda)).cpu().numpy() * w[:, None, None]
    assert relrms(a, b) < 1e-6


# ------------------------------------------------------------------- parallel beam


def _bp_module(cfg, nu, nv, buffersize=16, compat=True, precision="fp32"):
    bp = M.MultiProjectionBPparallel()
    bp.Configure(cfg, {"ProjectionBufferSize": str(buffersize), "SliceBlock": "32", "SubVolume": "1 1",
                       "referencecompat": str(compat).lower(), "precision": precision})
    bp.SetROI((0, cfg.ProjectionInfo.roi[1], nu, cfg.ProjectionInfo.roi[1] + nv))
    return bp


def _text(a):
    return " ".join("%.9g" % v for v in a)


@pytest.mark.parametrize("tilt", [False, True])
@pytest.mark.parametrize("direction", [0, 1])
def test_bp_parallel_bit_exact(cuda, tilt, direction):
    rng = np.random.default_rng(7)
    nproj, nv, nu = 45, 16, 64
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter, pi.eDirection, pi.bCorrectTilt, pi.fTiltAngle, pi.fTiltPivotPosition = 31.3, direction, tilt, 0.6, 2.0
    pi.roi = (0, 3, nu, 3 + nv)
    pi.nDims = (nu, nv, nproj)
    bp = _bp_module(cfg, nu, nv)
    bp.Process(dev(proj, cuda), {"angles": _text(ang), "weights": _text(w)})
    vol = bp.GetVolume().cpu().numpy()
    exp = O.bp_parallel(proj, ang, w, 31.3, direction=direction, buffersize=16, correcttilt=tilt, tiltangle=0.6,
                        tiltpivot=2.0, roi_y0=3, nslices=nv)
    assert np.array_equal(vol, exp)


@pytest.mark.parametrize("nproj,nv,nu", [(360, 64, 256), (17, 7, 33), (5, 4, 2), (1, 8, 31)])
def test_bp_parallel_sizes(cuda, nproj, nv, nu):
    rng = np.random.default_rng(nu)
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = np.full(nproj, np.float32(np.pi / nproj))
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.fCenter = (nu - 1) / 2.0
    cfg.ProjectionInfo.roi = (0, 0, nu, nv)
    bp = _bp_module(cfg, nu, nv)
    bp.Process(dev(proj, cuda), {"angles": _text(ang), "weights": _text(w)})
    exp = O.bp_parallel(proj, ang, w, (nu - 1) / 2.0, buffersize=16)
    assert np.array_equal(bp.GetVolume().cpu().numpy(), exp)


@pytest.mark.parametrize("variant", ["serial", "nn"])
@pytest.mark.parametrize("tilt", [False, True])
@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("nproj,nv,nu", [(45, 16, 64), (37, 7, 33), (61, 10, 96), (200, 40, 128)])
def test_bp_variants_bit_exact(cuda, variant, tilt, direction, nproj, nv, nu):
    """MultiProjectionBP (serial) and NearestNeighborBP on the GPU equal the oracle's
    restatements, which equal the compiled reference modules bit for bit: with and without
    tilt, both directions, slice counts that are and are not multiples of 4, staged (nu a
    multiple of 4, no tilt) and direct kernels."""
    rng = np.random.default_rng(nproj + 3 * nv + direction)
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    c = (nu - 1) / 2.0 + 0.31
    pi.fCenter, pi.eDirection, pi.bCorrectTilt, pi.fTiltAngle, pi.fTiltPivotPosition = c, direction, tilt, 0.6, 2.0
    pi.roi = (0, 3, nu, 3 + nv)
    pi.nDims = (nu, nv, nproj)
    bp = M.MultiProjectionBP() if variant == "serial" else M.NearestNeighborBP()
    bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    bp.SetROI((0, 3, nu, 3 + nv))
    bp.Process(dev(proj, cuda), {"angles": _text(ang), "weights": _text(w)})
    vol = bp.GetVolume().cpu().numpy()
    exp = O.bp_parallel(proj, ang, w, c, direction=direction, buffersize=16, correcttilt=tilt, tiltangle=0.6,
                        tiltpivot=2.0, roi_y0=3, nslices=nv, serial=variant == "serial", nn=variant == "nn")
    assert np.array_equal(vol, exp)
    status = ctypes.c_int()
    L.check(L.lib().mr_device_status(ctypes.byref(status)))
    assert status.value == 0


def test_bp_nearest_rows_equal_whole(cuda):
    """NearestNeighborBP by row blocks (the pipeline's form) equals the whole-volume call."""
    rng = np.random.default_rng(5)
    nproj, nv, nu = 90, 24, 128
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 2.0).astype(np.float32)
    w = np.ones(nproj, np.float32)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.fCenter = 63.2
    cfg.ProjectionInfo.roi = (0, 0, nu, nv)
    vols = []
    for rows in (None, [(0, 40), (40, 41), (41, nu)]):
        bp = M.NearestNeighborBP()
        bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
        bp.SetROI((0, 0, nu, nv))
        for r in rows or [None]:
            bp.Process(dev(proj, cuda), {"angles": _text(ang), "weights": _text(w)}, rows=r)
        vols.append(bp.GetVolume().cpu().numpy())
    assert np.array_equal(vols[0], vols[1])
    assert np.array_equal(vols[0], O.bp_parallel(proj, ang, w, 63.2, buffersize=16, nn=True))


def test_bp_parallel_all_projections_mode(cuda):
    """referencecompat=false backprojects every projection (no buffer-drop rule)."""
    rng = np.random.default_rng(8)
    nproj, nv, nu = 40, 8, 48
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 4.5).astype(np.float32)
    w = np.ones(nproj, np.float32)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.fCenter = 23.5
    cfg.ProjectionInfo.roi = (0, 0, nu, nv)
    bp = _bp_module(cfg, nu, nv, compat=False)
    bp.Process(dev(proj, cuda), {"angles": _text(ang), "weights": _text(w)})
    exp = O.bp_parallel(proj, ang, w, 23.5, buffersize=1024)  # one buffer flush: nothing dropped
    assert np.array_equal(bp.GetVolume().cpu().numpy(), exp)


# -------------------------------------------------------------------------- FDK


def _fdk_cfg(nu, nv, pp=None, direction=0, tilt=False):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint = pp if pp is not None else ((nu - 1) / 2.0, (nv - 1) / 2.0)
    pi.fCenter = (nu - 1) / 2.0 + 0.3
    pi.fResolution = (0.2, 0.2)
    pi.eDirection = direction
    pi.bCorrectTilt, pi.fTiltAngle, pi.fTiltPivotPosition = tilt, 0.5, nv / 2.0
    pi.nDims = (nu, nv, 0)
    cfg.MatrixInfo.fVoxelSize = (0.1, 0.1, 0.1)
    return cfg


def _ogeom(cfg):
    pi = cfg.ProjectionInfo
    return O.fdk_geom(pi.fSOD, pi.fSDD, pi.fpPoint, pi.fCenter, pi.fResolution, cfg.MatrixInfo.fVoxelSize,
                      pi.eDirection, pi.bCorrectTilt, pi.fTiltAngle, pi.fTiltPivotPosition)


def test_fdk_filter(cuda):
    rng = np.random.default_rng(11)
    nproj, nv, nu = 6, 40, 96
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32) + 1.0
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    cfg = _fdk_cfg(nu, nv)
    g = _ogeom(cfg)
    exp = O.fdk_prepare(proj, w, g)
    out = torch.empty((nproj, nv, nu), device=cuda)
    sc = np.float32(300.0) / np.float32(600.0)
    s2 = np.float32(np.float32(300.0 * 300.0) / np.float32(600.0 * 600.0))
    L.check(L.lib().mr_fdk_filter(dev(proj, cuda).data_ptr(), nu, nv, nproj, dev(w, cuda).data_ptr(), float(s2),
                                  float(sc), L.MR_F32, out.data_ptr(), None, stream()))
    assert relrms(out.cpu().numpy(), exp) < 1e-5


def _fdk_bp_gpu(cuda, mod, filt, ang, staged, dtype=L.MR_F32, scale=None, box=None):
    nproj, nv, nu = filt.shape
    xip, yip, zip_, s2, sc, uni = mod.partials(ang)
    bw, bh = ctypes.c_int(0), ctypes.c_int(0)
    if box is not None:
        bw.value, bh.value = box
    elif staged and uni:
        L.check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                                   zip_.ctypes.data_as(L.P_float), nu, nv, nproj, dtype, ctypes.byref(bw),
                                   ctypes.byref(bh)))
        assert bw.value > 0 and bh.value > 0
    vol = torch.empty((nv, nu, nu), device=cuda)
    X, Y, Z = (dev(a, cuda) for a in (xip, yip, zip_))
    src = dev(filt, cuda)
    L.check(L.lib().mr_fdk_backproject(src.data_ptr(), dtype, None if scale is None else scale.data_ptr(), nu, nv,
                                       nproj, X.data_ptr(), Y.data_ptr(), Z.data_ptr(), uni, mod._mask.data_ptr(),
                                       bw.value, bh.value, 0, vol.data_ptr(), stream()))
    status = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(status)))
    assert status.value == 0
    return vol.cpu().numpy(), uni


@pytest.mark.parametrize("staged", [True, False])
@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("pp", [None, (40.0, 31.3)])
@pytest.mark.parametrize("tilt", [False, True])
def test_fdk_backproject_bit_exact(cuda, staged, direction, pp, tilt):
    """Given identical prepared projections the GPU FDK volume equals the oracle's bit for bit,
    through the TMA-staged kernel and through the direct-load kernel."""
    rng = np.random.default_rng(12)
    nproj, nv, nu = 12, 40, 64
    cfg = _fdk_cfg(nu, nv, pp, direction, tilt)
    g = _ogeom(cfg)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 30.0).astype(np.float32)
    exp = O.fdk_bp(filt, ang, g)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    got, uni = _fdk_bp_gpu(cuda, mod, filt, ang, staged)
    assert uni == (0 if tilt else 1)
    assert np.array_equal(got, exp)


def test_fdk_staged_box_too_small_falls_back(cuda):
    """Footprints larger than the staging box take the direct-load path: same volume."""
    rng = np.random.default_rng(14)
    nproj, nv, nu = 6, 40, 64
    cfg = _fdk_cfg(nu, nv)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 60.0).astype(np.float32)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    got, _ = _fdk_bp_gpu(cuda, mod, filt, ang, True, box=(8, 8))
    assert np.array_equal(got, O.fdk_bp(filt, ang, _ogeom(cfg)))


@pytest.mark.parametrize("box", [(20, 44), (28, 40), (36, 36)])
def test_fdk_staged_mixed_fallback_groups(cuda, box):
    """Boxes that hold the footprints of some projections of a batch but not of others (the
    footprint's width on the detector turns with the angle): the staged and the direct-load
    projections of one group still accumulate in projection order, bit for bit."""
    rng = np.random.default_rng(15)
    nproj, nv, nu = 24, 40, 64
    cfg = _fdk_cfg(nu, nv)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 15.0 + 2.0).astype(np.float32)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    got, _ = _fdk_bp_gpu(cuda, mod, filt, ang, True, box=box)
    assert np.array_equal(got, O.fdk_bp(filt, ang, _ogeom(cfg)))


@pytest.mark.parametrize("shape", [(9, 72, 96), (5, 33, 40), (7, 64, 128)])
def test_fdk_staged_shapes(cuda, shape):
    """Partial slice tiles (nv not a multiple of 32), odd tile counts, wide detectors."""
    rng = np.random.default_rng(shape[1])
    nproj, nv, nu = shape
    cfg = _fdk_cfg(nu, nv)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 360.0 / nproj + 3.0).astype(np.float32)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    got, _ = _fdk_bp_gpu(cuda, mod, filt, ang, True)
    assert np.array_equal(got, O.fdk_bp(filt, ang, _ogeom(cfg)))


def test_fdk_module_end_to_end(cuda):
    rng = np.random.default_rng(13)
    nproj, nv, nu = 24, 48, 64
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32) + 0.5
    ang = (np.arange(nproj) * 15.0).astype(np.float32)
    w = np.full(nproj, np.float32(0.25))
    cfg = _fdk_cfg(nu, nv)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    p = {"angles": _text(ang), "weights": _text(w)}
    mod.Process(dev(proj[:10], cuda), {"angles": _text(ang[:10]), "weights": _text(w[:10])})
    mod.Process(dev(proj[10:], cuda), {"angles": _text(ang[10:]), "weights": _text(w[10:])})  # accumulates
    exp = O.fdk(proj, ang, w, _ogeom(cfg))
    assert relrms(mod.GetVolume().cpu().numpy(), exp) < 1e-5
    assert p  # parameters use the engine's text form


def test_fdk_rejects_short_detector(cuda):
    x = torch.zeros((1, 8, 16), device=cuda)
    st = L.lib().mr_fdk_filter(x.data_ptr(), 16, 8, 1, None, 1.0, 1.0, L.MR_F32, x.data_ptr(), None, stream())
    assert st == L.MR_ERR_ARGUMENT


@pytest.mark.parametrize("nproj,nv,nu,weighted", [(45, 70, 100, True), (203, 33, 64, False), (9, 4, 48, True),
                                                  (360, 96, 256, False)])
def test_bp_parallel_staged_equals_plain(cuda, nproj, nv, nu, weighted):
    """The TMA-staged parallel backprojector is bit-identical to the plain kernel (partial slice
    tiles, batches not filling the last stage, weights applied or pre-applied) and to the oracle."""
    rng = np.random.default_rng(nproj + nv)
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = np.sort(rng.uniform(0, 180, nproj)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.fCenter = (nu - 1) / 2.0 + 0.37
    cfg.ProjectionInfo.roi = (0, 0, nu, nv)
    vols = []
    for staging in (True, False):
        bp = _bp_module(cfg, nu, nv)
        bp.staging = staging
        bp.Process(dev(proj if weighted else proj * w[:, None, None], cuda), {"angles": _text(ang), "weights": _text(w)},
                   prefiltered_weights=not weighted)
        vols.append(bp.GetVolume().cpu().numpy())
    assert np.array_equal(vols[0], vols[1])
    if weighted:
        assert np.array_equal(vols[0], O.bp_parallel(proj, ang, w, (nu - 1) / 2.0 + 0.37, buffersize=16))
    status = ctypes.c_int()
    L.check(L.lib().mr_device_status(ctypes.byref(status)))
    assert status.value == 0
