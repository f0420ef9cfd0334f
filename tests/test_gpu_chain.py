"""Parity at the benchmark configurations and along the chains (gpu).

* The device chains (pipeline.ParallelChain, pipeline.FdkPipeline) against the same modules
  chained in the oracle, from uint16 counts to the volume: FullLogNorm -> [MorphSpotClean ->
  WaveletRingClean] -> ProjectionFilterSingle -> MultiProjectionBPparallel, and FullLogNorm ->
  FDKbp_single. The parallel chain at the C1 shape (360 projections of 256 x 64, centre
  127.5) is also compared with the reference's own modules chained on the CPU.
* FDK at the C2 geometry (512 x 512 detector at 0.2 mm, SOD 300 mm, SDD 600 mm, 512^3 voxels
  of 0.1 mm, angles of a 720-projection scan) and the C4 geometry (1024^2 detector, 1024^3
  voxels) on a few projections of those scans: backprojection bit for bit given the oracle's
  filtered projections, and the whole FDKbp_single module within 1e-5 relative RMS.

FP32 volumes: the chains differ from the oracle only where CUDA's logf differs from glibc's by
an ulp (FullLogNorm) and where the projection/FDK filters' FP32 FFT differs from the oracle's
FP64 FFT; the bar is the 1e-5 relative RMS of FP32 volumes.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M
from imagingsuite_b200 import phantom, pipeline

pytestmark = pytest.mark.gpu


def relrms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def _status_ok():
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    assert st.value == 0


def _parallel_chain(cuda, nu, nv, nproj, seed, defects):
    integ = phantom.parallel_integrals_torch(phantom.ellipsoids(seed), nproj, nu, nv, cuda)
    counts, flats, darks = phantom.counts_torch(integ, 3e4, 1000 + seed, 5, 5)
    if defects:
        phantom.inject_defects_torch(counts, flats, 3000 + seed)
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter = (nu - 1) / 2.0
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    pi.nOBCount, pi.nDCCount = 5, 5
    norm = M.FullLogNorm()
    norm.Configure(cfg, {"usenormregion": "false", "uselut": "false", "referenceaverage": "ImageAverage"})
    norm.SetReferenceImages(darks, flats)
    spot = ring = None
    if defects:
        spot = M.MorphSpotCleanModule()
        spot.Configure(cfg, {"connectivity": "conn8", "cleanmethod": "morphcleanreplace",
                             "detectionmethod": "morphdetectboth", "threshold": "0.1 0.1", "sigma": "0.01 0.01",
                             "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false", "clampdata": "false",
                             "minlevel": "-0.1", "maxlevel": "12", "threading": "false"})
        ring = M.WaveletRingClean()
        ring.Configure(cfg, {"wname": "daub15", "sigma": "0.05", "decnum": "2", "parallel": "false",
                             "method": "verticalfft"})
    filt = M.ProjectionFilterSingle()
    filt.Configure(cfg, {"filtertype": "hanning", "cutoff": "0.5", "order": "1", "usebias": "true",
                         "biasweight": "0.1", "paddingdoubler": "2"})
    bp = M.MultiProjectionBPparallel()
    bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1", "precision": "fp32",
                       "referencecompat": "true"})
    bp.SetROI((0, 0, nu, nv))
    angles = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    weights = np.full(nproj, np.float32(np.pi / nproj))
    chain = pipeline.ParallelChain(norm, filt, bp, angles, weights, spot=spot, ring=ring)
    vol = chain.run_device(counts).cpu().numpy()
    return (vol, counts.cpu().numpy().astype(np.float32), darks.cpu().numpy(), flats.cpu().numpy(), angles, weights,
            pi.fCenter)


def _oracle_parallel_chain(counts, darks, flats, angles, weights, centre, defects):
    refs = O.lognorm_refs(darks, flats, "ImageAverage", False)
    p = O.lognorm_apply(counts, refs.dark, refs.logflat, np.zeros(1, np.float32))
    if defects:
        # MorphSpotCleanModule runs the cleaner with edge 9 and without removeinfnan
        p = O.morphspotclean(p, "both", True, (0.1, 0.1), (0.01, 0.01), edge=9, clamp=False)
        p = O.waveletringclean(p, "daub15", 2, 0.05)
    plan = O.projfilter_plan(counts.shape[2], "hanning", 0.5, 1.0, True, 0.1, 2)
    p = O.projfilter(p, plan)
    return O.bp_parallel(p, angles, weights, centre, buffersize=16)


def test_parallel_chain_c1_matches_oracle_and_reference(cuda):
    """C1: FullLogNorm(u16) -> Hann filter -> MultiProjectionBPparallel on the device against
    the oracle chain and against the reference's own modules chained on the CPU."""
    nu, nv, nproj = 256, 64, 360
    vol, counts, darks, flats, ang, w, c = _parallel_chain(cuda, nu, nv, nproj, 1001, False)
    exp = _oracle_parallel_chain(counts, darks, flats, ang, w, c, False)
    assert relrms(vol, exp) < 1e-5
    if O.ref_available():
        p = O.ref_fulllognorm(counts, darks, flats, "ImageAverage", False)[0]
        p = O.ref_projfilter(p, "hanning", 0.5, 1.0, True, 0.1, 2)[0]
        ref = O.bp_parallel(p, ang, w, c, buffersize=16, use_ref=True)
        assert relrms(vol, ref) < 1e-5
    _status_ok()


def test_parallel_chain_with_cleaning_matches_oracle(cuda):
    """The C3 chain (spots and ring columns injected): FullLogNorm -> MorphSpotClean ->
    WaveletRingClean -> Hann filter -> backprojection, device vs oracle."""
    nu, nv, nproj = 128, 32, 120
    vol, counts, darks, flats, ang, w, c = _parallel_chain(cuda, nu, nv, nproj, 1003, True)
    exp = _oracle_parallel_chain(counts, darks, flats, ang, w, c, True)
    assert relrms(vol, exp) < 1e-5
    _status_ok()


def _fdk_config(nu, nv, nproj, pitch, voxel):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint, pi.fCenter = ((nu - 1) / 2.0 + 0.13, (nv - 1) / 2.0 - 0.21), (nu - 1) / 2.0 + 0.07
    pi.fResolution = (pitch, pitch)
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    pi.nOBCount, pi.nDCCount = 10, 10
    cfg.MatrixInfo.fVoxelSize = (voxel,) * 3
    cfg.MatrixInfo.nDims = (nu, nu, nv)
    return cfg


def _ogeom(cfg):
    pi = cfg.ProjectionInfo
    return O.fdk_geom(pi.fSOD, pi.fSDD, pi.fpPoint, pi.fCenter, pi.fResolution, cfg.MatrixInfo.fVoxelSize)


def test_fdk_pipeline_matches_oracle_chain(cuda):
    """FdkPipeline.run_device (FullLogNorm(u16) -> FDK ramp filter -> FDK backprojection)
    against FullLogNorm -> FDKbp_single in the oracle."""
    nu, nv, nproj = 96, 64, 48
    cfg = _fdk_config(nu, nv, nproj, 0.8, 0.4)
    integ = phantom.cone_integrals_torch(phantom.ellipsoids(1004), nproj, nu, nv, 300.0, 600.0, 0.8, nu * 0.4, cuda)
    counts, flats, darks = phantom.counts_torch(integ, 5e4, 2004, 10, 10)
    angles = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    weights = np.full(nproj, np.float32(1.0 / nproj))
    pipe = pipeline.FdkPipeline(cfg, angles, weights, darks, flats)
    vol = pipe.run_device(counts).cpu().numpy()
    refs = O.lognorm_refs(darks.cpu().numpy(), flats.cpu().numpy(), "ImageAverage", False)
    p = O.lognorm_apply(counts.cpu().numpy().astype(np.float32), refs.dark, refs.logflat, np.zeros(1, np.float32))
    exp = O.fdk(p, angles, weights, _ogeom(cfg))
    assert relrms(vol, exp) < 1e-5
    _status_ok()


@pytest.mark.parametrize("name,nu,nscan,pitch,voxel,pick", [
    ("C2", 512, 720, 0.2, 0.1, (0, 97, 251, 360, 533)),
    ("C4", 1024, 1024, 0.2, 0.1, (0, 301)),
])
def test_fdk_benchmark_geometry(cuda, name, nu, nscan, pitch, voxel, pick):
    """The benchmark geometries at full detector and volume size, on a few projections of the
    scan: the backprojection of the oracle's filtered projections is bit-identical, and the
    FDKbp_single module (ramp filter + backprojection) is within 1e-5 relative RMS."""
    nv = nu
    cfg = _fdk_config(nu, nv, nscan, pitch, voxel)
    g = _ogeom(cfg)
    rng = np.random.default_rng(nu)
    pick = np.asarray(pick)
    proj = (rng.standard_normal((pick.size, nv, nu)) * 0.2 + 1.0).astype(np.float32)
    angles = (pick * 360.0 / nscan).astype(np.float32)
    weights = np.full(pick.size, np.float32(1.0 / nscan))
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    text = lambda v: " ".join("%.9g" % x for x in v)
    mod.Process(torch.from_numpy(proj).to(cuda), {"angles": text(angles), "weights": text(weights)})
    got = mod.GetVolume().cpu().numpy()
    # the oracle's FDKbp_single: its ramp filter and scaling, then its backprojection
    filt = O.fdk_prepare(proj, weights, g)
    exp_bp = O.fdk_bp(filt, angles, g)
    assert relrms(got, exp_bp) < 1e-5, name
    del got
    # backprojection alone, bit for bit, from the oracle's prepared projections
    xip, yip, zip_, s2, sc, uni = mod.partials(angles)
    bw, bh = ctypes.c_int(0), ctypes.c_int(0)
    L.check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                               zip_.ctypes.data_as(L.P_float), nu, nv, pick.size, L.MR_F32, ctypes.byref(bw),
                               ctypes.byref(bh)))
    X, Y, Z = (torch.from_numpy(a).to(cuda) for a in (xip, yip, zip_))
    src = torch.from_numpy(filt).to(cuda)
    vol = torch.empty((nv, nu, nu), device=cuda)
    L.check(L.lib().mr_fdk_backproject(src.data_ptr(), L.MR_F32, None, nu, nv, pick.size, X.data_ptr(), Y.data_ptr(),
                                       Z.data_ptr(), uni, mod._mask.data_ptr(), bw.value, bh.value, 0, vol.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream))
    assert np.array_equal(vol.cpu().numpy(), exp_bp), name
    _status_ok()
