"""The device-resident FDK chain (gpu): the end-to-end form that streams the counts in by
groups of projections and copies the volume out by slice blocks while the next block is
backprojected gives the same volume, bit for bit, as the one-shot device form, and so do
the slice blocks of mr_fdk_backproject_slab against one whole-volume call."""
import ctypes

import numpy as np
import pytest
import torch

from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M
from imagingsuite_b200 import pipeline

pytestmark = pytest.mark.gpu


def _config(nu, nv, nproj):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint, pi.fCenter = ((nu - 1) / 2 + 0.13, (nv - 1) / 2 - 0.21), (nu - 1) / 2 + 0.07
    pi.fResolution = (3.2, 3.2)
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    pi.nOBCount, pi.nDCCount = 3, 2
    cfg.MatrixInfo.fVoxelSize = (1.6, 1.6, 1.6)
    cfg.MatrixInfo.nDims = (nu, nu, nv)
    return cfg


@pytest.mark.parametrize("nu,nv,nproj,chunks,slabs", [(64, 96, 20, 6, 8), (96, 64, 13, 4, 2)])
def test_host_pipeline_equals_device_pipeline(cuda, nu, nv, nproj, chunks, slabs):
    rng = np.random.default_rng(nu + nproj)
    dev = torch.device("cuda", 0)
    darks = torch.from_numpy(rng.normal(100, 3, (2, nv, nu)).astype(np.float32)).to(dev)
    flats = torch.from_numpy(rng.normal(20000, 100, (3, nv, nu)).astype(np.float32)).to(dev)
    counts = rng.integers(3000, 18000, (nproj, nv, nu)).astype(np.uint16)
    angles = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    weights = np.full(nproj, np.float32(1.0 / nproj))
    pipe = pipeline.FdkPipeline(_config(nu, nv, nproj), angles, weights, darks, flats)
    ref = pipe.run_device(torch.from_numpy(counts.view(np.int16)).to(dev).view(torch.uint16)).clone()
    host = torch.from_numpy(counts.view(np.int16)).view(torch.uint16).pin_memory()
    for _ in range(2):
        out = torch.full((nv, nu, nu), np.nan, dtype=torch.float32).pin_memory()
        pipe.run_host(host, out, dev, chunks=chunks, slabs=slabs)
        torch.cuda.synchronize()
        assert torch.equal(out, ref.cpu())
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    assert st.value == 0


def _parallel_modules(nu, nv, nproj, darks, flats, spot_ring):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter = (nu - 1) / 2.0
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    pi.nOBCount, pi.nDCCount = flats.shape[0], darks.shape[0]
    norm = M.FullLogNorm()
    norm.Configure(cfg, {"usenormregion": "false", "uselut": "false", "referenceaverage": "ImageAverage"})
    norm.SetReferenceImages(darks, flats)
    spot = ring = None
    if spot_ring:
        spot = M.MorphSpotCleanModule()
        spot.Configure(cfg, {"connectivity": "conn8", "cleanmethod": "morphcleanreplace",
                             "detectionmethod": "morphdetectboth", "threshold": "0.1 0.1", "sigma": "0.01 0.01",
                             "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false", "clampdata": "false",
                             "minlevel": "-0.1", "maxlevel": "12", "threading": "false"})
        ring = M.WaveletRingClean()
        ring.Configure(cfg, {"wname": "daub4", "sigma": "0.05", "decnum": "2", "parallel": "false",
                             "method": "verticalfft"})
    filt = M.ProjectionFilterSingle()
    filt.Configure(cfg, {"filtertype": "hanning", "cutoff": "0.5", "order": "1", "usebias": "true",
                         "biasweight": "0.1", "paddingdoubler": "2"})
    bp = M.MultiProjectionBPparallel()
    bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1", "precision": "fp32",
                       "referencecompat": "true"})
    bp.SetROI((0, 0, nu, nv))
    return norm, filt, bp, spot, ring


@pytest.mark.parametrize("nu,nv,nproj,chunks,blocks,spot_ring", [(64, 24, 30, 4, 3, True), (128, 16, 45, 8, 8, False),
                                                                    (96, 12, 21, 3, 5, True)])
def test_parallel_chain_host_equals_device(cuda, nu, nv, nproj, chunks, blocks, spot_ring):
    """Counts in by projection groups (FullLogNorm and MorphSpotClean per group), ring cleaning
    and filter on the block, backprojection by row blocks copied out while the next runs: the
    same volume as the one-shot device chain, bit for bit."""
    from imagingsuite_b200 import phantom

    dev = torch.device("cuda", 0)
    integ = phantom.parallel_integrals_torch(phantom.ellipsoids(1001), nproj, nu, nv, dev)
    counts, flats, darks = phantom.counts_torch(integ, 3e4, 2001, 4, 3)
    angles = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    weights = np.full(nproj, np.float32(np.pi / nproj))
    norm, filt, bp, spot, ring = _parallel_modules(nu, nv, nproj, darks, flats, spot_ring)
    chain = pipeline.ParallelChain(norm, filt, bp, angles, weights, spot=spot, ring=ring)
    ref = chain.run_device(counts).clone()
    host = counts.cpu().pin_memory()
    for _ in range(2):
        out = torch.full(ref.shape, np.nan, dtype=torch.float32).pin_memory()
        chain.run_host(host, out, dev, chunks=chunks, blocks=blocks)
        torch.cuda.synchronize()
        assert torch.equal(out, ref.cpu())
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    assert st.value == 0


@pytest.mark.parametrize("world", [2, 3])
def test_fdk_slabs_with_row_windows_equal_whole(cuda, world):
    """Each rank's share (distributed.cone_slab_plan): FullLogNorm and the ramp filter on the
    slab's detector-row window only, the slab's slices backprojected. The rows outside the
    window are poisoned with NaN, so a voxel reading outside its window would show. Every slab
    equals the same slices of the whole-volume reconstruction bit for bit."""
    nu, nv, nproj = 64, 96, 20
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", 0)
    darks = torch.from_numpy(rng.normal(100, 3, (2, nv, nu)).astype(np.float32)).to(dev)
    flats = torch.from_numpy(rng.normal(20000, 100, (3, nv, nu)).astype(np.float32)).to(dev)
    counts = rng.integers(3000, 18000, (nproj, nv, nu)).astype(np.uint16)
    angles = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    weights = np.full(nproj, np.float32(1.0 / nproj))
    pipe = pipeline.FdkPipeline(_config(nu, nv, nproj), angles, weights, darks, flats)
    whole = pipe.run_device(torch.from_numpy(counts.view(np.int16)).to(dev).view(torch.uint16)).cpu().numpy()
    plan = pipe.slab_plan(world)
    assert any(s.rows < nv for s in plan)
    for s in plan:
        rows = torch.from_numpy(np.ascontiguousarray(counts[:, s.row_start:s.row_stop]).view(np.int16)).to(dev)
        pipe.run_slab(rows.view(torch.uint16), s)
        pipe._slab_bufs[2].fill_(float("nan"))  # rows outside the next window stay NaN
        vol = pipe.run_slab(rows.view(torch.uint16), s).cpu().numpy()
        assert np.array_equal(vol[s.start:s.stop], whole[s.start:s.stop]), s
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    assert st.value == 0


def test_fdk_filter_rows_equals_whole_detector_rows(cuda):
    """mr_fdk_filter_rows on windows inside, at the top and at the bottom of the detector gives
    the whole-detector filter's rows; windows that miss the copied edge row are refused."""
    nu, nv, nproj = 48, 40, 3
    rng = np.random.default_rng(8)
    x = torch.from_numpy(rng.standard_normal((nproj, nv, nu)).astype(np.float32)).to(cuda)
    w = torch.from_numpy(rng.uniform(0.5, 1.5, nproj).astype(np.float32)).to(cuda)
    st = torch.cuda.current_stream().cuda_stream
    full = torch.empty_like(x)
    L.check(L.lib().mr_fdk_filter(x.data_ptr(), nu, nv, nproj, w.data_ptr(), 0.25, 0.5, L.MR_F32, full.data_ptr(), None,
                                  st))
    # even windows: the filter transforms two rows at a time, so the whole detector's row pairs
    # are kept (bit-identical rows)
    for r0, r1 in ((0, 10), (8, 30), (30, 40), (12, 14), (0, 40)):
        src = x[:, r0:r1].contiguous()
        out = torch.empty_like(src)
        L.check(L.lib().mr_fdk_filter_rows(src.data_ptr(), nu, r1 - r0, r0, nv, nproj, w.data_ptr(), 0.25, 0.5,
                                           L.MR_F32, out.data_ptr(), None, st))
        assert torch.equal(out, full[:, r0:r1]), (r0, r1)
    bad = torch.empty((nproj, 3, nu), device=cuda)
    for r0 in (1, 36):  # rows 1..3 need row 5; rows 36..38 need row 34
        assert L.lib().mr_fdk_filter_rows(bad.data_ptr(), nu, 3, r0, nv, nproj, w.data_ptr(), 0.25, 0.5, L.MR_F32,
                                          bad.data_ptr(), None, st) == L.MR_ERR_ARGUMENT
