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
