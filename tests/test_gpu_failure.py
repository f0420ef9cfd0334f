"""Failure detection on the device without a fault (gpu).

* Bounded waits: with the per-batch wait limit at 0 tries (mr_set_wait_limit) every TMA-staged
  backprojection block gives up at its first batch, sets the device error word, waits (with
  the default limit) for the copies it has in flight and returns; the host reads the word
  (mr_device_status, TransferMatrix, the pipelines' check_device), the context stays usable,
  and with the default limit restored the same call is bit-exact again.
* Allocation failures: the allocation-failure hook makes a module's scratch allocation fail;
  the module raises a ReconException carrying MR_ERR_ALLOCATION and works on the next call.
* NaN input: counted (mr_data_validator, ReconEngine::validateImage) and logged, not a crash.
"""
import ctypes
import logging

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M
from imagingsuite_b200 import phantom, pipeline

pytestmark = pytest.mark.gpu


def _word():
    st = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(st)))
    return st.value


def _text(a):
    return " ".join("%.9g" % v for v in a)


@pytest.fixture
def zero_wait_limit():
    assert _word() == 0
    L.check(L.lib().mr_set_wait_limit(0))
    try:
        yield
    finally:
        L.check(L.lib().mr_set_wait_limit(-1))


def _fdk_module(nu, nv):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint = ((nu - 1) / 2.0, (nv - 1) / 2.0)
    pi.fCenter = (nu - 1) / 2.0 + 0.3
    pi.fResolution = (0.2, 0.2)
    pi.nDims = (nu, nv, 0)
    cfg.MatrixInfo.fVoxelSize = (0.1, 0.1, 0.1)
    mod = M.FDKbp_single()
    mod.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    mod.SetROI((0, 0, nu, nv))
    g = O.fdk_geom(pi.fSOD, pi.fSDD, pi.fpPoint, pi.fCenter, pi.fResolution, cfg.MatrixInfo.fVoxelSize)
    return mod, g


def _fdk_staged(cuda, mod, filt, ang):
    nproj, nv, nu = filt.shape
    xip, yip, zip_, *_ , uni = mod.partials(ang)
    assert uni
    bw, bh = ctypes.c_int(0), ctypes.c_int(0)
    L.check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                               zip_.ctypes.data_as(L.P_float), nu, nv, nproj, L.MR_F32, ctypes.byref(bw),
                               ctypes.byref(bh)))
    vol = torch.full((nv, nu, nu), 7.0, device=cuda)
    X, Y, Z = (torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in (xip, yip, zip_))
    src = torch.from_numpy(filt).to(cuda)
    L.check(L.lib().mr_fdk_backproject(src.data_ptr(), L.MR_F32, None, nu, nv, nproj, X.data_ptr(), Y.data_ptr(),
                                       Z.data_ptr(), uni, mod._mask.data_ptr(), bw.value, bh.value, 0,
                                       vol.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return vol


def test_fdk_wait_expiry_reported_and_recovered(cuda, zero_wait_limit):
    rng = np.random.default_rng(21)
    nproj, nv, nu = 24, 40, 64
    mod, g = _fdk_module(nu, nv)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 15.0).astype(np.float32)
    _fdk_staged(cuda, mod, filt, ang)
    assert _word() == 1
    assert _word() == 0  # reading clears it
    L.check(L.lib().mr_set_wait_limit(-1))
    got = _fdk_staged(cuda, mod, filt, ang).cpu().numpy()
    assert _word() == 0
    assert np.array_equal(got, O.fdk_bp(filt, ang, g))


def test_fdk_wait_expiry_single_batch(cuda, zero_wait_limit):
    """One batch of projections: only the expired batch has a copy in flight to wait for."""
    rng = np.random.default_rng(22)
    nproj, nv, nu = 3, 32, 64
    mod, _ = _fdk_module(nu, nv)
    filt = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    _fdk_staged(cuda, mod, filt, (np.arange(nproj) * 40.0).astype(np.float32))
    assert _word() == 1


def _bp_module(nu, nv):
    cfg = M.ReconConfig()
    cfg.ProjectionInfo.fCenter = (nu - 1) / 2.0 + 0.2
    cfg.ProjectionInfo.roi = (0, 0, nu, nv)
    bp = M.MultiProjectionBPparallel()
    bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    bp.SetROI((0, 0, nu, nv))
    return bp


def test_parallel_wait_expiry_raises_at_transfer(cuda, zero_wait_limit):
    """The staged parallel backprojector under the module: TransferMatrix (the engine's read-back
    of the block) raises a ReconException with MR_ERR_DEVICE; the next block is exact."""
    rng = np.random.default_rng(23)
    nproj, nv, nu = 90, 32, 128
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 2.0).astype(np.float32)
    w = np.ones(nproj, np.float32)
    bp = _bp_module(nu, nv)
    bp.Process(torch.from_numpy(proj).to(cuda), {"angles": _text(ang), "weights": _text(w)})
    out = torch.empty((nv, nu, nu), device=cuda)
    with pytest.raises(M.ReconException) as e:
        M.TransferMatrix(bp, out, (0, 0, nu, nv))
    assert isinstance(e.value, L.MrError) and e.value.status == L.MR_ERR_DEVICE
    L.check(L.lib().mr_set_wait_limit(-1))
    bp = _bp_module(nu, nv)
    bp.Process(torch.from_numpy(proj).to(cuda), {"angles": _text(ang), "weights": _text(w)})
    M.TransferMatrix(bp, out, (0, 0, nu, nv))
    exp = O.bp_parallel(proj, ang, w, (nu - 1) / 2.0 + 0.2, buffersize=16)
    assert np.array_equal(bp.GetVolume().cpu().numpy(), exp)


def _counts(cuda, nu, nv, nproj, seed=1):
    integ = phantom.parallel_integrals_torch(phantom.ellipsoids(seed), nproj, nu, nv, cuda)
    return phantom.counts_torch(integ, 3e4, 100 + seed, 5, 5)


def _cfg(nu, nv, nproj):
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter = (nu - 1) / 2.0
    pi.roi = pi.projection_roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    pi.nOBCount, pi.nDCCount = 5, 5
    return cfg


_SPOT = {"connectivity": "conn8", "cleanmethod": "morphcleanreplace", "detectionmethod": "morphdetectboth",
         "threshold": "0.1 0.1", "sigma": "0.01 0.01", "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false",
         "clampdata": "false", "minlevel": "-0.1", "maxlevel": "12", "threading": "false"}
_RING = {"wname": "daub15", "sigma": "0.05", "decnum": "2", "parallel": "false", "method": "verticalfft"}


@pytest.mark.parametrize("module", ["MorphSpotCleanModule", "WaveletRingClean", "FullLogNormLUT"])
def test_allocation_failure_hook(cuda, module):
    nu, nv, nproj = 128, 16, 64
    counts, flats, darks = _counts(cuda, nu, nv, nproj)
    cfg = _cfg(nu, nv, nproj)
    norm = M.FullLogNorm()
    norm.Configure(cfg, {"usenormregion": "false", "uselut": "true" if module == "FullLogNormLUT" else "false",
                         "referenceaverage": "ImageAverage"})
    norm.SetReferenceImages(darks, flats)
    if module == "FullLogNormLUT":
        run = lambda: norm.Process(counts, {}).clone()  # noqa: E731
    else:
        base = norm.ProcessCore(counts, {}).clone()
        mod = M.MorphSpotCleanModule() if module == "MorphSpotCleanModule" else M.WaveletRingClean()
        mod.Configure(cfg, _SPOT if module == "MorphSpotCleanModule" else _RING)

        def run():
            p = base.clone()
            mod.Process(p, {})
            return p
    exp = run().cpu().numpy()
    L.check(L.lib().mr_debug_fail_allocation(0))
    try:
        with pytest.raises(M.ReconException) as e:
            run()
            torch.cuda.synchronize()
    finally:
        L.check(L.lib().mr_debug_fail_allocation(-1))
    assert e.value.status == L.MR_ERR_ALLOCATION
    assert "allocation-failure hook" in str(e.value)
    assert np.array_equal(run().cpu().numpy(), exp)
    assert _word() == 0


def test_allocation_failure_second_table_of_fdk_filter(cuda):
    """mr_fdk_filter allocates twiddles, then the response: the second failing frees the first
    and the call reports MR_ERR_ALLOCATION; nothing was launched into the output."""
    nproj, nv, nu = 4, 16, 64
    x = torch.randn((nproj, nv, nu), device=cuda) + 1.0
    w = torch.ones(nproj, device=cuda)
    out = torch.full((nproj, nv, nu), 3.0, device=cuda)
    L.check(L.lib().mr_debug_fail_allocation(1))
    try:
        st = L.lib().mr_fdk_filter(x.data_ptr(), nu, nv, nproj, w.data_ptr(), 0.25, 0.5, L.MR_F32, out.data_ptr(), None,
                                   torch.cuda.current_stream().cuda_stream)
    finally:
        L.check(L.lib().mr_debug_fail_allocation(-1))
    assert st == L.MR_ERR_ALLOCATION
    assert b"mr_fdk_filter: response" in L.lib().mr_last_error()
    assert bool((out == 3.0).all())
    L.check(L.lib().mr_fdk_filter(x.data_ptr(), nu, nv, nproj, w.data_ptr(), 0.25, 0.5, L.MR_F32, out.data_ptr(),
                                  None, torch.cuda.current_stream().cuda_stream))
    assert not bool((out == 3.0).any())


@pytest.mark.parametrize("n,offset", [(0, 0), (1, 0), (7, 1), (4096, 0), (1 << 20, 3), (3 * (1 << 20) + 5, 2)])
def test_data_validator_counts(cuda, n, offset):
    rng = np.random.default_rng(n + offset)
    a = rng.standard_normal(n + offset).astype(np.float32)
    if n:
        k = max(1, n // 97)
        a[offset + rng.integers(0, n, k)] = np.nan
        a[offset + rng.integers(0, n, k)] = np.inf
        a[offset + rng.integers(0, n, k)] = -np.inf
        a[offset + rng.integers(0, n, k)] = np.float32(3e38)  # large but finite
        nanbits = np.array([0x7fc00001, 0xffc00000, 0x7f800001], np.uint32).view(np.float32)
        a[offset:offset + 3 if n >= 3 else offset + n] = nanbits[: min(3, n)]
    t = torch.from_numpy(a).to(cuda)
    counts = torch.full((2,), 99, dtype=torch.int64, device=cuda)
    L.check(L.lib().mr_data_validator(t.data_ptr() + 4 * offset, n, counts.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream))
    v = a[offset:]
    assert counts.cpu().tolist() == [int(np.isnan(v).sum()), int(np.isinf(v).sum())]


def test_chain_counts_nan_input(cuda, caplog):
    """NaN counts through the parallel chain with validation on: every module's output is
    counted (the engine's warning names the module), the block completes."""
    nu, nv, nproj = 128, 16, 60
    counts, flats, darks = _counts(cuda, nu, nv, nproj, 7)
    fcounts = counts.float()
    fcounts[3, 5, 7] = float("nan")
    fcounts[10, 0, 0:4] = float("nan")
    cfg = _cfg(nu, nv, nproj)
    cfg.System.bValidateData = True
    norm = M.FullLogNorm()
    norm.Configure(cfg, {"usenormregion": "false", "uselut": "false", "referenceaverage": "ImageAverage"})
    norm.SetReferenceImages(darks, flats)
    filt = M.ProjectionFilterSingle()
    filt.Configure(cfg, {"filtertype": "hanning", "cutoff": "0.5", "order": "1", "usebias": "true",
                         "biasweight": "0.1", "paddingdoubler": "2"})
    bp = _bp_module(nu, nv)
    ang = (np.arange(nproj) * 3.0).astype(np.float32)
    chain = pipeline.ParallelChain(norm, filt, bp, ang, np.full(nproj, np.float32(np.pi / nproj)),
                                   validate=cfg.System.bValidateData)
    expected_norm = int(torch.isnan(norm.ProcessCore(fcounts, {}).clone()).sum())
    assert expected_norm == 5
    with caplog.at_level(logging.WARNING, logger="imagingsuite_b200"):
        vol = chain.run_device(fcounts)
    torch.cuda.synchronize()
    msgs = [r.getMessage() for r in caplog.records]
    assert "Encountered 0 infs and 5 NaNs in FullLogNorm" in msgs
    assert any(m.endswith("in ProjectionFilterSingle") for m in msgs)  # the filter spreads NaN along rows
    assert vol is not None and bool(torch.isnan(vol).any())
    chain.check_device()
