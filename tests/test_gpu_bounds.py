"""The bounds-checked build (gpu): libmrcuda_checked.so (-DMR_BOUNDS_CHECK) runs the main kernels
on small shapes with an index check at each gather site; no check fails, and every output equals
the product library's bit for bit (the checks only read), the matched forward projection to
float summation (its shared-memory atomics add in a varying order)."""
import ctypes

import numpy as np
import pytest
import torch

from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import joseph as J
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu


def _text(a):
    return " ".join("%.9g" % v for v in a)


def _workloads(cuda):
    """Small cases through the modules (whichever library L.lib() returns); their outputs."""
    rng = np.random.default_rng(31)
    out = {}
    # FDK: staged and direct
    nproj, nv, nu = 24, 40, 64
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = 300.0, 600.0
    pi.fpPoint = ((nu - 1) / 2.0 + 0.13, (nv - 1) / 2.0 - 0.21)
    pi.fCenter = (nu - 1) / 2.0 + 0.07
    pi.fResolution = (0.2, 0.2)
    pi.nDims = (nu, nv, nproj)
    cfg.MatrixInfo.fVoxelSize = (0.1, 0.1, 0.1)
    proj = torch.from_numpy((rng.standard_normal((nproj, nv, nu)) * 0.1 + 1.0).astype(np.float32)).to(cuda)
    ang = (np.arange(nproj) * 15.0).astype(np.float32)
    w = np.full(nproj, np.float32(1.0 / nproj))
    for staged in (True, False):
        fdk = M.FDKbp_single()
        fdk.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
        fdk.staging = staged
        fdk.SetROI((0, 0, nu, nv))
        fdk.Process(proj.clone(), {"angles": _text(ang), "weights": _text(w)})
        out[f"fdk_{staged}"] = fdk.GetVolume().cpu().numpy()
    # parallel beam: staged, direct, serial with tilt, nearest neighbour
    nproj, nv, nu = 45, 12, 96
    p = torch.from_numpy(rng.standard_normal((nproj, nv, nu)).astype(np.float32)).to(cuda)
    ang = (np.arange(nproj) * 4.0).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    for name, cls, tilt, staged in (("par_staged", M.MultiProjectionBPparallel, False, True),
                                    ("par_direct", M.MultiProjectionBPparallel, False, False),
                                    ("serial_tilt", M.MultiProjectionBP, True, True),
                                    ("nearest", M.NearestNeighborBP, False, True)):
        c = M.ReconConfig()
        c.ProjectionInfo.fCenter = (nu - 1) / 2.0 + 0.3
        c.ProjectionInfo.roi = (0, 0, nu, nv)
        c.ProjectionInfo.nDims = (nu, nv, nproj)
        c.ProjectionInfo.bCorrectTilt, c.ProjectionInfo.fTiltAngle = tilt, 0.6
        bp = cls()
        bp.Configure(c, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
        bp.staging = staged
        bp.SetROI((0, 0, nu, nv))
        bp.Process(p.clone(), {"angles": _text(ang), "weights": _text(w)})
        out[name] = bp.GetVolume().cpu().numpy()
    # the matched pair (shared-memory forward, tilted adjoint)
    op = J.MatchedOperator(64, 8, (np.arange(30) * 6.0).astype(np.float32))
    x = torch.from_numpy(rng.standard_normal((64, 64, 8)).astype(np.float32)).to(cuda)
    out["mbp_forward"] = op.forward(x, 32.3, 0.4).cpu().numpy()
    y = torch.from_numpy(rng.standard_normal((30, 8, 64)).astype(np.float32)).to(cuda)
    out["mbp_adjoint"] = op.adjoint(y, 32.3, 0.4).cpu().numpy()
    # ring cleaning and MorphSpotClean on a small stack
    nproj, nv, nu = 64, 16, 128
    img = torch.from_numpy((rng.standard_normal((nproj, nv, nu)) * 0.05 + 1.0).astype(np.float32)).to(cuda)
    img[5, 3, 40] = 4.0
    img[9, 7, 70] = -2.0
    c = M.ReconConfig()
    c.ProjectionInfo.roi = (0, 0, nu, nv)
    ring = M.WaveletRingClean()
    ring.Configure(c, {"wname": "daub15", "sigma": "0.05", "decnum": "2", "parallel": "false",
                       "method": "verticalfft"})
    r = img.clone()
    ring.Process(r, {})
    out["ringclean"] = r.cpu().numpy()
    spot = M.MorphSpotCleanModule()
    spot.Configure(c, {"connectivity": "conn8", "cleanmethod": "morphcleanreplace",
                       "detectionmethod": "morphdetectboth", "threshold": "0.1 0.1", "sigma": "0.01 0.01",
                       "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false", "clampdata": "false",
                       "minlevel": "-0.1", "maxlevel": "12", "threading": "false"})
    sp = img.clone()
    spot.Process(sp, {})
    out["spotclean"] = sp.cpu().numpy()
    torch.cuda.synchronize()
    return out


def test_checked_build_finds_no_bad_index_and_matches(cuda, monkeypatch):
    checked = L.load(L.CHECKED_LIB_PATH)
    product = _workloads(cuda)
    monkeypatch.setattr(L, "_lib", checked)
    word = ctypes.c_ulonglong(1)
    L.check(checked.mr_bounds_status(ctypes.byref(word)))  # clear
    got = _workloads(cuda)
    L.check(checked.mr_bounds_status(ctypes.byref(word)))
    assert word.value == 0, f"bounds check failed at site {word.value >> 40}, index {word.value & ((1 << 40) - 1)}"
    st = ctypes.c_int(-1)
    L.check(checked.mr_device_status(ctypes.byref(st)))
    assert st.value == 0
    for k, v in product.items():
        if k == "mbp_forward":  # shared-memory atomics: the order of the additions varies
            assert np.sqrt(np.sum((got[k] - v) ** 2) / np.sum(v ** 2)) < 1e-6, k
        else:
            assert np.array_equal(got[k], v), k


def test_product_build_reports_no_bounds_word(cuda):
    word = ctypes.c_ulonglong(7)
    L.check(L.lib().mr_bounds_status(ctypes.byref(word)))
    assert word.value == 0
