"""GetSlice with and without the matrix ROI, and TransferMatrix, against the reference's own
BackProjectorModuleBase::GetSlice (compiled from source): on the CPU with host tensors, and on
the GPU with the modules' device volumes."""
import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import modules as M

CASES = [None, (0, 0, 10, 6), (3, 2, 9, 11), (5, 7, 5, 7)]


def _module(zxy: bool, vol: torch.Tensor, roi):
    bp = M.MultiProjectionBPparallel() if zxy else M.FDKbp_single()
    bp.mConfig.MatrixInfo.bUseROI = roi is not None
    if roi is not None:
        bp.mConfig.MatrixInfo.roi = roi
    bp.volume = vol
    return bp


def _volume(zxy, seed=0):
    rng = np.random.default_rng(seed)
    # ZXY: (ny, nx, nz); XYZ: (nz, ny, nx); nx = 13, ny = 12, nz = 5
    shape = (12, 13, 5) if zxy else (5, 12, 13)
    return rng.standard_normal(shape).astype(np.float32)


@pytest.mark.parametrize("zxy", [True, False])
@pytest.mark.parametrize("roi", CASES)
def test_getslice_matches_reference(ref_lib, zxy, roi):
    vol = _volume(zxy)
    bp = _module(zxy, torch.from_numpy(vol), roi)
    for idx in (0, 2, 4):
        got = bp.GetSlice(idx).numpy()
        assert np.array_equal(got, O.ref_getslice(vol, zxy, idx, roi))


@pytest.mark.parametrize("zxy", [True, False])
def test_getslice_errors(zxy):
    vol = torch.from_numpy(_volume(zxy))
    with pytest.raises(M.ReconException, match="Slice index greater than matrix size"):
        _module(zxy, vol, None).GetSlice(5)
    with pytest.raises(M.ReconException, match="outside"):
        _module(zxy, vol, (4, 0, 13, 3)).GetSlice(0)


def test_transfer_matrix_places_block():
    vol = _volume(True, 3)
    bp = _module(True, torch.from_numpy(vol), (3, 2, 9, 11))
    engine = torch.zeros((9, 10, 7))
    M.TransferMatrix(bp, engine, (0, 4, 0, 8), first_slice=2)  # slices 4..7 -> planes 2..5
    for i in range(4):
        assert np.array_equal(engine[2 + i].numpy(), vol[2:12, 3:10, i])
    assert not engine[0:2].any() and not engine[6:].any()


@pytest.mark.gpu
@pytest.mark.parametrize("zxy", [True, False])
@pytest.mark.parametrize("roi", CASES)
def test_getslice_device(cuda, zxy, roi):
    vol = _volume(zxy, 1)
    bp = _module(zxy, torch.from_numpy(vol).to(cuda), roi)
    got = bp.GetSlice(3)
    assert got.is_cuda
    assert np.array_equal(got.cpu().numpy(), O.ref_getslice(vol, zxy, 3, roi))


@pytest.mark.gpu
@pytest.mark.parametrize("cone", [False, True])
def test_matrix_roi_mask_and_slices_match_reference(cuda, ref_lib, cone):
    """With MatrixInfo.bUseROI the modules restrict the circle mask as BuildCircleMask does
    and GetSlice crops to the ROI: volume and slices against the reference modules."""
    rng = np.random.default_rng(11)
    nproj, nv, nu = 24, 16, 64
    proj = (rng.standard_normal((nproj, nv, nu)) * 0.2 + 1.0).astype(np.float32)
    ang = (np.arange(nproj) * (360.0 if cone else 180.0) / nproj).astype(np.float32)
    w = np.full(nproj, np.float32(1.0 / nproj))
    roi = (6, 4, 40, 50)
    c = O.RefBpConfig()
    c.center = (nu - 1) / 2.0 + 0.27
    c.cone = int(cone)
    c.sod, c.sdd = 300.0, 600.0
    c.ppoint[0], c.ppoint[1] = (nu - 1) / 2.0 + 0.13, (nv - 1) / 2.0 - 0.21
    c.resolution[0] = c.resolution[1] = 0.2
    c.voxelsize[0] = c.voxelsize[1] = c.voxelsize[2] = 0.1
    c.use_matrix_roi = 1
    for i, v in enumerate(roi):
        c.matrix_roi[i] = v
    params = {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"}
    name = "FDKbp_single" if cone else "MultiProjBPparallel"
    ev, es = O.ref_bp_module(proj, ang, w, name, c, (0, 0, nu, nv), params)
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter, pi.fSOD, pi.fSDD = c.center, 300.0, 600.0
    pi.fpPoint, pi.fResolution = (c.ppoint[0], c.ppoint[1]), (0.2, 0.2)
    pi.roi = (0, 0, nu, nv)
    pi.nDims = (nu, nv, nproj)
    cfg.MatrixInfo.fVoxelSize = (0.1, 0.1, 0.1)
    cfg.MatrixInfo.bUseROI, cfg.MatrixInfo.roi = True, roi
    bp = M.FDKbp_single() if cone else M.MultiProjectionBPparallel()
    bp.Configure(cfg, params)
    bp.SetROI((0, 0, nu, nv))
    text = lambda a: " ".join("%.9g" % v for v in a)
    bp.Process(torch.from_numpy(proj).to(cuda), {"angles": text(ang), "weights": text(w)})
    gv = bp.GetVolume().cpu().numpy().reshape(-1)
    gs = np.stack([bp.GetSlice(i).cpu().numpy() for i in range(bp.GetNSlices())])
    assert gs.shape == es.shape
    if cone:  # FP32 FFT ramp filter against the reference build's FP64 FFT
        rel = lambda a, b: np.sqrt(np.mean((a.astype(np.float64) - b) ** 2) / np.mean(b.astype(np.float64) ** 2))
        assert rel(gv, ev) < 1e-5 and rel(gs, es) < 1e-5
        assert np.array_equal(gv == 0, ev == 0)  # the same masked voxels
    else:
        assert np.array_equal(gv, ev) and np.array_equal(gs, es)
