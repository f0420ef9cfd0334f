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
