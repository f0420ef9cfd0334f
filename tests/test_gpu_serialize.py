"""Slice serialisation on the GPU (gpu): mr_slices_u16 against the oracle's restatement of
ExtractSlice + ImageCaster<unsigned short, float> (pinned against the reference on the CPU),
bit for bit, for both volume layouts, ROIs, partial slice ranges and the edge values."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M

pytestmark = pytest.mark.gpu


def _volume(rng, shape):
    v = (rng.standard_normal(shape) * 0.02).astype(np.float32)
    flat = v.reshape(-1)
    flat[:4] = [np.inf, -np.inf, np.nan, 0.0]
    return v


@pytest.mark.parametrize("shape", [(40, 33, 70), (7, 64, 129), (64, 96, 96)])
@pytest.mark.parametrize("alignment", ["MatrixXYZ", "MatrixZXY"])
@pytest.mark.parametrize("roi", [None, (3, 2, 30, 5)])
def test_slices_match_oracle(cuda, shape, alignment, roi):
    rng = np.random.default_rng(sum(shape))
    vol = _volume(rng, shape)
    plane = 1 if alignment == "MatrixXYZ" else 4
    nslices = shape[0] if alignment == "MatrixXYZ" else shape[2]
    first, count = 2, nslices - 3
    got = M.slices_u16(torch.from_numpy(vol).cuda(), alignment, (-0.03, 0.05), first, count, roi).cpu().numpy()
    exp = O.slices_u16(vol, plane, first, count, -0.03, 0.05, roi)
    assert got.shape == exp.shape
    assert np.array_equal(got, exp)


def test_whole_volume_and_errors(cuda):
    rng = np.random.default_rng(5)
    vol = _volume(rng, (16, 48, 48))
    t = torch.from_numpy(vol).cuda()
    got = M.slices_u16(t, "MatrixXYZ", (-0.05, 0.05)).cpu().numpy()
    assert np.array_equal(got, O.slices_u16(vol, 1, 0, 16, -0.05, 0.05))
    out = torch.empty((1, 48, 48), dtype=torch.uint16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert L.lib().mr_slices_u16(t.data_ptr(), 1, 48, 48, 16, 10, 7, None, -1.0, 1.0, out.data_ptr(), st) == \
        L.MR_ERR_ARGUMENT
    assert L.lib().mr_slices_u16(t.data_ptr(), 1, 48, 48, 16, 0, 1, None, 1.0, 1.0, out.data_ptr(), st) == \
        L.MR_ERR_ARGUMENT
    assert L.lib().mr_slices_u16(t.data_ptr(), 2, 48, 48, 16, 0, 1, None, -1.0, 1.0, out.data_ptr(), st) == \
        L.MR_ERR_ARGUMENT
    status = ctypes.c_int(-1)
    L.check(L.lib().mr_device_status(ctypes.byref(status)))
    assert status.value == 0
