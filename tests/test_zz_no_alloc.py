"""mr_quantize_noalloc: the allocation-free form of mr_quantize (gpu).

Some callers cannot allocate device memory (a framework that owns every allocation, a
plugin host that forbids cudaMalloc); mr_quantize_noalloc keeps its scratch in a static
device array instead. This file is collected last so that a failure here comes after every
other test has run. It passes alone in a fresh process and after the other tests: the first
call on the device looks up the array's address, later calls reuse it, and every call
clears the part of the array it uses.
"""
import ctypes

import numpy as np
import pytest
import torch

from imagingsuite_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _run(fn, x, per, nproj, dtype):
    out = torch.empty(x.numel(), dtype=torch.uint16, device=x.device)
    scale = torch.empty(nproj, dtype=torch.float32, device=x.device)
    L.check(fn(x.data_ptr(), per, nproj, dtype, out.data_ptr(), scale.data_ptr(),
               torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out.cpu().numpy(), scale.cpu().numpy()


@pytest.mark.parametrize("dtype", [L.MR_BF16, L.MR_F16])
def test_noalloc_matches_quantize_twice(cuda, dtype):
    lib = L.lib()
    rng = np.random.default_rng(99)
    # two calls in a row; the second has smaller magnitudes and fewer projections, so any
    # maxima left over from the first call would show up in its scales
    for nproj, per, amp in ((37, 4096, 50.0), (11, 3000, 0.01)):
        x = torch.from_numpy((rng.standard_normal((nproj, per)) * amp).astype(np.float32)).to(cuda)
        q_ref, s_ref = _run(lib.mr_quantize, x, per, nproj, dtype)
        q_new, s_new = _run(lib.mr_quantize_noalloc, x, per, nproj, dtype)
        # same kernels, same inputs: identical bits (the tolerance of the other quantize tests is exact equality)
        assert np.array_equal(s_new, s_ref)
        assert np.array_equal(q_new, q_ref)
    status = ctypes.c_int(-1)
    L.check(lib.mr_device_status(ctypes.byref(status)))
    assert status.value == 0


def test_noalloc_at_its_maximum(cuda):
    """Exactly 65536 projections (the array's size, one more than a grid's y extent) work and
    equal mr_quantize run on the same projections in two calls (mr_quantize takes at most
    65535 per call; every projection is scaled on its own)."""
    lib = L.lib()
    nproj, per = 65536, 4
    rng = np.random.default_rng(7)
    x = torch.from_numpy((rng.standard_normal((nproj, per)) * np.exp(rng.uniform(-20, 20, (nproj, 1))))
                         .astype(np.float32)).to(cuda)
    q_new, s_new = _run(lib.mr_quantize_noalloc, x, per, nproj, L.MR_F16)
    q_a, s_a = _run(lib.mr_quantize, x[:65535].contiguous(), per, 65535, L.MR_F16)
    q_b, s_b = _run(lib.mr_quantize, x[65535:].contiguous(), per, 1, L.MR_F16)
    assert np.array_equal(s_new, np.concatenate([s_a, s_b]))
    assert np.array_equal(q_new, np.concatenate([q_a, q_b]))


def test_noalloc_rejects_oversize(cuda):
    lib = L.lib()
    x = torch.zeros(4, device=cuda)
    out = torch.empty(4, dtype=torch.uint16, device=cuda)
    st = lib.mr_quantize_noalloc(x.data_ptr(), 1, 65537, L.MR_BF16, out.data_ptr(), x.data_ptr(), None)
    assert st == L.MR_ERR_ARGUMENT
    assert b"65536" in lib.mr_last_error()
