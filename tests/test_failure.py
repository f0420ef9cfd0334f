"""Failure detection and tracing on the host (no GPU): the library's hooks load and answer,
the modules trace their calls and turn library failures into ReconException, and the chain
cancels between modules when the progress callback asks for it (InteractionBase::SetProgress
returning true, ReconEngine.cpp:1283-1290)."""
import inspect

import numpy as np
import pytest
import torch

from imagingsuite_b200 import _lib as L
from imagingsuite_b200 import modules as M
from imagingsuite_b200 import pipeline


def test_hooks_answer_without_a_device():
    lib = L.lib()
    assert lib.mr_trace_push(b"test range") == L.MR_OK
    assert lib.mr_trace_push(b"nested") == L.MR_OK
    assert lib.mr_trace_pop() == L.MR_OK
    assert lib.mr_trace_pop() == L.MR_OK
    assert lib.mr_trace_push(None) == L.MR_ERR_ARGUMENT
    assert lib.mr_debug_fail_allocation(3) == L.MR_OK
    assert lib.mr_debug_fail_allocation(-1) == L.MR_OK
    assert lib.mr_set_wait_limit(10) == L.MR_OK
    assert lib.mr_set_wait_limit(-1) == L.MR_OK


def test_data_validator_rejects_null_counts():
    assert L.lib().mr_data_validator(None, 0, None, None) == L.MR_ERR_ARGUMENT
    assert L.lib().mr_data_validator(None, 5, 8, None) == L.MR_ERR_ARGUMENT


MODULES = [M.FullLogNorm, M.MorphSpotCleanModule, M.WaveletRingClean, M.BasicRingClean, M.MedianMixRingClean,
           M.SpotClean2, M.GammaSpotClean, M.ProjectionFilterSingle, M.MultiProjectionBPparallel,
           M.MultiProjectionBP, M.NearestNeighborBP, M.FDKbp_single]


@pytest.mark.parametrize("cls", MODULES, ids=lambda c: c.__name__)
def test_module_calls_are_traced(cls):
    for name in ("Configure", "Process"):
        fn = getattr(cls, name)
        assert hasattr(fn, "__wrapped__"), f"{cls.__name__}.{name}"
        assert inspect.signature(fn) == inspect.signature(fn.__wrapped__)


def test_library_failure_is_a_recon_exception():
    e = M.LibraryFailure("FullLogNorm.Process", L.MrError(L.MR_ERR_ALLOCATION, "scratch: 8 bytes"))
    assert isinstance(e, M.ReconException) and isinstance(e, L.MrError)
    assert e.status == L.MR_ERR_ALLOCATION
    assert "FullLogNorm.Process" in str(e) and "scratch" in str(e)


class _Recorder:
    """Stand-ins for the configured modules: record the calls, no device work."""

    def __init__(self, log, name):
        self.log, self.name = log, name

    def ProcessCore(self, img, coeff, weights=None):
        self.log.append(self.name)
        return img

    def Process(self, proj, params, prefiltered_weights=False):
        self.log.append(self.name)
        return 0

    def GetVolume(self):
        return "volume"


class _Volume:
    def zero_(self):
        pass


@pytest.mark.parametrize("cancel_at", [None, 0, 2, 4])
def test_chain_cancels_between_modules(cancel_at):
    log = []
    norm, spot, ring, filt, bp = (_Recorder(log, n) for n in ("norm", "spot", "ring", "filter", "bp"))
    bp.volume = _Volume()
    chain = pipeline.ParallelChain(norm, filt, bp, np.zeros(4, np.float32), np.ones(4, np.float32), spot=spot,
                                   ring=ring)
    asked = []

    def progress(fraction, message):
        asked.append((fraction, message))
        return len(asked) - 1 == cancel_at

    out = chain.run_device(torch.zeros(1), progress=progress)
    order = ["norm", "spot", "ring", "filter", "bp"]
    if cancel_at is None:
        assert out == "volume" and log == order
    else:
        assert out is None and log == order[:cancel_at]
    assert [m for _, m in asked][:3] == ["Processing: FullLogNorm", "Processing: MorphSpotClean",
                                         "Processing: WaveletRingClean"][:len(asked)]
    assert all(0.0 <= f < 1.0 for f, _ in asked)
