"""Device-resident reconstruction chains (the block loop of ReconEngine::Process3D,
frameworks/tomography/Framework/ReconFramework/src/ReconEngine.cpp:1314-1714, for one block).

``FdkPipeline``: FullLogNorm -> FDKbp_single (ramp filter + cone-beam backprojection),
``ParallelPipeline``: FullLogNorm -> ProjectionFilterSingle (+ fused projection weights) ->
MultiProjectionBPparallel. Projections stay in HBM between modules; ``run_host`` is the
end-to-end form that takes uint16 counts in host memory and returns the volume in host
memory (one H2D and one D2H copy per block).
"""
from __future__ import annotations

import numpy as np
import torch

from . import modules as M


def _text(a) -> str:
    return " ".join("%.9g" % v for v in np.asarray(a, np.float32))


class FdkPipeline:
    def __init__(self, config: M.ReconConfig, angles, weights, darks: torch.Tensor, flats: torch.Tensor,
                 precision: str = "fp32", norm_params: dict | None = None):
        self.config = config
        self.angles = np.asarray(angles, np.float32)
        self.weights = np.asarray(weights, np.float32)
        self.norm = M.FullLogNorm()
        self.norm.Configure(config, norm_params or {"usenormregion": "false", "uselut": "false",
                                                    "referenceaverage": "ImageAverage"})
        self.norm.SetReferenceImages(darks, flats)
        self.fdk = M.FDKbp_single()
        self.fdk.Configure(config, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1",
                                    "precision": precision})
        nu, nv = config.ProjectionInfo.roi[2], config.ProjectionInfo.roi[3]
        self.nu, self.nv = nu, nv
        self.fdk.SetROI((0, 0, nu, nv))
        self._params = {"angles": _text(self.angles), "weights": _text(self.weights)}
        self._norm_buf = None

    def run_device(self, counts: torch.Tensor) -> torch.Tensor:
        """counts: uint16 (nproj, nv, nu) on the device. Returns the volume (nv, nu, nu)."""
        if self._norm_buf is None or self._norm_buf.shape != counts.shape:
            self._norm_buf = torch.empty(counts.shape, dtype=torch.float32, device=counts.device)
        self.fdk._first = True  # the first batch overwrites the whole volume
        proj = self.norm.ProcessCore(counts, {}) if counts.dtype == torch.float32 else self._lognorm_into(counts)
        self.fdk.Process(proj, self._params)
        return self.fdk.GetVolume()

    def _lognorm_into(self, counts):
        from . import _lib as L

        nproj, nv, nu = counts.shape
        dl = torch.zeros(1, device=counts.device)
        L.check(L.lib().mr_lognorm_apply(counts.data_ptr(), L.MR_U16, nv * nu, nproj, self.norm.mDark.data_ptr(),
                                         self.norm.mFlatField.data_ptr(), dl.data_ptr(), 1,
                                         int(self.norm.nDCCount > 0), int(self.norm.nOBCount > 0),
                                         self._norm_buf.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return self._norm_buf

    def run_host(self, counts_host: torch.Tensor, out_host: torch.Tensor, device) -> torch.Tensor:
        """counts_host: pinned uint16 (nproj, nv, nu); out_host: pinned float32 (nv, nu, nu)."""
        counts = counts_host.to(device, non_blocking=True)
        vol = self.run_device(counts)
        out_host.copy_(vol, non_blocking=True)
        return out_host


class ParallelPipeline:
    def __init__(self, config: M.ReconConfig, angles, weights, darks: torch.Tensor, flats: torch.Tensor,
                 filter_params: dict | None = None, precision: str = "fp32", referencecompat: bool = True):
        self.config = config
        self.angles = np.asarray(angles, np.float32)
        self.weights = np.asarray(weights, np.float32)
        self.norm = M.FullLogNorm()
        self.norm.Configure(config, {"usenormregion": "false", "uselut": "false", "referenceaverage": "ImageAverage"})
        self.norm.SetReferenceImages(darks, flats)
        self.filter = M.ProjectionFilterSingle()
        self.filter.Configure(config, filter_params or {"filtertype": "hanning", "cutoff": "0.5", "order": "1",
                                                        "usebias": "true", "biasweight": "0.1",
                                                        "paddingdoubler": "2"})
        self.bp = M.MultiProjectionBPparallel()
        self.bp.Configure(config, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1",
                                   "precision": precision, "referencecompat": str(referencecompat).lower()})
        roi = config.ProjectionInfo.roi
        self.roi = tuple(int(v) for v in roi)
        self.bp.SetROI(self.roi)
        self._params = {"angles": _text(self.angles), "weights": _text(self.weights)}

    def run_device(self, counts: torch.Tensor) -> torch.Tensor:
        self.bp.volume.zero_()
        proj = self.norm.ProcessCore(counts, {})
        w = torch.from_numpy(self.weights).to(counts.device)
        self.filter.ProcessCore(proj, {}, weights=w)
        self.bp.Process(proj, self._params, prefiltered_weights=True)
        return self.bp.GetVolume()
