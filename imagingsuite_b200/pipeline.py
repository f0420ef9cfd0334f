"""Device-resident reconstruction chains (the block loop of ReconEngine::Process3D,
frameworks/tomography/Framework/ReconFramework/src/ReconEngine.cpp:1314-1714, for one block).

``FdkPipeline``: FullLogNorm -> FDKbp_single (ramp filter + cone-beam backprojection),
``ParallelPipeline``: FullLogNorm -> ProjectionFilterSingle (+ fused projection weights) ->
MultiProjectionBPparallel, ``ParallelChain``: the same with MorphSpotClean and
WaveletRingClean between normalisation and filter, from configured module instances.
Projections stay in HBM between modules; ``run_host`` is the end-to-end form that takes
uint16 counts in host memory and returns the volume in host memory, with the copies
overlapped with the computation (counts in by groups of projections, the volume out by
blocks of slices or rows while the next block is backprojected).
"""
from __future__ import annotations

import numpy as np
import torch

from . import modules as M


def _text(a) -> str:
    return " ".join("%.9g" % v for v in np.asarray(a, np.float32))


def _check_device(where: str) -> None:
    from . import _lib as L

    try:
        L.check_device()
    except L.MrError as e:
        raise M.LibraryFailure(where, e) from e


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

    @staticmethod
    def check_device() -> None:
        """Raises LibraryFailure (a ReconException) when a kernel of the finished work left the
        device error word of an expired bounded wait; synchronises the device."""
        _check_device("FdkPipeline")

    def _lognorm_into(self, counts, out=None):
        from . import _lib as L

        nproj, nv, nu = counts.shape
        out = self._norm_buf if out is None else out
        dl = torch.zeros(1, device=counts.device)
        dark, flat = self.norm.mDark, self.norm.mFlatField
        L.check(L.lib().mr_lognorm_apply(counts.data_ptr(), L.MR_U16, nv * nu, nproj,
                                         None if dark is None else dark.data_ptr(),
                                         None if flat is None else flat.data_ptr(), dl.data_ptr(), 1,
                                         int(self.norm.nDCCount > 0), int(self.norm.nOBCount > 0),
                                         out.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return out

    def slab_plan(self, world: int):
        """The volume's z-slabs for `world` ranks with their detector-row windows
        (distributed.cone_slab_plan on this geometry's partials)."""
        from .distributed import cone_slab_plan

        xip, yip, zip_, *_ = self.fdk.partials(self.angles)
        return cone_slab_plan(self.nv, world, xip, yip, zip_, self.nu)

    def run_slab(self, counts_rows: torch.Tensor, slab) -> torch.Tensor:
        """One rank's share of the volume (FP32): counts_rows are the uint16 counts of the
        slab's detector-row window (nproj, slab.rows, nu) on the device; FullLogNorm and the
        ramp filter run on those rows only (mr_fdk_filter_rows), and the slab's slices are
        backprojected (mr_fdk_backproject_slab). Returns the volume buffer (nv, nu, nu), of which
        slices [slab.start, slab.stop) hold this slab; they equal the whole-volume call's."""
        from . import _lib as L

        if self.fdk.precision != "fp32":
            raise M.ReconException("FdkPipeline.run_slab: FP32 only")
        nproj, rows, nu = counts_rows.shape
        if rows != slab.rows or nu != self.nu:
            raise M.ReconException("FdkPipeline.run_slab: counts do not match the slab's row window")
        dev = counts_rows.device
        if getattr(self, "_slab_bufs", None) is None or self._slab_bufs[0].shape != counts_rows.shape:
            self._slab_bufs = (torch.empty(counts_rows.shape, dtype=torch.float32, device=dev),
                               torch.empty(counts_rows.shape, dtype=torch.float32, device=dev),
                               torch.empty((nproj, self.nv, nu), dtype=torch.float32, device=dev))
        norm, win, filt = self._slab_bufs
        geo = self.fdk.prepare(self.angles, self.weights, dev)
        w, *_, s2, sc, uni, box, maps = geo
        st = torch.cuda.current_stream(dev).cuda_stream
        off = slab.row_start * nu
        dark, flat = self.norm.mDark, self.norm.mFlatField
        dl = torch.zeros(1, device=dev)
        L.check(L.lib().mr_lognorm_apply(counts_rows.data_ptr(), L.MR_U16, rows * nu, nproj,
                                         None if dark is None else dark.data_ptr() + 4 * off,
                                         None if flat is None else flat.data_ptr() + 4 * off, dl.data_ptr(), 1,
                                         int(self.norm.nDCCount > 0), int(self.norm.nOBCount > 0), norm.data_ptr(),
                                         st))
        L.check(L.lib().mr_fdk_filter_rows(norm.data_ptr(), nu, rows, slab.row_start, self.nv, nproj, w.data_ptr(),
                                           s2, sc, L.MR_F32, win.data_ptr(), None, st))
        filt[:, slab.row_start:slab.row_stop].copy_(win)
        self.fdk.backproject(filt, None, geo, k_range=slab.cbct_range(self.nv), accumulate=False)
        return self.fdk.GetVolume()

    def run_host(self, counts_host: torch.Tensor, out_host: torch.Tensor, device, chunks: int = 8,
                 slabs: int = 8) -> torch.Tensor:
        """counts_host: pinned uint16 (nproj, nv, nu); out_host: pinned float32 (nv, nu, nu).

        FP32: the counts go to the device in `chunks` groups of projections on a copy stream,
        and FullLogNorm, the ramp filter and the backprojection of the first slice block
        (ReconEngine's slice blocks) for a group start as soon as it has landed; the other
        `slabs` - 1 blocks are then backprojected with all projections, and each finished block
        is copied to the host while the next one is computed. A voxel still adds its
        projections in order (the first block continues its sums from the volume between
        groups), so every value equals the one-shot path's. The result is complete when the
        current stream is synchronised. Other precisions copy, reconstruct and copy back in
        sequence."""
        if self.fdk.precision != "fp32":
            counts = counts_host.to(device, non_blocking=True)
            vol = self.run_device(counts)
            out_host.copy_(vol, non_blocking=True)
            return out_host
        nproj, nv, nu = counts_host.shape
        comp = torch.cuda.current_stream(device)
        if getattr(self, "_copy_stream", None) is None:
            self._copy_stream = torch.cuda.Stream(device)
            self._counts_d = torch.empty(counts_host.shape, dtype=torch.uint16, device=device)
            self._norm_buf = torch.empty(counts_host.shape, dtype=torch.float32, device=device)
            self._filt_d = torch.empty(counts_host.shape, dtype=torch.float32, device=device)
        cs, counts, proj, filt = self._copy_stream, self._counts_d, self._norm_buf, self._filt_d
        geo = self.fdk.prepare(self.angles, self.weights, device)
        cs.wait_stream(comp)  # buffers are free once the previous work on them is done
        bounds = [nproj * c // chunks for c in range(chunks + 1)]
        landed = []
        with torch.cuda.stream(cs):
            for a, b in zip(bounds[:-1], bounds[1:]):
                counts[a:b].copy_(counts_host[a:b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                landed.append(ev)
        # slabs of cbct slices k (multiples of 32, the backprojector's slice tile); cbct slice k
        # is final volume slice nv - 1 - k
        step = max(32, -(-nv // (slabs * 32)) * 32)
        started = False
        for (a, b), ev in zip(zip(bounds[:-1], bounds[1:]), landed):
            if b == a:
                continue
            comp.wait_event(ev)
            self._lognorm_into(counts[a:b], proj[a:b])
            self.fdk.ramp_filter(proj[a:b], geo, first=a, out=filt[a:b])
            self.fdk.backproject(filt[a:b], None, geo, k_range=(0, min(nv, step)), first=a, accumulate=started)
            started = True
        self.fdk._first = True
        for k0 in range(0, nv, step):
            k1 = min(nv, k0 + step)
            if k0 > 0:
                self.fdk.backproject(filt, None, geo, k_range=(k0, k1))
            done = torch.cuda.Event()
            done.record(comp)
            cs.wait_event(done)
            with torch.cuda.stream(cs):
                out_host[nv - k1:nv - k0].copy_(self.fdk.volume[nv - k1:nv - k0], non_blocking=True)
        self.fdk._first = False
        comp.wait_stream(cs)
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


class ParallelChain:
    """ReconEngine's block chain for parallel beam from configured modules: FullLogNorm ->
    [MorphSpotClean] -> [WaveletRingClean] -> ProjectionFilterSingle (projection weights
    fused) -> MultiProjectionBPparallel (weights not applied again)."""

    def __init__(self, norm: M.FullLogNorm, filt: M.ProjectionFilterSingle, bp: M.MultiProjectionBPparallel,
                 angles, weights, spot: M.MorphSpotCleanModule | None = None, ring: M.WaveletRingClean | None = None,
                 validate: bool = False):
        self.norm, self.filt, self.bp, self.spot, self.ring = norm, filt, bp, spot, ring
        self.validate = validate  # the engine's ReconConfig.System.bValidateData
        self.angles = np.asarray(angles, np.float32)
        self.weights = np.asarray(weights, np.float32)
        self._params = {"angles": _text(self.angles), "weights": _text(self.weights)}
        self._w = None
        self._copy_stream = None

    def _weights_on(self, device):
        if self._w is None or self._w.device != device:
            self._w = torch.from_numpy(self.weights).to(device)
        return self._w

    def run_device(self, counts: torch.Tensor, progress=None) -> torch.Tensor | None:
        """counts: uint16 (or float32) (nproj, nv, nu) on the device. Returns the volume
        (ny, nx, nz).

        progress(fraction, message) -> bool stands for InteractionBase::SetProgress: it is asked
        before each module, as ReconEngine::Process3D does (ReconEngine.cpp:1283-1290), and a
        True answer cancels the block between two modules (nothing of the block is left
        running; returns None). With `validate` (System.bValidateData) the projections
        are counted for NaNs and infinities after each preprocessing module and after the
        backprojection (validate_image, which logs the engine's warning)."""
        validate = self.validate
        stages = ["FullLogNorm"] + (["MorphSpotClean"] if self.spot is not None else []) + \
                 (["WaveletRingClean"] if self.ring is not None else []) + ["ProjectionFilterSingle", "BackProject"]
        self.bp.volume.zero_()
        proj = None
        for k, name in enumerate(stages):
            if progress is not None and progress(k / len(stages), f"Processing: {name}"):
                return None
            if name == "FullLogNorm":
                proj = self.norm.ProcessCore(counts, {})
            elif name == "MorphSpotClean":
                self.spot.ProcessCore(proj, {})
            elif name == "WaveletRingClean":
                self.ring.ProcessCore(proj, {})
            elif name == "ProjectionFilterSingle":
                self.filt.ProcessCore(proj, {}, weights=self._weights_on(counts.device))
            else:
                self.bp.Process(proj, self._params, prefiltered_weights=True)
            if validate:
                M.validate_image(proj, name if name != "BackProject" else "Projections post recon BackProject3D")
        return self.bp.GetVolume()

    @staticmethod
    def check_device() -> None:
        """Raises LibraryFailure (a ReconException) when a kernel of the finished work left the
        device error word of an expired bounded wait; synchronises the device."""
        _check_device("ParallelChain")

    def run_host(self, counts_host: torch.Tensor, out_host: torch.Tensor, device, chunks: int = 2,
                 blocks: int = 8) -> torch.Tensor:
        """counts_host: pinned uint16 (nproj, nv, nu); out_host: pinned float32 volume (ny, nx, nz).

        The counts go to the device in `chunks` groups of projections on a copy stream;
        FullLogNorm and MorphSpotClean (per projection) of a group start as soon as it has
        landed (few groups: MorphSpotClean runs one image per CTA and needs hundreds of images
        per launch to fill the GPU). Ring cleaning (per sinogram) and the filter then run on
        the whole block, and the volume is backprojected in `blocks` blocks of rows
        (contiguous in the z-fastest layout), each copied to the host while the next one is
        computed. Blocks below 64 MiB of counts or of volume are not split. Every value equals
        run_device's. The result is complete when the current stream is synchronised."""
        nproj, nv, nu = counts_host.shape
        if counts_host.numel() * 2 < (64 << 20):
            chunks = 1
        if out_host.numel() * 4 < (64 << 20):
            blocks = 1
        comp = torch.cuda.current_stream(device)
        if self._copy_stream is None or getattr(self, "_shape", None) != tuple(counts_host.shape):
            self._copy_stream = torch.cuda.Stream(device)
            self._counts_d = torch.empty(counts_host.shape, dtype=torch.uint16, device=device)
            self._proj_d = torch.empty(counts_host.shape, dtype=torch.float32, device=device)
            self._shape = tuple(counts_host.shape)
        cs, counts, proj = self._copy_stream, self._counts_d, self._proj_d
        w = self._weights_on(device)
        cs.wait_stream(comp)  # the buffers are free once the previous work on them is done
        bounds = [nproj * c // chunks for c in range(chunks + 1)]
        landed = []
        with torch.cuda.stream(cs):
            for a, b in zip(bounds[:-1], bounds[1:]):
                counts[a:b].copy_(counts_host[a:b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                landed.append(ev)
        for (a, b), ev in zip(zip(bounds[:-1], bounds[1:]), landed):
            if b == a:
                continue
            comp.wait_event(ev)
            self.norm.ProcessCore(counts[a:b], {}, out=proj[a:b])
            if self.spot is not None:
                self.spot.ProcessCore(proj[a:b], {})
        if self.ring is not None:
            self.ring.ProcessCore(proj, {})
        self.filt.ProcessCore(proj, {}, weights=w)
        ny = self.bp.volume.shape[0]
        self.bp.volume.zero_()
        step = max(8, -(-ny // (blocks * 8)) * 8)  # multiples of the backprojector's 8-row tiles
        for y0 in range(0, ny, step):
            y1 = min(ny, y0 + step)
            self.bp.Process(proj, self._params, prefiltered_weights=True, rows=(y0, y1))
            done = torch.cuda.Event()
            done.record(comp)
            cs.wait_event(done)
            with torch.cuda.stream(cs):
                out_host[y0:y1].copy_(self.bp.volume[y0:y1], non_blocking=True)
        comp.wait_stream(cs)
        return out_host
