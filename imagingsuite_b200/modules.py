"""MuhRec preprocessing and backprojector modules on the mrcuda kernels.

Each class mirrors a reference module of the tomography framework: the same class name,
the same ``Configure(config, parameters)`` parameter names and meanings, the same
``SetROI``/``Process`` call sequence that ``ReconEngine::Process3D`` / ``BackProject3D``
drive (frameworks/tomography/Framework/ReconFramework/src/ReconEngine.cpp:1314-1714), and
the same exceptions for bad input (``ReconException`` here). Data are torch tensors on a
CUDA device; projections have the kipl ``TImage<float,3>`` layout ``(nproj, nv, nu)``.
Every computation runs in ``libmrcuda.so``; there is no CPU path.

Modules added beside the reference ones accept two extra parameters:
``precision`` (``fp32`` | ``bf16`` | ``fp16``: storage of filtered projections in the
backprojectors) and ``referencecompat`` (``true`` reproduces the reference's buffer rule of
MultiProjectionBPparallel, which skips the last projection of every full buffer).
"""
from __future__ import annotations

import ctypes
import functools
import logging
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from ._lib import check


class ReconException(RuntimeError):
    """Mirror of ReconException (frameworks/tomography/Framework/ReconFramework/include/ReconException.h)."""


class LibraryFailure(ReconException, L.MrError):
    """A failed library call inside a module: a ReconException to the engine (as the reference's
    modules raise it, ReconEngine.cpp:810-833) that keeps the library's status code."""

    def __init__(self, where: str, err: L.MrError):
        L.MrError.__init__(self, err.status, f"{where}: {getattr(err, 'message', err)}")


_MODULE_CALLS = ("Configure", "SetROI", "SetReferenceImages", "Process", "ProcessCore", "GetSlice")


def _module(cls):
    """Class decorator of the modules: each of their public calls runs inside an NVTX range
    '<module>.<call>' (the reference times every Process, ProcessModuleBase.cpp:129-149) and
    turns a library failure into LibraryFailure."""
    for name in _MODULE_CALLS:
        fn = cls.__dict__.get(name)
        if fn is not None:
            setattr(cls, name, _module_call(fn, name))
    return cls


def _module_call(fn, call: str):
    @functools.wraps(fn)
    def run(self, *args, **kwargs):
        lib = L.lib()
        where = f"{type(self).__name__}.{call}"
        lib.mr_trace_push(where.encode())
        try:
            return fn(self, *args, **kwargs)
        except LibraryFailure:
            raise
        except L.MrError as e:
            raise LibraryFailure(where, e) from e
        finally:
            lib.mr_trace_pop()

    return run


# ---------------------------------------------------------------------------- config


@dataclass
class ProjectionInfo:
    """Subset of ReconConfig::cProjections (ReconConfig.h:77-175) read by the hot path."""

    nDims: tuple = (0, 0, 0)
    fResolution: tuple = (0.1, 0.1)
    fCenter: float = 0.0
    fSOD: float = 100.0
    fSDD: float = 100.0
    fpPoint: tuple = (0.0, 0.0)
    fTiltAngle: float = 0.0
    fTiltPivotPosition: float = 0.0
    bCorrectTilt: bool = False
    nOBCount: int = 0
    nDCCount: int = 0
    roi: tuple = (0, 0, 0, 0)
    projection_roi: tuple = (0, 0, 0, 0)
    dose_roi: tuple = (0, 0, 0, 0)
    eDirection: int = 0  # kipl::base::RotationDirCW = 0, RotationDirCCW = 1


@dataclass
class MatrixInfo:
    """Subset of ReconConfig::cMatrix (ReconConfig.h:177-200)."""

    nDims: tuple = (0, 0, 0)
    fVoxelSize: tuple = (0.1, 0.1, 0.1)
    bUseROI: bool = False
    roi: tuple = (0, 0, 0, 0)  # x0, y0, x1, y1 of the slices, inclusive (GetSlice crops to it)


@dataclass
class SystemInfo:
    """Subset of ReconConfig::cSystem (ReconConfig.cpp:245-255,552): bValidateData turns on the
    engine's NaN/infinity count after each module (ReconEngine::validateImage)."""

    bValidateData: bool = False


@dataclass
class ReconConfig:
    ProjectionInfo: ProjectionInfo = field(default_factory=ProjectionInfo)
    MatrixInfo: MatrixInfo = field(default_factory=MatrixInfo)
    System: SystemInfo = field(default_factory=SystemInfo)


logger = logging.getLogger("imagingsuite_b200")


def validate_image(data: torch.Tensor, description: str) -> int:
    """ReconEngine::validateImage (ReconEngine.cpp:1724-1740): counts the NaNs and infinities of
    a float tensor on the device (mr_data_validator) and logs the engine's warning when there
    are any. Returns their number (reads it back, so the current stream is synchronised)."""
    _require_cuda(data, "data")
    if data.dtype != torch.float32:
        raise ReconException("validate_image: float32 data expected")
    counts = torch.empty(2, dtype=torch.int64, device=data.device)
    check(L.lib().mr_data_validator(data.data_ptr(), data.numel(), counts.data_ptr(), _stream()))
    nan, inf = (int(v) for v in counts.cpu())
    if nan or inf:
        logger.warning("Encountered %d infs and %d NaNs in %s", inf, nan, description)
    return nan + inf


def _string2bool(s: str) -> bool:
    v = str(s).strip().lower()
    if v in ("true", "1", "yes", "on"):
        return True
    if v in ("false", "0", "no", "off"):
        return False
    raise ReconException(f"Could not convert {s!r} to bool")


def _get(parameters: dict, name: str) -> str:
    # ModuleConfig GetStringParameter (core/modules/ModuleConfig/src/ParameterHandling.cpp:25-40)
    if name not in parameters:
        raise ReconException(f"The parameter {name} was not found in the parameter list")
    return str(parameters[name])


def _float_vector(text: str, n: int) -> np.ndarray:
    """GetFloatParameterVector (ParameterHandling.cpp:55-77): n values from a space separated list."""
    vals = np.array(str(text).split(), dtype=np.float32)
    if vals.size < n:
        raise ReconException(f"Parameter list has {vals.size} values, {n} needed")
    return vals[:n]


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _require_cuda(t: torch.Tensor, what: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ReconException(f"{what} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ReconException(f"{what} must be contiguous")


_DT = {torch.float32: L.MR_F32, torch.uint16: L.MR_U16}
_PRECISION = {"fp32": L.MR_F32, "bf16": L.MR_BF16, "fp16": L.MR_F16}
_AVERAGE = {"imagesum": 0, "imageaverage": 1, "imagemedian": 2, "imageweightedaverage": 3, "imagemin": 4,
            "imagemax": 5}


# ------------------------------------------------------------------------ FullLogNorm


@_module
class FullLogNorm:
    """FullLogNorm (frameworks/tomography/Preprocessing/StdPreprocModules/src/NormPlugins.cpp:243-552).

    Reference frames are given in memory (``SetReferenceImages(darks, flats)``) instead of
    read from files by ``LoadReferenceImages``; their doses follow ``ReferenceLoader``
    (NormPlugins.cpp:91-230)."""

    def __init__(self):
        self.bUseNormROI = True
        self.bUseLUT = False
        self.referenceaverage = "ImageWeightedAverage"
        self.nOBCount = self.nDCCount = 0
        self.dose_roi = (0, 0, 0, 0)
        self.fDarkDose = 0.0
        self.fFlatDose = 1.0
        self.mDark = None
        self.mFlatField = None  # log of the flat field after SetReferenceImages

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        pi = config.ProjectionInfo
        self.nOBCount, self.nDCCount = int(pi.nOBCount), int(pi.nDCCount)
        self.bUseNormROI = _string2bool(_get(parameters, "usenormregion"))
        self.bUseLUT = _string2bool(parameters.get("uselut", "false"))
        self.referenceaverage = _get(parameters, "referenceaverage")
        if self.referenceaverage.lower() not in _AVERAGE:
            raise ReconException(f"Unknown reference average method {self.referenceaverage}")
        self.dose_roi = tuple(int(v) for v in pi.dose_roi)
        return 0

    def GetParameters(self) -> dict:
        return {"usenormregion": "true" if self.bUseNormROI else "false",
                "uselut": "true" if self.bUseLUT else "false", "referenceaverage": self.referenceaverage}

    def _frame_doses(self, frames: torch.Tensor) -> np.ndarray:
        n, nv, nu = frames.shape
        out = torch.empty(n, dtype=torch.float32, device=frames.device)
        roi = (ctypes.c_size_t * 4)(*self.dose_roi)
        check(L.lib().mr_projection_dose(frames.data_ptr(), _DT[frames.dtype], nu, nv, n, roi, out.data_ptr(),
                                         _stream()))
        return out.cpu().numpy()

    def _average(self, frames: torch.Tensor) -> torch.Tensor:
        n, nv, nu = frames.shape
        m = _AVERAGE[self.referenceaverage.lower()]
        out = torch.empty((nv, nu), dtype=torch.float32, device=frames.device)
        check(L.lib().mr_reference_average(frames.data_ptr(), nu, nv, n, m, out.data_ptr(), _stream()))
        return out

    def SetReferenceImages(self, darks: torch.Tensor, flats: torch.Tensor) -> None:
        """Average the reference frames, compute their doses, store dark and log(flat)."""
        for t, w in ((darks, "dark frames"), (flats, "flat frames")):
            _require_cuda(t, w)
        darks = darks.float() if darks.dtype != torch.float32 else darks
        flats = flats.float() if flats.dtype != torch.float32 else flats
        nd, nf = darks.shape[0], flats.shape[0]
        self.nDCCount, self.nOBCount = nd, nf
        f32 = np.float32
        darkdose = f32(0.0)
        self.mDark = self.mFlatField = None
        if nd:
            doses = self._frame_doses(darks) if self.bUseNormROI else np.zeros(nd, np.float32)
            acc = f32(0.0)
            for i in range(nd):
                acc = doses[i] if i == 0 else f32(acc + doses[i])
            darkdose = f32(acc / f32(nd))
            self.mDark = self._average(darks)
        flatdose = f32(1.0)
        if nf:
            doses = self._frame_doses(flats) if self.bUseNormROI else np.ones(nf, np.float32)
            acc = f32(0.0)
            for i in range(nf):
                t = f32(doses[i] - darkdose)
                acc = t if i == 0 else f32(acc + t)
            flatdose = f32(acc / f32(nf))
            flat = self._average(flats)
            # FullLogNorm::SetReferenceImages (NormPlugins.cpp:300-311): the reference dose must be finite
            dose = f32(1.0) / flatdose if flatdose != 0 else f32(np.inf)
            if np.isnan(dose):
                raise ReconException("The reference dose is a NaN")
            if np.isinf(dose):
                raise ReconException("The reference dose is Inf")
            self.mFlatField = torch.empty_like(flat)
            check(L.lib().mr_lognorm_logflat(self.mDark.data_ptr() if nd else flat.data_ptr(), flat.data_ptr(),
                                             flat.numel(), int(nd > 0), float(flatdose), self.mFlatField.data_ptr(),
                                             _stream()))
        self.fDarkDose, self.fFlatDose = float(darkdose), float(flatdose)
        # without flats the module runs -log(I - D) + dose (NormPlugins.cpp:498-540); without
        # darks I - D is I
        self._refs_set = True

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict, out: torch.Tensor | None = None) -> torch.Tensor:
        """ProcessCore 3D. ``img`` is float32 or uint16 (raw counts); returns float32 (in
        ``out`` when given, else in place for float32 input or in a new tensor).
        Doses come from ``coeff['dose']`` (text, as the engine passes them) or, when absent,
        are computed on the device over the dose ROI (ProjectionReader::GetProjectionDose)."""
        _require_cuda(img, "projections")
        if not getattr(self, "_refs_set", False):
            raise ReconException("FullLogNorm: reference images are not set")
        nproj, nv, nu = img.shape
        if self.nOBCount and self.mFlatField.numel() != nv * nu:
            raise ReconException(f"Flat field ({self.mFlatField.shape[1]}, {self.mFlatField.shape[0]}), does not match "
                                 f"projection ({nu}, {nv})")
        if self.nDCCount and self.mDark.numel() != nv * nu:
            raise ReconException(f"Dark field ({self.mDark.shape[1]}, {self.mDark.shape[0]}), does not match "
                                 f"projection ({nu}, {nv})")
        if self.bUseNormROI:
            doses = (_float_vector(coeff["dose"], nproj) if "dose" in coeff else self._frame_doses(img))
            doses = np.ascontiguousarray(doses, np.float32)
            dl = np.empty_like(doses)
            check(L.lib().mr_lognorm_doselog(doses.ctypes.data_as(L.P_float), nproj, self.fDarkDose,
                                             dl.ctypes.data_as(L.P_float)))
        else:
            dl = np.zeros(1, np.float32)
        doselog = torch.from_numpy(dl).to(img.device)
        if out is None:
            out = img if img.dtype == torch.float32 else torch.empty(img.shape, dtype=torch.float32, device=img.device)
        elif out.shape != img.shape or out.dtype != torch.float32 or not out.is_contiguous():
            raise ReconException("FullLogNorm: out must be a contiguous float32 tensor of the projections' shape")
        apply = L.lib().mr_lognorm_apply_lut if self.bUseLUT else L.lib().mr_lognorm_apply
        check(apply(img.data_ptr(), _DT[img.dtype], nv * nu, nproj, _ptr(self.mDark), _ptr(self.mFlatField),
                    doselog.data_ptr(), doselog.numel(), int(self.nDCCount > 0), int(self.nOBCount > 0),
                    out.data_ptr(), _stream()))
        return out


# ------------------------------------------------------------------- MorphSpotClean

_CONN = {"conn4": 0, "conn8": 1}
_DETECT = {"morphdetectholes": 0, "morphdetectpeaks": 1, "morphdetectboth": 2}


def morph_spot_clean(img: torch.Tensor, detect: int = 0, conn8: bool = True, th=(0.025, 0.025), sigma=(0.0, 0.0),
                     edge: int = 9, clamp: bool = False, minlevel: float = -0.1, maxlevel: float = 7.0,
                     removeinfnan: bool = False) -> torch.Tensor:
    """ImagingAlgorithms::MorphSpotClean::process (replace mode) in place on (n, nv, nu) or (nv, nu)."""
    _require_cuda(img, "image")
    if img.dtype != torch.float32:
        raise ReconException("MorphSpotClean expects float32 images")
    nv, nu = img.shape[-2:]
    n = img.numel() // (nv * nu)
    t = np.asarray(th, np.float32)
    s = np.asarray(sigma, np.float32)
    check(L.lib().mr_morphspotclean(img.data_ptr(), nu, nv, n, int(detect), int(conn8), t.ctypes.data_as(L.P_float),
                                    s.ctypes.data_as(L.P_float), int(edge), int(clamp), float(minlevel),
                                    float(maxlevel), int(removeinfnan), _stream()))
    return img


@_module
class MorphSpotCleanModule:
    """MorphSpotCleanModule (StdPreprocModules/src/MorphSpotCleanModule.cpp:14-183). As in
    the reference's single-threaded path (ProcessSingle :142-181) the cleaner runs with its
    own edge smoothing length (9; the `edgesmooth` parameter is read but not applied) and
    without inf/NaN removal (`removeinfnan` is read but not applied); clamping follows
    `clampdata` on that path and is off with `threading` (ProcessParallelStd never sets the
    cleaner's limits)."""

    def __init__(self):
        self.m_eConnectivity = "conn4"
        self.m_eDetectionMethod = "morphdetectpeaks"
        self.m_eCleanMethod = "morphcleanreplace"
        self.m_fThreshold = [0.1, 0.1]
        self.m_fSigma = [0.01, 0.01]
        self.m_nEdgeSmoothLength = 5
        self.m_nMaxArea = 30
        self.m_bRemoveInfNaN = False
        self.m_bClampData = False
        self.m_fMinLevel = -0.1
        self.m_fMaxLevel = 7.0
        self.m_bThreading = False

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        try:
            conn = _get(parameters, "connectivity")
            clean = _get(parameters, "cleanmethod")
            det = _get(parameters, "detectionmethod")
            if conn not in _CONN or clean not in ("morphcleanreplace", "morphcleanfill") or det not in _DETECT:
                return -1
            self.m_eConnectivity, self.m_eCleanMethod, self.m_eDetectionMethod = conn, clean, det
            self.m_fThreshold = [float(np.float32(v)) for v in _get(parameters, "threshold").split()]
            self.m_fSigma = [float(np.float32(v)) for v in _get(parameters, "sigma").split()]
            self.m_nEdgeSmoothLength = int(_get(parameters, "edgesmooth"))
            self.m_nMaxArea = int(_get(parameters, "maxarea"))
            self.m_bRemoveInfNaN = _string2bool(_get(parameters, "removeinfnan"))
            self.m_bClampData = _string2bool(_get(parameters, "clampdata"))
            self.m_fMinLevel = float(np.float32(_get(parameters, "minlevel")))
            self.m_fMaxLevel = float(np.float32(_get(parameters, "maxlevel")))
            self.m_bThreading = _string2bool(_get(parameters, "threading"))
        except (ReconException, ValueError):
            return -1
        return 0

    def GetParameters(self) -> dict:
        return {"connectivity": self.m_eConnectivity, "cleanmethod": self.m_eCleanMethod,
                "detectionmethod": self.m_eDetectionMethod, "threshold": " ".join(map(str, self.m_fThreshold)),
                "sigma": " ".join(map(str, self.m_fSigma)), "edgesmooth": str(self.m_nEdgeSmoothLength),
                "maxarea": str(self.m_nMaxArea), "removeinfnan": str(self.m_bRemoveInfNaN).lower(),
                "clampdata": str(self.m_bClampData).lower(), "minlevel": str(self.m_fMinLevel),
                "maxlevel": str(self.m_fMaxLevel), "threading": str(self.m_bThreading).lower()}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        if self.m_eCleanMethod != "morphcleanreplace":
            raise ReconException("MorphSpotClean: only morphcleanreplace is supported by this module")
        # threading=true takes the reference's ProcessParallelStd (MorphSpotCleanModule.cpp:
        # 226-269), whose cleaners never get setLimits: no clamping there
        clamp = self.m_bClampData and not self.m_bThreading
        return morph_spot_clean(img, _DETECT[self.m_eDetectionMethod], self.m_eConnectivity == "conn8",
                                self.m_fThreshold[:2], self.m_fSigma[:2], edge=9, clamp=clamp,
                                minlevel=self.m_fMinLevel, maxlevel=self.m_fMaxLevel, removeinfnan=False)


# ------------------------------------------------------------------ WaveletRingClean


def stripe_filter(sino: torch.Tensor, wname: str = "daub15", decnum: int = 2, sigma: float = 0.05) -> torch.Tensor:
    """ImagingAlgorithms::StripeFilter::process (VerticalComponentFFT) in place on sinograms
    (n, ntheta, nu) or (ntheta, nu)."""
    _require_cuda(sino, "sinogram")
    ntheta, nu = sino.shape[-2:]
    n = sino.numel() // (ntheta * nu)
    check(L.lib().mr_stripefilter(sino.data_ptr(), nu, ntheta, n, wname.encode(), int(decnum), float(sigma),
                                  _stream()))
    return sino


@_module
class WaveletRingClean:
    """WaveletRingClean (StdPreprocModules/src/WaveletRingClean.cpp:17-146). As in the
    reference, `method` is read but every sinogram is filtered with VerticalComponentFFT."""

    def __init__(self):
        self.m_sWName = "daub15"
        self.m_fSigma = 0.05
        self.m_nDecNum = 2
        self.m_bParallelProcessing = False
        self.m_eCleanMethod = "verticalfft"

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        self.m_sWName = _get(parameters, "wname")
        self.m_fSigma = float(np.float32(_get(parameters, "sigma")))
        self.m_nDecNum = int(_get(parameters, "decnum"))
        self.m_bParallelProcessing = _string2bool(_get(parameters, "parallel"))
        method = _get(parameters, "method")
        if method not in ("verticalzero", "verticalfft"):
            raise ReconException(f"Could not translate string ({method}) to stripe filter operation")
        self.m_eCleanMethod = method
        return 0

    def GetParameters(self) -> dict:
        return {"wname": self.m_sWName, "sigma": str(self.m_fSigma), "decnum": str(self.m_nDecNum),
                "parallel": "true" if self.m_bParallelProcessing else "false", "method": self.m_eCleanMethod}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        _require_cuda(img, "projections")
        nproj, nv, nu = img.shape
        st = L.lib().mr_waveletringclean(img.data_ptr(), nu, nv, nproj, self.m_sWName.encode(), self.m_nDecNum,
                                         self.m_fSigma, _stream())
        if st != L.MR_OK:
            raise LibraryFailure("Failed to process the projections using stripe filter",
                                 L.MrError(st, L.lib().mr_last_error().decode()))
        return img


# ------------------------------------------------------------ alternative ring cleaners


def _require_f32(t: torch.Tensor, what: str) -> None:
    _require_cuda(t, what)
    if t.dtype != torch.float32:
        raise ReconException(f"{what} must be float32")


def compute_weights(angles, scan_arc=(0.0, 360.0), golden_section: bool = False):
    """ComputeWeights (frameworks/tomography/Framework/ReconFramework/src/ReconHelpers.cpp:
    365-488) on projection angles in acquisition order, as BuildFileList lists them: returns the
    (angles, weights) of the weighted projection map in its order (host computation). The
    backprojectors' `weights` list is these weights times 1 / (0.1 * pixel size)."""
    a = np.ascontiguousarray(angles, dtype=np.float32)
    arc = np.asarray(scan_arc, dtype=np.float32)
    oa = np.zeros(max(a.size, 1), np.float32)
    ow = np.zeros(max(a.size, 1), np.float32)
    m = ctypes.c_size_t(0)
    check(L.lib().mr_compute_weights(a.ctypes.data_as(L.P_float), a.size, arc.ctypes.data_as(L.P_float),
                                     int(golden_section), oa.ctypes.data_as(L.P_float), ow.ctypes.data_as(L.P_float),
                                     ctypes.byref(m)))
    return oa[:m.value].copy(), ow[:m.value].copy()


def projection_lists(angles, weights, rotation: float = 0.0, resolution: float = 0.0) -> dict:
    """The `angles` and `weights` texts ProjectionReader::Read hands the backprojectors
    (frameworks/tomography/Framework/ReconFramework/src/ProjectionReader.cpp:907-919): angle +
    MatrixInfo.fRotation and weight * 1 / (0.1 * pixel size) (1 when the pixel size is not
    positive), in float, each written as a default-formatted stream value (6 significant
    digits, `%g`). The backprojectors then read these rounded values, as in the engine."""
    f32 = np.float32
    res = f32(resolution)
    rw = f32(1.0) / (res * f32(0.1) if f32(0) < res else f32(1.0))
    a = [f32(v) + f32(rotation) for v in np.asarray(angles, np.float32)]
    w = [f32(v) * rw for v in np.asarray(weights, np.float32)]
    return {"angles": " ".join(f"{float(v):g}" for v in a) + " ",
            "weights": " ".join(f"{float(v):g}" for v in w) + " "}


def median_filter(img: torch.Tensor, kx: int, ky: int) -> torch.Tensor:
    """kipl TMedianFilter<float,2> with a kx x ky window (odd sizes up to 5) on one image (nv, nu)
    or a stack (n, nv, nu); returns a new tensor."""
    _require_f32(img, "image")
    src = img
    nv, nu = src.shape[-2:]
    n = src.numel() // (nu * nv) if src.numel() else 0
    out = torch.empty_like(src)
    st = L.lib().mr_median_filter(src.data_ptr(), nu, nv, n, kx, ky, out.data_ptr(), _stream())
    if st != L.MR_OK:
        raise LibraryFailure("median filter failed", L.MrError(st, L.lib().mr_last_error().decode()))
    return out


@_module
class BasicRingClean:
    """BasicRingClean (StdPreprocModules/src/BasicRingClean.cpp:17-95): every projection minus
    (mean projection - its 3x3 median). No parameters. The reference also writes mean.tif,
    med.tif and diff.tif to its working directory as debug output; these are not written."""

    def __init__(self):
        pass

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        return 0

    def GetParameters(self) -> dict:
        return {}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        _require_f32(img, "projections")
        nproj, nv, nu = img.shape
        st = L.lib().mr_basicringclean(img.data_ptr(), nu, nv, nproj, _stream())
        if st != L.MR_OK:
            raise LibraryFailure("BasicRingClean failed", L.MrError(st, L.lib().mr_last_error().decode()))
        return img


@_module
class MedianMixRingClean:
    """MedianMixRingClean (StdPreprocModules/src/MedianMixRingClean.cpp:21-138): weights from
    a sigmoid of |mean projection - its 3x3 median| (threshold = sigmoid level, width = sigmoid
    width), then each projection mixed with its 5x5 median by those weights."""

    def __init__(self):
        self.m_fSigma = float(np.float32(0.0025))
        self.m_fLambda = float(np.float32(0.025))

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        self.m_fSigma = float(np.float32(_get(parameters, "width")))
        self.m_fLambda = float(np.float32(_get(parameters, "threshold")))
        return 0

    def GetParameters(self) -> dict:
        return {"threshold": "0.025", "width": "0.0025"}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        _require_f32(img, "projections")
        nproj, nv, nu = img.shape
        st = L.lib().mr_medianmixringclean(img.data_ptr(), nu, nv, nproj, self.m_fLambda, self.m_fSigma, _stream())
        if st != L.MR_OK:
            raise LibraryFailure("MedianMixRingClean failed", L.MrError(st, L.lib().mr_last_error().decode()))
        return img


_SPOT_METHODS = {"stddev": 0, "ring": 1, "median": 2, "minmax": 3, "trikernel": 4}


@_module
class SpotClean2:
    """SpotClean2 (StdPreprocModules/src/SpotClean2.cpp:42-130) over ImagingAlgorithms::SpotClean
    (core/algorithms/ImagingAlgorithms/src/SpotClean.cpp): detection image, sigmoid weights
    (gamma = level, sigma = width), exclusion of regions larger than maxarea, spots outside
    [minlevel, maxlevel], neighbour-mean filling; `iterations` passes. As in the reference's
    string2enum, an unknown detection method name selects ring."""

    def __init__(self):
        self.m_fGamma = float(np.float32(0.1))
        self.m_fSigma = float(np.float32(0.001))
        self.m_nIterations = 1
        self.m_fMaxLevel = 5.0
        self.m_fMinLevel = float(np.float32(-0.1))
        self.m_nMaxArea = 20
        self.m_eDetectionMethod = "ring"

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        self.m_fGamma = float(np.float32(_get(parameters, "gamma")))
        self.m_fSigma = float(np.float32(_get(parameters, "sigma")))
        self.m_nIterations = int(_get(parameters, "iterations"))
        self.m_fMaxLevel = float(np.float32(_get(parameters, "maxlevel")))
        self.m_fMinLevel = float(np.float32(_get(parameters, "minlevel")))
        self.m_nMaxArea = int(_get(parameters, "maxarea"))
        method = _get(parameters, "detectionmethod")
        self.m_eDetectionMethod = method if method in _SPOT_METHODS else "ring"
        return 0

    def GetParameters(self) -> dict:
        return {"gamma": f"{self.m_fGamma:g}", "sigma": f"{self.m_fSigma:g}", "iterations": str(self.m_nIterations),
                "maxlevel": f"{self.m_fMaxLevel:g}", "minlevel": f"{self.m_fMinLevel:g}",
                "maxarea": str(self.m_nMaxArea), "detectionmethod": self.m_eDetectionMethod}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        _require_f32(img, "projections")
        # a single image goes through SpotClean::Process(TImage<float,2>), which cleans once
        # whatever `iterations` says (SpotClean.cpp:64-76)
        img3, iters = (img.view(1, *img.shape), 1) if img.dim() == 2 else (img, self.m_nIterations)
        nproj, nv, nu = img3.shape
        st = L.lib().mr_spotclean2(img3.data_ptr(), nu, nv, nproj, _SPOT_METHODS[self.m_eDetectionMethod],
                                   self.m_fGamma, self.m_fSigma, iters, self.m_fMinLevel,
                                   self.m_fMaxLevel, self.m_nMaxArea, _stream())
        if st != L.MR_OK:
            raise LibraryFailure("SpotClean2 failed", L.MrError(st, L.lib().mr_last_error().decode()))
        return img


@_module
class GammaSpotClean:
    """GammaSpotCleanModule (StdPreprocModules/src/GammaSpotCleanModule.cpp:10-153). The
    reference keeps the parameters but its ProcessCore returns without touching the
    projections (the cleaning calls are commented out there), so this module does the same:
    the projections pass through unchanged and no device work is issued."""

    def __init__(self):
        self.m_fSigma = float(np.float32(0.8))
        self.m_fThreshold3 = 25.0
        self.m_fThreshold5 = 100.0
        self.m_fThreshold7 = 400.0
        self.m_nMedianSize = 3

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        self.m_fThreshold3 = float(np.float32(_get(parameters, "threshold3")))
        self.m_fThreshold5 = float(np.float32(_get(parameters, "threshold5")))
        self.m_fThreshold7 = float(np.float32(_get(parameters, "threshold7")))
        self.m_fSigma = float(np.float32(_get(parameters, "sigma")))
        self.m_nMedianSize = int(_get(parameters, "mediansize"))
        return 0

    def GetParameters(self) -> dict:
        return {"threshold3": f"{self.m_fThreshold3:g}", "threshold5": f"{self.m_fThreshold5:g}",
                "threshold7": f"{self.m_fThreshold7:g}", "sigma": f"{self.m_fSigma:g}",
                "mediansize": str(self.m_nMedianSize)}

    def SetROI(self, roi) -> bool:
        return False

    def Process(self, img: torch.Tensor, coeff: dict | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {})

    def ProcessCore(self, img: torch.Tensor, coeff: dict) -> torch.Tensor:
        _require_cuda(img, "projections")
        return img


# ------------------------------------------------------------ ProjectionFilterSingle


@_module
class ProjectionFilterSingle:
    """ProjectionFilterSingle (StdPreprocModules/src/ProjectionFilter.cpp:230-376)."""

    def __init__(self):
        self.m_FilterType = "Hamming"
        self.m_fCutOff = 0.5
        self.m_fOrder = 1.0
        self.m_bUseBias = True
        self.m_fBiasWeight = 0.1
        self.m_nPaddingDoubler = 2
        self._plan = None
        self.nImageSize = 0

    def __del__(self):
        if getattr(self, "_plan", None):
            L.lib().mr_projfilter_destroy(self._plan)
            self._plan = None

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        roi = config.ProjectionInfo.roi
        n = int(roi[2]) - int(roi[0])
        self.m_FilterType = _get(parameters, "filtertype")
        self.m_fCutOff = float(np.float32(_get(parameters, "cutoff")))
        self.m_fOrder = float(np.float32(_get(parameters, "order")))
        self.m_bUseBias = _string2bool(_get(parameters, "usebias"))
        self.m_fBiasWeight = float(np.float32(_get(parameters, "biasweight")))
        self.m_nPaddingDoubler = int(_get(parameters, "paddingdoubler"))
        self.nImageSize = n
        self.BuildFilter(n)
        return 0

    def BuildFilter(self, n: int) -> None:
        if self._plan:
            L.lib().mr_projfilter_destroy(self._plan)
            self._plan = None
        plan = ctypes.c_void_p()
        st = L.lib().mr_projfilter_create(n, self.m_FilterType.encode(), self.m_fCutOff, self.m_fOrder,
                                          int(self.m_bUseBias), self.m_fBiasWeight, self.m_nPaddingDoubler,
                                          ctypes.byref(plan))
        if st != L.MR_OK:
            raise LibraryFailure(type(self).__name__, L.MrError(st, L.lib().mr_last_error().decode()))
        self._plan = plan

    def GetParameters(self) -> dict:
        return {"filtertype": self.m_FilterType, "cutoff": str(self.m_fCutOff), "order": str(self.m_fOrder),
                "usebias": "true" if self.m_bUseBias else "false", "biasweight": str(self.m_fBiasWeight),
                "paddingdoubler": str(self.m_nPaddingDoubler)}

    def filter_tables(self):
        nfft, ins = ctypes.c_size_t(), ctypes.c_size_t()
        check(L.lib().mr_projfilter_info(self._plan, ctypes.byref(nfft), ctypes.byref(ins), None, None))
        f = np.zeros(nfft.value // 2, np.float32)
        p = np.zeros(max(ins.value, 1), np.float32)
        check(L.lib().mr_projfilter_info(self._plan, None, None, f.ctypes.data_as(L.P_float),
                                         p.ctypes.data_as(L.P_float)))
        return nfft.value, ins.value, f, p[: ins.value]

    def Process(self, img: torch.Tensor, coeff: dict | None = None, weights: torch.Tensor | None = None) -> torch.Tensor:
        return self.ProcessCore(img, coeff if coeff is not None else {}, weights)

    def ProcessCore(self, img: torch.Tensor, coeff: dict, weights: torch.Tensor | None = None) -> torch.Tensor:
        """Filters every detector row in place. ``weights`` (optional, one per projection)
        fuses the backprojector's projection weighting into the output."""
        if img.numel() == 0:
            raise ReconException("Empty projection image")
        _require_cuda(img, "projections")
        if img.dtype != torch.float32:
            raise ReconException("ProjectionFilterSingle expects float32 projections")
        nproj, nv, nu = img.shape
        if nu != self.nImageSize:
            raise ReconException(f"Projection width {nu} does not match the configured ROI width {self.nImageSize}")
        if weights is not None:
            _require_cuda(weights, "weights")
        check(L.lib().mr_projfilter_apply(self._plan, img.data_ptr(), img.data_ptr(), nproj * nv, _ptr(weights), nv,
                                          _stream()))
        return img


# --------------------------------------------------------------- backprojector base


@_module
class _BackProjectorBase:
    def __init__(self, name: str):
        self.m_sModuleName = name
        self.mConfig = ReconConfig()
        self.nProjectionBufferSize = 16
        self.nSliceBlock = 32
        self.nSubVolume = (1, 1)
        self.precision = "fp32"
        self.referencecompat = True
        self.volume = None

    def Configure(self, config: ReconConfig, parameters: dict) -> int:
        self.mConfig = config
        self.nProjectionBufferSize = int(_get(parameters, "ProjectionBufferSize"))
        self.nSliceBlock = int(_get(parameters, "SliceBlock"))
        sv = str(_get(parameters, "SubVolume")).split()
        self.nSubVolume = tuple(int(v) for v in sv[:2])
        self.precision = str(parameters.get("precision", "fp32")).lower()
        if self.precision not in _PRECISION:
            raise ReconException(f"Unknown precision {self.precision}")
        self.referencecompat = _string2bool(parameters.get("referencecompat", "true"))
        return 0

    def Initialize(self) -> int:
        return 0

    def GetParameters(self) -> dict:
        return {"ProjectionBufferSize": str(self.nProjectionBufferSize), "SliceBlock": str(self.nSliceBlock),
                "SubVolume": f"{self.nSubVolume[0]} {self.nSubVolume[1]}", "precision": self.precision,
                "referencecompat": "true" if self.referencecompat else "false"}

    def GetVolume(self) -> torch.Tensor:
        return self.volume

    def _slice_window(self, nx: int, ny: int):
        """BackProjectorModuleBase::GetSlice's slice window (BackProjectorModuleBase.cpp:62-84):
        the whole slice, or with MatrixInfo.bUseROI the inclusive crop roi[0]..roi[2] by
        roi[1]..roi[3]. The reference copies the crop without checking it against the volume;
        here a crop outside the slice raises."""
        mi = self.mConfig.MatrixInfo
        if not mi.bUseROI:
            return 0, 0, nx, ny
        x0, y0, x1, y1 = (int(v) for v in mi.roi)
        w, h = x1 - x0 + 1, y1 - y0 + 1
        if x0 < 0 or y0 < 0 or w <= 0 or h <= 0 or x0 + w > nx or y0 + h > ny:
            raise ReconException(f"Matrix ROI {tuple(mi.roi)} is outside the {nx} x {ny} slice")
        return x0, y0, w, h


def _restrict_mask(mask: np.ndarray, nx: int, mi: MatrixInfo, cone: bool) -> None:
    """The matrix-ROI part of BackProjectorModuleBase::BuildCircleMask
    (BackProjectorModuleBase.cpp:196-214), in place on the (first, second) pairs per row: rows
    inside roi[1]..roi[3] keep x in [roi[0], roi[2]] (parallel beam) or, mirrored,
    [nx - roi[2], nx - roi[0]] (cone beam); rows outside get an empty range."""
    if not mi.bUseROI:
        return
    r0, r1, r2, r3 = (int(v) for v in mi.roi)
    m = mask.reshape(-1, 2)
    for i in range(m.shape[0]):
        if r1 <= i <= r3:
            lo, hi = (r0, r2) if not cone else (nx - r2, nx - r0)
            m[i, 0] = max(int(m[i, 0]), lo)
            m[i, 1] = min(int(m[i, 1]), hi)
        else:
            m[i] = 0


def TransferMatrix(backprojector, volume: torch.Tensor, dims, first_slice: int = 0) -> bool:
    """ReconEngine::TransferMatrix (ReconEngine.cpp:531-574): the block's slices i = 0 ..
    dims[3] - dims[1] - 1 of the backprojector (GetSlice, with the matrix ROI) are copied into
    planes dims[1] - first_slice + i of the engine volume (planes, rows, columns). Errors of
    GetSlice are re-raised with the reference's context; so is a device error word left by a
    bounded wait that expired in the block's backprojection (the first point at which the
    block's volume is read back)."""
    try:
        vol = getattr(backprojector, "volume", None)
        if isinstance(vol, torch.Tensor) and vol.is_cuda:
            L.check_device()
        for i in range(int(dims[3]) - int(dims[1])):
            volume[int(dims[1]) - first_slice + i].copy_(backprojector.GetSlice(i))
    except L.MrError as e:
        raise LibraryFailure("Transfer matrix from backprojector failed with ReconException", e) from e
    except ReconException as e:
        raise ReconException(f"Transfer matrix from backprojector failed with ReconException\n{e}") from e
    return False


@_module
class MultiProjectionBPparallel(_BackProjectorBase):
    """MultiProjectionBPparallel (StdBackProjectors/src/MultiProjBPparallel.cpp) with the
    StdBackProjectorBase driver (StdBackProjectorBase.cpp). Volume is MatrixZXY:
    tensor (ny, nx, nz) = (nu, nu, nv), z fastest."""

    _variant = L.MR_BP_MULTIPROJ_PARALLEL

    def __init__(self):
        super().__init__("Multi projection BP parallel")
        self.SizeU = self.SizeV = 0
        self._mask = None
        self._roi = (0, 0, 0, 0)
        self.staging = True  # TMA-staged projection rows (False: direct global loads; same results)

    def SetROI(self, roi) -> None:
        pi = self.mConfig.ProjectionInfo
        self._roi = tuple(int(v) for v in roi)
        self.SizeU = self._roi[2] - self._roi[0]
        self.SizeV = self._roi[3] - self._roi[1]
        if self.SizeU < 2:
            raise ReconException("The projection ROI is too narrow")
        dev = torch.device("cuda", torch.cuda.current_device())
        self.volume = torch.zeros((self.SizeU, self.SizeU, self.SizeV), dtype=torch.float32, device=dev)
        mask = np.zeros(2 * self.SizeU, np.uint32)
        nslices = int(pi.nDims[1]) if pi.nDims[1] else self.SizeV
        check(L.lib().mr_bp_circle_mask(self.SizeU, self.SizeU, int(pi.bCorrectTilt), float(pi.fTiltAngle), nslices,
                                        mask.ctypes.data_as(L.P_u32)))
        _restrict_mask(mask, self.SizeU, self.mConfig.MatrixInfo, cone=False)
        self.mask_host = mask
        self._mask = torch.from_numpy(mask.view(np.int32)).to(dev)

    def used_projections(self, nproj: int) -> np.ndarray:
        """Indices the reference backprojects: StdBackProjectorBase::Process 2D flushes a full
        buffer without its last entry (StdBackProjectorBase.cpp:104-113)."""
        k = np.arange(nproj)
        if not self.referencecompat:
            return k
        b = self.nProjectionBufferSize
        return k[(k % b) != (b - 1)]

    def Process(self, projections: torch.Tensor, parameters: dict, prefiltered_weights: bool = False,
                rows: tuple | None = None) -> int:
        """Backprojects projections (nproj, nv, nu) with ``parameters['angles']`` and
        ``parameters['weights']`` (space separated text, as ReconEngine passes them).
        ``prefiltered_weights`` marks projections already multiplied by their weights
        (the fused filter path); the weights are then not applied again. ``rows`` = (y0, y1)
        restricts the backprojection to the volume rows y0 <= y < y1 (mr_bp_parallel_rows)."""
        if self.volume is None:
            raise ReconException("The target matrix is not allocated.")
        _require_cuda(projections, "projections")
        nproj, nv, nu = projections.shape
        if nu != self.SizeU or nv != self.SizeV:
            raise ReconException(f"Projection size ({nu}, {nv}) does not match the ROI ({self.SizeU}, {self.SizeV})")
        weights = _float_vector(_get(parameters, "weights"), nproj)
        angles = _float_vector(_get(parameters, "angles"), nproj)
        pi = self.mConfig.ProjectionInfo
        sel = self.used_projections(nproj)
        if sel.size == 0:
            return 0
        dev = projections.device
        # per-projection geometry on the device, kept while the angles, weights and geometry
        # settings stay the same (a block backprojected in row ranges reuses it)
        key = (angles.tobytes(), weights.tobytes(), sel.tobytes(), str(dev), self.SizeU, float(pi.fCenter),
               int(pi.eDirection), bool(pi.bCorrectTilt), float(pi.fTiltAngle), float(pi.fTiltPivotPosition),
               self._roi[1])
        if getattr(self, "_geo_key", None) != key:
            ang = np.ascontiguousarray(angles[sel])
            s = np.empty_like(ang)
            c = np.empty_like(ang)
            su = np.empty_like(ang)
            check(L.lib().mr_bp_parallel_geometry(ang.ctypes.data_as(L.P_float), ang.size, self.SizeU,
                                                  float(pi.fCenter), int(pi.eDirection), s.ctypes.data_as(L.P_float),
                                                  c.ctypes.data_as(L.P_float), su.ctypes.data_as(L.P_float)))
            toff, tinc = ctypes.c_float(0), ctypes.c_float(0)
            if pi.bCorrectTilt:
                check(L.lib().mr_bp_parallel_tilt(float(pi.fTiltAngle), float(pi.fTiltPivotPosition), self._roi[1],
                                                  ctypes.byref(toff), ctypes.byref(tinc)))
            self._geo = (torch.from_numpy(np.stack([s, c, su, weights[sel]])).to(dev),
                         torch.from_numpy(sel.astype(np.int32)).to(dev), toff, tinc)
            self._geo_key = key
        geo, idx, toff, tinc = self._geo
        proj = projections
        dtype = _PRECISION[self.precision]
        scale = None
        if dtype != L.MR_F32:
            proj, scale = quantize(projections, self.precision)
        args = (dtype, _ptr(scale), None if prefiltered_weights else geo[3].data_ptr(), idx.data_ptr(),
                geo[0].data_ptr(), geo[1].data_ptr(), geo[2].data_ptr(), sel.size, self.SizeU, self.SizeV,
                self._mask.data_ptr(), int(pi.bCorrectTilt), toff.value, tinc.value, self.volume.data_ptr(), _stream())
        if self._variant != L.MR_BP_MULTIPROJ_PARALLEL:
            y0, y1 = (0, self.SizeU) if rows is None else (int(rows[0]), int(rows[1]))
            check(L.lib().mr_bp_parallel_variant(self._variant, proj.data_ptr(), nproj, *args[:-2], y0, y1,
                                                 *args[-2:]))
        elif rows is not None:
            check(L.lib().mr_bp_parallel_rows(proj.data_ptr(), nproj, *args[:-2], int(rows[0]), int(rows[1]),
                                              *args[-2:]))
        elif self.staging:
            check(L.lib().mr_bp_parallel_staged(proj.data_ptr(), nproj, *args))
        else:
            check(L.lib().mr_bp_parallel(proj.data_ptr(), *args))
        return 0

    def GetSlice(self, idx: int) -> torch.Tensor:
        """BackProjectorModuleBase::GetSlice for MatrixZXY (BackProjectorModuleBase.cpp:62-128):
        slice[y][x] = volume[y0 + y][x0 + x][idx] over the slice window (the whole slice, or
        the matrix ROI's inclusive crop)."""
        if idx >= self.volume.shape[2]:
            raise ReconException(f"Slice index greater than matrix size (ZXY matrix). Slice index is {idx} and "
                                 f"Matrix Sixe is: {self.volume.shape[2]}")
        x0, y0, w, h = self._slice_window(self.volume.shape[1], self.volume.shape[0])
        return self.volume[y0:y0 + h, x0:x0 + w, idx].contiguous()

    def GetNSlices(self) -> int:
        return self.volume.shape[2]


@_module
class MultiProjectionBP(MultiProjectionBPparallel):
    """MultiProjectionBP, the reference's serial backprojector (factory name "MultiProjBP",
    StdBackProjectors/src/MultiProjBP.cpp:36-146). Without tilt correction it computes exactly
    what MultiProjectionBPparallel computes (the same positions, weights and accumulation order,
    pinned against the compiled reference). With tilt correction it subtracts the centre offset
    after the x term and shifts the interpolation weight by one `4 tan(tilt)` per group of 4
    slices (MultiProjBP.cpp:61-84), where the parallel one shifts it twice
    (MultiProjBPparallel.cpp:88-99): mr_bp_parallel_variant(MR_BP_MULTIPROJ_SERIAL)."""

    _variant = L.MR_BP_MULTIPROJ_SERIAL

    def __init__(self):
        super().__init__()
        self.m_sModuleName = "Multi projection BP"


@_module
class NearestNeighborBP(MultiProjectionBPparallel):
    """NearestNeighborBP (factory name "NNMultiProjBP", StdBackProjectors/src/NNMultiProjBP.cpp:
    36-121): the same positions as MultiProjectionBP, each voxel adding the one sample at the
    truncated detector position (no interpolation); with tilt correction the centre offset is
    subtracted after the x term and there is no per-slice shift
    (mr_bp_parallel_variant(MR_BP_NEAREST))."""

    _variant = L.MR_BP_NEAREST

    def __init__(self):
        super().__init__()
        self.m_sModuleName = "NearestNeighborBP"


@_module
class FDKbp_single(_BackProjectorBase):
    """FDKbp_single (FDKBackProjectors/src/fdkbp_single.cpp) with the FdkReconBase driver
    (fdkreconbase.cpp). Volume is MatrixXYZ: tensor (nz, ny, nx) = (nv, nu, nu), x fastest."""

    def __init__(self):
        super().__init__("FDKbp_single")
        self._first = True
        self.staging = True  # TMA-staged footprints (False: direct global loads; same results)

    def SetROI(self, roi) -> None:
        self._roi = tuple(int(v) for v in roi)
        if self._roi[0] != 0 or self._roi[1] != 0:
            raise ReconException("FDKbp_single: only a full-detector ROI starting at (0, 0) is supported")
        self.SizeU = self._roi[2] - self._roi[0]
        self.SizeV = self._roi[3] - self._roi[1]
        pi = self.mConfig.ProjectionInfo
        dev = torch.device("cuda", torch.cuda.current_device())
        self.volume = torch.zeros((self.SizeV, self.SizeU, self.SizeU), dtype=torch.float32, device=dev)
        mask = np.zeros(2 * self.SizeU, np.uint32)
        nslices = int(pi.nDims[1]) if pi.nDims[1] else self.SizeV
        check(L.lib().mr_bp_circle_mask(self.SizeU, self.SizeU, int(pi.bCorrectTilt), float(pi.fTiltAngle), nslices,
                                        mask.ctypes.data_as(L.P_u32)))
        _restrict_mask(mask, self.SizeU, self.mConfig.MatrixInfo, cone=True)
        self._mask = torch.from_numpy(mask.view(np.int32)).to(dev)
        self._first = True
        self._geo_key = None

    def geometry(self) -> L.FdkGeom:
        pi, mi = self.mConfig.ProjectionInfo, self.mConfig.MatrixInfo
        g = L.FdkGeom()
        g.sod, g.sdd = pi.fSOD, pi.fSDD
        g.ppoint[0], g.ppoint[1] = pi.fpPoint
        g.center = pi.fCenter
        g.resolution[0], g.resolution[1] = pi.fResolution
        g.voxelsize[0], g.voxelsize[1], g.voxelsize[2] = mi.fVoxelSize
        g.direction = int(pi.eDirection)
        g.correcttilt = int(pi.bCorrectTilt)
        g.tiltangle = pi.fTiltAngle
        g.tiltpivot = pi.fTiltPivotPosition
        return g

    def partials(self, angles: np.ndarray):
        nu, nv, n = self.SizeU, self.SizeV, angles.size
        xip = np.empty((n, nu, 3), np.float32)
        yip = np.empty((n, nu, 3), np.float32)
        zip_ = np.empty((n, nv, 3), np.float32)
        s2, sc, uni = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        g = self.geometry()
        a = np.ascontiguousarray(angles, np.float32)
        check(L.lib().mr_fdk_partials(ctypes.byref(g), nu, nv, a.ctypes.data_as(L.P_float), n,
                                      xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                                      zip_.ctypes.data_as(L.P_float), ctypes.byref(s2), ctypes.byref(sc),
                                      ctypes.byref(uni)))
        return xip, yip, zip_, s2.value, sc.value, uni.value

    def maps64(self, angles: np.ndarray) -> np.ndarray:
        """FP64 per-projection detector maps (nproj, 12) (mr_fdk_maps64)."""
        a = np.ascontiguousarray(angles, np.float32)
        m = np.zeros((a.size, 12), np.float64)
        g = self.geometry()
        check(L.lib().mr_fdk_maps64(ctypes.byref(g), self.SizeU, self.SizeV, a.ctypes.data_as(L.P_float), a.size,
                                    m.ctypes.data_as(L.P_double)))
        return m

    def Process(self, projections: torch.Tensor, parameters: dict) -> int:
        if self.volume is None:
            raise ReconException("The target matrix is not allocated.")
        _require_cuda(projections, "projections")
        if projections.dtype != torch.float32:
            raise ReconException("FDKbp_single expects float32 projections")
        nproj, nv, nu = projections.shape
        if nu != self.SizeU or nv != self.SizeV:
            raise ReconException(f"Projection size ({nu}, {nv}) does not match the ROI ({self.SizeU}, {self.SizeV})")
        weights = _float_vector(_get(parameters, "weights"), nproj)
        angles = _float_vector(_get(parameters, "angles"), nproj)
        geo = self.prepare(angles, weights, projections.device)
        filt, scale = self.ramp_filter(projections, geo, *self._filter_out(projections))
        self.backproject(filt, scale, geo)
        self._first = False
        return 0

    def _filter_out(self, projections: torch.Tensor):
        """(first, out, scale) for ramp_filter: the filtered projections' buffer and the 16-bit
        path's per-projection scales, kept between calls of the same shape and precision (a
        block of projections is several GB: no allocation per call)."""
        dtype = torch.float32 if _PRECISION[self.precision] == L.MR_F32 else torch.uint16
        buf = getattr(self, "_filt_buf", None)
        if buf is None or buf.shape != projections.shape or buf.dtype != dtype or buf.device != projections.device:
            self._filt_buf = self._filt_scale = None  # release the old buffers first
            self._filt_buf = torch.empty(projections.shape, dtype=dtype, device=projections.device)
            self._filt_scale = None if dtype == torch.float32 else \
                torch.empty(projections.shape[0], dtype=torch.float32, device=projections.device)
        return 0, self._filt_buf, self._filt_scale

    def prepare(self, angles: np.ndarray, weights: np.ndarray, dev):
        """Per-projection geometry (partials or FP64 maps, staging box, filter weights) on the
        device; it depends only on the configuration and the angles, so it is kept while they
        stay the same."""
        nu, nv, nproj = self.SizeU, self.SizeV, angles.size
        dtype = _PRECISION[self.precision]
        key = (angles.tobytes(), weights.tobytes(), str(dev), dtype)
        if getattr(self, "_geo_key", None) != key:
            xip, yip, zip_, s2, sc, uni = self.partials(angles)
            bw, bh = ctypes.c_int(0), ctypes.c_int(0)
            maps = None
            if uni and dtype != L.MR_F32:
                # precision form: FP64 detector maps (the kernel forms each tile origin in FP64)
                m64 = self.maps64(angles)
                check(L.lib().mr_fdk_box_maps(m64.ctypes.data_as(L.P_double), nu, nv, nproj, dtype, ctypes.byref(bw),
                                              ctypes.byref(bh)))
                maps = torch.from_numpy(m64).to(dev)
            elif uni:
                check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                                         zip_.ctypes.data_as(L.P_float), nu, nv, nproj, dtype,
                                         ctypes.byref(bw), ctypes.byref(bh)))
            self._geo = (torch.from_numpy(weights).to(dev), *(torch.from_numpy(a).to(dev) for a in (xip, yip, zip_)),
                         s2, sc, uni, (bw.value, bh.value), maps)
            self._geo_key = key
        return self._geo

    def ramp_filter(self, projections: torch.Tensor, geo, first: int = 0, out=None, scale=None):
        """FDK ramp filter (mr_fdk_filter) of projections, which are projections first,
        first+1, ... of the geometry; returns (filtered, per-projection scale or None)."""
        w, X, Y, Z, s2, sc, uni, box, maps = geo
        nproj, nv, nu = projections.shape
        dtype = _PRECISION[self.precision]
        if out is None:
            out = torch.empty_like(projections) if dtype == L.MR_F32 else \
                torch.empty(projections.shape, dtype=torch.uint16, device=projections.device)
            scale = None if dtype == L.MR_F32 else torch.empty(nproj, dtype=torch.float32, device=projections.device)
        check(L.lib().mr_fdk_filter(projections.data_ptr(), nu, nv, nproj, w[first:].data_ptr(), s2, sc, dtype,
                                    out.data_ptr(), _ptr(scale), _stream()))
        return out, scale

    def backproject(self, filt: torch.Tensor, scale, geo, k_range=None, first: int = 0,
                    accumulate: bool | None = None) -> None:
        """Backprojection of filtered projections into the volume (overwriting it for the first
        batch of projections, adding afterwards, unless `accumulate` says otherwise); filt
        holds projections first, first+1, ... of the geometry; k_range = (k_begin, k_end)
        restricts it to those cbct slices (final volume slices nv-1-k), FP32 only."""
        w, X, Y, Z, s2, sc, uni, box, maps = geo
        nproj, nv, nu = filt.shape
        acc = int(not self._first) if accumulate is None else int(accumulate)
        X, Y, Z = X[first:first + nproj], Y[first:first + nproj], Z[first:first + nproj]
        dtype = _PRECISION[self.precision]
        st = _stream()
        box = box if self.staging else (0, 0)
        if maps is not None and box[0] > 0 and nu % 8 == 0:
            if k_range is not None:
                raise ReconException("FDKbp_single: slice ranges are supported in FP32 only")
            check(L.lib().mr_fdk_backproject_fast(filt.data_ptr(), dtype, scale.data_ptr(), nu, nv, nproj,
                                                  maps[first:first + nproj].data_ptr(), self._mask.data_ptr(), box[0],
                                                  box[1], acc, self.volume.data_ptr(), st))
        else:
            kb, ke = k_range if k_range is not None else (0, nv)
            check(L.lib().mr_fdk_backproject_slab(filt.data_ptr(), dtype, _ptr(scale), nu, nv, nproj, X.data_ptr(),
                                                  Y.data_ptr(), Z.data_ptr(), uni, self._mask.data_ptr(),
                                                  box[0] if maps is None else 0, box[1] if maps is None else 0,
                                                  acc, kb, ke, self.volume.data_ptr(), st))

    def GetSlice(self, idx: int) -> torch.Tensor:
        """BackProjectorModuleBase::GetSlice for MatrixXYZ (BackProjectorModuleBase.cpp:62-128):
        slice[y][x] = volume[idx][y0 + y][x0 + x] over the slice window."""
        if idx >= self.volume.shape[0]:
            raise ReconException(f"Slice index greater than matrix size (XYZ matrix). Slice index is {idx} and "
                                 f"Matrix Sixe is: {self.volume.shape[0]}")
        x0, y0, w, h = self._slice_window(self.volume.shape[2], self.volume.shape[1])
        return self.volume[idx, y0:y0 + h, x0:x0 + w].contiguous()

    def GetNSlices(self) -> int:
        return self.volume.shape[0]


def quantize(proj: torch.Tensor, precision: str):
    """Per-projection power-of-two scaled 16-bit copy (mr_quantize) of float projections
    (nproj, nv, nu). Returns (bits as uint16 tensor, scales)."""
    _require_cuda(proj, "projections")
    nproj = proj.shape[0]
    per = proj[0].numel()
    out = torch.empty(proj.shape, dtype=torch.uint16, device=proj.device)
    scale = torch.empty(nproj, dtype=torch.float32, device=proj.device)
    check(L.lib().mr_quantize(proj.data_ptr(), per, nproj, _PRECISION[precision], out.data_ptr(), scale.data_ptr(),
                              _stream()))
    return out, scale


# ------------------------------------------------------------------- slice serialisation


def slices_u16(volume: torch.Tensor, matrix_alignment: str, gray_interval, first: int = 0, count: int | None = None,
               roi=None) -> torch.Tensor:
    """The uint16 slices ReconEngine::Serialize writes as TIFF16 (ReconEngine.cpp:576-700 ->
    kipl::io::WriteImageStack), cast on the device (mr_slices_u16): ``volume`` is a
    backprojector's volume tensor, ``matrix_alignment`` "MatrixXYZ" (FDK, tensor (nz, ny, nx),
    slices along z, plane XY) or "MatrixZXY" (parallel beam, tensor (ny, nx, nz), slices
    along z, plane YZ); ``gray_interval`` = MatrixInfo.fGrayInterval (lo, hi); ``roi`` =
    MatrixInfo.roi (x0, y0, x1, y1, inclusive) or None. Returns (count, h, w) uint16."""
    _require_cuda(volume, "volume")
    if volume.dtype != torch.float32 or volume.dim() != 3 or not volume.is_contiguous():
        raise ReconException("slices_u16: volume must be a contiguous float32 3-D tensor")
    if matrix_alignment == "MatrixXYZ":
        plane = L.MR_PLANE_XY
        nz, ny, nx = volume.shape
        d0, d1, d2, nslices, na, nb = nx, ny, nz, nz, nx, ny
    elif matrix_alignment == "MatrixZXY":
        plane = L.MR_PLANE_YZ
        ny, nx, nz = volume.shape
        d0, d1, d2, nslices, na, nb = nz, nx, ny, nz, nx, ny
    else:
        raise ReconException(f"slices_u16: unknown matrix alignment {matrix_alignment}")
    count = nslices - first if count is None else count
    if roi is None:
        w, h, r = na, nb, None
    else:
        x0, x1 = sorted((int(roi[0]), int(roi[2])))
        y0, y1 = sorted((int(roi[1]), int(roi[3])))
        w, h = x1 - x0 + 1, y1 - y0 + 1
        r = (ctypes.c_size_t * 4)(*[int(v) for v in roi])
    out = torch.empty((max(count, 0), h, w), dtype=torch.uint16, device=volume.device)
    check(L.lib().mr_slices_u16(volume.data_ptr(), plane, d0, d1, d2, first, count, r, float(gray_interval[0]),
                                float(gray_interval[1]), out.data_ptr(), _stream()))
    return out
