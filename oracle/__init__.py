"""Python access to the oracles (test infrastructure only).

Two CPU libraries check the CUDA path:

* ``liboracle.so`` - the C restatement of the reference algorithms (``mr_oracle.c``);
* ``_ref/libmuhrec_ref.so`` - the reference's own modules compiled from source by
  ``ref/Makefile`` (present wherever the reference tree was available at build time;
  the built file travels with the repository snapshot).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this package. The product library never loads either file.

Array convention: projections are numpy ``float32`` arrays of shape ``(nproj, nv, nu)``
(kipl ``TImage<float,3>`` order, u fastest).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_SZ = ctypes.POINTER(ctypes.c_size_t)
_sz = ctypes.c_size_t
_f = ctypes.c_float

FILTERS = {"ram-lak": 0, "shepp-logan": 1, "hanning": 2, "hamming": 3, "butterworth": 4}
AVERAGE = {"ImageSum": 0, "ImageAverage": 1, "ImageMedian": 2, "ImageWeightedAverage": 3, "ImageMin": 4, "ImageMax": 5}


def _p(a: np.ndarray, t=_F):
    return a.ctypes.data_as(t)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


_orc = None
_ref = None


def orc() -> ctypes.CDLL:
    """The C restatement library (raises if it was not built)."""
    global _orc
    if _orc is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        lib = ctypes.CDLL(path)
        lib.orc_frame_dose.restype = ctypes.c_float
        lib.orc_projfilter_size.restype = ctypes.c_size_t
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libmuhrec_ref.so"))


def ref() -> ctypes.CDLL:
    """The reference modules compiled from source (raises if absent)."""
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libmuhrec_ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle missing: {path} (run make -C oracle ref)")
        lib = ctypes.CDLL(path)
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_frame_dose.restype = ctypes.c_float
        lib.ref_quiet_logging()
        _ref = lib
    return _ref


def _check_ref(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("reference module failed: " + ref().ref_last_error().decode(errors="replace"))


# ----------------------------------------------------------------- averaging / dose


def average(stack, method: str = "ImageAverage", use_ref: bool = False) -> np.ndarray:
    stack = _f32(stack)
    n, nv, nu = stack.shape
    out = np.empty((nv, nu), np.float32)
    if use_ref:
        _check_ref(ref().ref_average(_p(stack), _sz(nu), _sz(nv), _sz(n), AVERAGE[method], _p(out)))
    else:
        if orc().orc_average(_p(stack), _sz(nu), _sz(nv), _sz(n), AVERAGE[method], _p(out)) != 0:
            raise ValueError(f"average method {method} not restated")
    return out


def frame_dose(frame, roi) -> float:
    frame = _f32(frame)
    r = np.ascontiguousarray(roi, dtype=np.uint64).astype(np.uintp)
    return float(orc().orc_frame_dose(_p(frame), _sz(frame.shape[-1]), _p(r, _SZ)))


# ----------------------------------------------------------------------- FullLogNorm


@dataclass
class LogNormRefs:
    dark: np.ndarray
    logflat: np.ndarray
    darkdose: float
    flatdose: float


def lognorm_refs(darks, flats, method="ImageAverage", usenormregion=False, dose_roi=(0, 0, 0, 0)) -> LogNormRefs:
    """NormBase::ReferenceLoader + FullLogNorm::SetReferenceImages (NormPlugins.cpp:91-341)."""
    darks, flats = _f32(darks), _f32(flats)
    nd, nf = darks.shape[0], flats.shape[0]
    nv, nu = flats.shape[1:]
    dark = average(darks, method) if nd else np.zeros((nv, nu), np.float32)
    darkdose = np.float32(0.0)
    if nd:
        acc = np.float32(0.0)
        for i in range(nd):
            t = np.float32(frame_dose(darks[i], dose_roi)) if usenormregion else np.float32(0.0)
            acc = t if i == 0 else np.float32(acc + t)
        darkdose = np.float32(acc / np.float32(nd))
    flatdose = np.float32(1.0)
    flat = average(flats, method) if nf else np.zeros((nv, nu), np.float32)
    if nf:
        acc = np.float32(0.0)
        for i in range(nf):
            t = (np.float32(frame_dose(flats[i], dose_roi)) if usenormregion else np.float32(1.0)) - darkdose
            t = np.float32(t)
            acc = t if i == 0 else np.float32(acc + t)
        flatdose = np.float32(acc / np.float32(nf))
    logflat = np.empty_like(flat)
    orc().orc_lognorm_logflat(_p(dark), _p(flat), _sz(flat.size), int(nd > 0), _f(flatdose), _p(logflat))
    return LogNormRefs(dark, logflat, float(darkdose), float(flatdose))


def lognorm_doselog(doses, darkdose: float) -> np.ndarray:
    doses = _f32(doses)
    out = np.empty_like(doses)
    orc().orc_lognorm_doselog(_p(doses), _sz(doses.size), _f(darkdose), _p(out))
    return out


def lognorm_apply(proj, dark, logflat, doselog, ndc=True, nob=True, uselut=False) -> np.ndarray:
    """FullLogNorm::ProcessCore 3D (NormPlugins.cpp:411-552) on float projections; uselut
    selects the LogLUT path."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    dark, logflat, doselog = _f32(dark), _f32(logflat), _f32(doselog)
    nproj = out.shape[0]
    npix = out[0].size
    fn = orc().orc_lognorm_apply_lut if uselut else orc().orc_lognorm_apply
    fn(_p(out), _sz(npix), _sz(nproj), _p(dark), _p(logflat), _p(doselog), _sz(doselog.size), int(ndc), int(nob))
    return out


def log_lut():
    """FullLogNorm's LogLUT(1 << 16, 0, 65535): (table, (lo, hi, slope, intercept))."""
    lut = np.empty(1 << 16, np.float32)
    param = np.empty(4, np.float32)
    orc().orc_log_lut(_p(lut), _p(param))
    return lut, param


def ref_fulllognorm(proj, darks, flats, method="ImageAverage", usenormregion=False, dose_roi=(0, 0, 0, 0),
                    uselut=False):
    """The reference FullLogNorm module on float projections. Returns (out, dark, logflat, doses, (dd, fd))."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    darks, flats = _f32(darks), _f32(flats)
    nproj, nv, nu = out.shape
    dark = np.zeros((nv, nu), np.float32)
    logflat = np.zeros((nv, nu), np.float32)
    doses = np.zeros(nproj, np.float32)
    rd = np.zeros(2, np.float32)
    roi = np.asarray(dose_roi, dtype=np.uintp)
    _check_ref(ref().ref_fulllognorm(_p(out), _sz(nu), _sz(nv), _sz(nproj), _p(darks), _sz(darks.shape[0]),
                                     _p(flats), _sz(flats.shape[0]), AVERAGE[method], int(usenormregion),
                                     _p(roi, _SZ), _p(dark), _p(logflat), _p(doses), _p(rd), int(uselut)))
    return out, dark, logflat, doses, (float(rd[0]), float(rd[1]))


# --------------------------------------------------------------------- ProjectionFilter


@dataclass
class FilterPlan:
    nu: int
    nfft: int
    ninsert: int
    filter: np.ndarray
    pad: np.ndarray


def projfilter_plan(nu, filtertype="hanning", cutoff=0.5, order=1.0, usebias=True, biasweight=0.1,
                    paddingdoubler=2) -> FilterPlan:
    nfft = int(orc().orc_projfilter_size(_sz(nu), int(paddingdoubler)))
    filt = np.zeros(nfft // 2, np.float32)
    pad = np.zeros(nfft, np.float32)
    ins = _sz(0)
    rc = orc().orc_projfilter_build(_sz(nu), FILTERS[filtertype.lower()], _f(cutoff), _f(order), int(usebias),
                                    _f(biasweight), int(paddingdoubler), _p(filt), _p(pad), ctypes.byref(ins))
    if rc != 0:
        raise ValueError("Cut off frequency is not in valid range")
    return FilterPlan(nu, nfft, ins.value, filt, pad[: ins.value].copy())


def projfilter(proj, plan: FilterPlan) -> np.ndarray:
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    rows = out.size // plan.nu
    orc().orc_projfilter_apply(_p(out), _sz(plan.nu), _sz(rows), _p(plan.filter), _p(plan.pad),
                               _sz(plan.nfft), _sz(plan.ninsert))
    return out


def ref_projfilter(proj, filtertype="hanning", cutoff=0.5, order=1.0, usebias=True, biasweight=0.1,
                   paddingdoubler=2):
    """The reference ProjectionFilterSingle module. Returns (out, filter, nfft)."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    nproj, nv, nu = out.shape
    nfft = int(orc().orc_projfilter_size(_sz(nu), int(paddingdoubler)))
    filt = np.zeros(nfft // 2, np.float32)
    n = _sz(0)
    _check_ref(ref().ref_projfilter(_p(out), _sz(nu), _sz(nv), _sz(nproj), filtertype.encode(), _f(cutoff),
                                    _f(order), int(usebias), _f(biasweight), int(paddingdoubler), _p(filt),
                                    ctypes.byref(n)))
    return out, filt, n.value


# ---------------------------------------------------------------------- parallel BP


def bp_parallel(proj, angles, weights, center, direction=0, buffersize=16, correcttilt=False, tiltangle=0.0,
                tiltpivot=0.0, roi_y0=0, nslices=None, use_ref=False, serial=False, nn=False) -> np.ndarray:
    """MultiProjectionBPparallel through StdBackProjectorBase::Process 3D (serial: the serial
    MultiProjectionBP; nn: NearestNeighborBP).

    Returns the ZXY volume, shape (nu [y], nu [x], nv [z])."""
    proj = _f32(proj)
    nproj, nv, nu = proj.shape
    angles, weights = _f32(angles), _f32(weights)
    vol = np.zeros((nu, nu, nv), np.float32)
    if use_ref:
        _check_ref(ref().ref_bp_parallel(_p(proj), _sz(nu), _sz(nv), _sz(nproj), _p(angles), _p(weights), _f(center),
                                         int(direction), _sz(buffersize), int(correcttilt), _f(tiltangle),
                                         _f(tiltpivot), _sz(roi_y0), 2 if nn else int(serial), _p(vol)))
    else:
        rc = orc().orc_bp_parallel_variant(_p(proj), _sz(nu), _sz(nv), _sz(nproj), _p(angles), _p(weights),
                                           _f(center), int(direction), _sz(buffersize), int(correcttilt),
                                           _f(tiltangle), _f(tiltpivot), _sz(roi_y0),
                                           _sz(nslices if nslices is not None else nv), 2 if nn else int(serial),
                                           _p(vol))
        if rc != 0:
            raise ValueError("invalid parallel-beam backprojection arguments")
    return vol


# ---------------------------------------------------------------------------- FDK


class FdkGeom(ctypes.Structure):
    _fields_ = [("sod", ctypes.c_float), ("sdd", ctypes.c_float), ("ppoint", ctypes.c_float * 2),
                ("center", ctypes.c_float), ("resolution", ctypes.c_float * 2), ("voxelsize", ctypes.c_float * 3),
                ("direction", ctypes.c_int), ("correcttilt", ctypes.c_int), ("tiltangle", ctypes.c_float),
                ("tiltpivot", ctypes.c_float)]


def fdk_geom(sod, sdd, ppoint, center, resolution, voxelsize, direction=0, correcttilt=False, tiltangle=0.0,
             tiltpivot=0.0) -> FdkGeom:
    g = FdkGeom()
    g.sod, g.sdd = sod, sdd
    g.ppoint[0], g.ppoint[1] = ppoint
    g.center = center
    g.resolution[0], g.resolution[1] = resolution
    g.voxelsize[0], g.voxelsize[1], g.voxelsize[2] = voxelsize
    g.direction = int(direction)
    g.correcttilt = int(correcttilt)
    g.tiltangle = tiltangle
    g.tiltpivot = tiltpivot
    return g


def fdk(proj, angles, weights, geom: FdkGeom, use_ref=False) -> np.ndarray:
    """FDKbp_single through FdkReconBase::Process 3D. Returns the XYZ volume (nv, nu, nu)."""
    proj = _f32(proj)
    nproj, nv, nu = proj.shape
    angles, weights = _f32(angles), _f32(weights)
    if use_ref:
        vol = np.empty((nv, nu, nu), np.float32)  # the harness copies the whole volume out
        _check_ref(ref().ref_fdk(_p(proj), _sz(nu), _sz(nv), _sz(nproj), _p(angles), _p(weights),
                                 ctypes.byref(geom), _p(vol), None))
    else:
        vol = np.zeros((nv, nu, nu), np.float32)
        orc().orc_fdk(_p(proj), _sz(nu), _sz(nv), _sz(nproj), _p(angles), _p(weights), ctypes.byref(geom), _p(vol))
    return vol


def ref_getslice(vol, zxy: bool, idx: int, roi=None) -> np.ndarray:
    """The reference BackProjectorModuleBase::GetSlice on `vol` (numpy, C order: (ny, nx, nz)
    for MatrixZXY, (nz, ny, nx) for MatrixXYZ); roi = MatrixInfo.roi with bUseROI, or None."""
    vol = _f32(vol)
    d2, d1, d0 = vol.shape
    out = np.empty(vol.size, np.float32)
    dims = np.zeros(2, np.uintp)
    r = np.asarray(roi if roi is not None else (0, 0, 0, 0), dtype=np.uintp)
    _check_ref(ref().ref_getslice(_p(vol), _sz(d0), _sz(d1), _sz(d2), int(zxy), int(roi is not None), _p(r, _SZ),
                                  _sz(idx), _p(out), _p(dims, _SZ)))
    return out[: int(dims[0]) * int(dims[1])].reshape(int(dims[1]), int(dims[0]))


# ------------------------------------------------------ module libraries (plugin loading)


def _lines(d: dict | None) -> bytes:
    return "".join(f"{k}={v}\n" for k, v in (d or {}).items()).encode()


def _parse_module_lines(text: str) -> dict:
    out: dict = {}
    for ln in text.splitlines():
        if "|" in ln:
            mod, kv = ln.split("|", 1)
            k, v = kv.split("=", 1)
            out.setdefault(mod, {})[k] = v
    return out


def ref_plugin_module_list(sofile: str, application: str) -> tuple[int, dict]:
    """GetModuleList of a module library, called as ReconEngine's module configuration does."""
    buf = ctypes.create_string_buffer(1 << 16)
    _check_ref(ref().ref_plugin_module_list(sofile.encode(), application.encode(), buf, _sz(len(buf))))
    text = buf.value.decode()
    return int(text.splitlines()[0].split("=")[1]), _parse_module_lines(text)


def ref_plugin_has_module(sofile: str, application: str, name: str) -> bool:
    found = ctypes.c_int(-1)
    _check_ref(ref().ref_plugin_has_module(sofile.encode(), application.encode(), name.encode(), ctypes.byref(found)))
    return bool(found.value)


def ref_module_parameters(name: str, backprojector: bool = False) -> dict:
    """GetParameters of the reference's own module of that name (its defaults)."""
    buf = ctypes.create_string_buffer(1 << 14)
    _check_ref(ref().ref_module_parameters(name.encode(), int(backprojector), buf, _sz(len(buf))))
    return _parse_module_lines(buf.value.decode()).get(name, {})


def ref_write_mat(img, fname: str) -> None:
    img = _f32(img)
    _check_ref(ref().ref_write_mat(_p(img), _sz(img.shape[1]), _sz(img.shape[0]), fname.encode()))


def ref_preproc_module(proj, name: str, params: dict, sofile: str | None = None, coeff: dict | None = None,
                       refpath: str = "", obmask: str = "", nob: int = 0, obfirst: int = 1, dcmask: str = "",
                       ndc: int = 0, dcfirst: int = 1, dose_roi=None, roi=None) -> np.ndarray:
    """Configure (+ SetROI when roi is given) + Process 3D of a preprocessing module on a copy of
    proj: the reference's own module (sofile None) or module `name` of the library `sofile`
    loaded through the reference's ModuleItem."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    nproj, nv, nu = out.shape
    dr = None if dose_roi is None else np.asarray(dose_roi, np.uintp)
    r = None if roi is None else np.asarray(roi, np.uintp)
    _check_ref(ref().ref_preproc_module(sofile.encode() if sofile else None, name.encode(), _lines(params),
                                        _lines(coeff), refpath.encode(), obmask.encode(), _sz(nob), _sz(obfirst),
                                        dcmask.encode(), _sz(ndc), _sz(dcfirst),
                                        None if dr is None else _p(dr, _SZ), None if r is None else _p(r, _SZ),
                                        _p(out), _sz(nu), _sz(nv), _sz(nproj)))
    return out


class RefBpConfig(ctypes.Structure):
    _fields_ = [("center", ctypes.c_float), ("direction", ctypes.c_int), ("correcttilt", ctypes.c_int),
                ("tiltangle", ctypes.c_float), ("tiltpivot", ctypes.c_float), ("cone", ctypes.c_int),
                ("sod", ctypes.c_float), ("sdd", ctypes.c_float), ("ppoint", ctypes.c_float * 2),
                ("resolution", ctypes.c_float * 2), ("voxelsize", ctypes.c_float * 3),
                ("use_matrix_roi", ctypes.c_int), ("matrix_roi", ctypes.c_size_t * 4)]


def ref_bp_module(proj, angles, weights, name: str, cfg: RefBpConfig, roi, params: dict,
                  sofile: str | None = None):
    """Configure + SetROI + Process 3D of a backprojector (the reference's own, or `name` of the
    library `sofile` through BackProjItem); returns (volume in kipl order as a numpy array of
    the module's matrix alignment, GetSlice of every slice as (nslices, h, w))."""
    proj = _f32(proj)
    nproj, nv, nu = proj.shape
    a, w = _f32(angles), _f32(weights)
    vol = np.empty(nu * nu * nv, np.float32)
    slices = np.empty(nu * nu * nv, np.float32)
    dims = np.zeros(3, np.uintp)
    r = np.asarray(roi, np.uintp)
    _check_ref(ref().ref_bp_module(sofile.encode() if sofile else None, name.encode(), _lines(params),
                                   ctypes.byref(cfg), _p(r, _SZ), _p(proj), _sz(nproj), _p(a), _p(w), _p(vol),
                                   _p(slices), _p(dims, _SZ)))
    sw, sh, ns = (int(d) for d in dims)
    return vol, slices[: ns * sw * sh].reshape(ns, sh, sw)


class RefFdkSession:
    """The reference FDKbp_single configured once (Configure + SetROI for the full detector)
    and then given projections by repeated Process 3D calls, each adding into the same volume
    (the way ReconEngine keeps one backprojector per slice block). Times the reference per
    projection without its per-block set-up."""

    def __init__(self, nu, nv, nproj_total, geom: FdkGeom):
        lib = ref()
        lib.ref_fdk_session_create.restype = ctypes.c_void_p
        lib.ref_fdk_session_process.argtypes = [ctypes.c_void_p, _F, _sz, _F, _F]
        lib.ref_fdk_session_volume.argtypes = [ctypes.c_void_p, _F]
        lib.ref_fdk_session_destroy.argtypes = [ctypes.c_void_p]
        self.nu, self.nv = nu, nv
        self.h = lib.ref_fdk_session_create(_sz(nu), _sz(nv), _sz(nproj_total), ctypes.byref(geom))
        if not self.h:
            raise RuntimeError("reference module failed: " + lib.ref_last_error().decode(errors="replace"))

    def process(self, proj, angles, weights) -> None:
        proj = _f32(proj)
        assert proj.shape[1:] == (self.nv, self.nu)
        a, w = _f32(angles), _f32(weights)
        _check_ref(ref().ref_fdk_session_process(self.h, _p(proj), _sz(proj.shape[0]), _p(a), _p(w)))

    def volume(self) -> np.ndarray:
        vol = np.empty((self.nv, self.nu, self.nu), np.float32)
        _check_ref(ref().ref_fdk_session_volume(self.h, _p(vol)))
        return vol

    def close(self) -> None:
        if self.h:
            ref().ref_fdk_session_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def fdk_ramp(img) -> np.ndarray:
    out = np.array(img, dtype=np.float32, copy=True, order="C")
    h, w = out.shape
    orc().orc_fdk_ramp(_p(out), _sz(w), _sz(h))
    return out


def fdk_projmatrix(geom: FdkGeom, nu: int, angle: float) -> np.ndarray:
    pm = np.zeros(12, np.float32)
    orc().orc_fdk_projmatrix(ctypes.byref(geom), _sz(nu), _f(angle), _p(pm))
    return pm


def fdk_prepare(proj, weights, geom: FdkGeom) -> np.ndarray:
    """img *= weight, ramp filter, rescale - the per-projection preparation before FDK BP."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    nproj, nv, nu = out.shape
    w = _f32(weights)
    orc().orc_fdk_prepare(_p(out), _sz(nu), _sz(nv), _sz(nproj), _p(w), ctypes.byref(geom))
    return out


def fdk_bp(filtered, angles, geom: FdkGeom) -> np.ndarray:
    """FDK backprojection + final mirror of prepared projections. Returns (nv, nu, nu)."""
    filtered = _f32(filtered)
    nproj, nv, nu = filtered.shape
    a = _f32(angles)
    vol = np.zeros((nv, nu, nu), np.float32)
    orc().orc_fdk_bp(_p(filtered), _sz(nu), _sz(nv), _sz(nproj), _p(a), ctypes.byref(geom), _p(vol))
    return vol


def fdk_maps64(geom: FdkGeom, nu, nv, angles) -> np.ndarray:
    """FP64 detector maps (nproj, 12) of the FDK geometry (FDKbp's double geometry)."""
    a = _f32(angles)
    m = np.zeros((a.size, 12), np.float64)
    orc().orc_fdk_maps64(ctypes.byref(geom), _sz(nu), _sz(nv), _p(a), _sz(a.size), _p(m, ctypes.POINTER(ctypes.c_double)))
    return m


def fdk_bp64(filtered, maps, slices, mask=None) -> np.ndarray:
    """FP64 backprojection of FP32 filtered projections for output slices ``slices`` of the
    final volume. Returns (len(slices), nu, nu) float64."""
    filtered = _f32(filtered)
    nproj, nv, nu = filtered.shape
    maps = np.ascontiguousarray(maps, np.float64)
    sl = np.ascontiguousarray(slices, np.int32)
    m = np.ascontiguousarray(circle_mask(nu, nu) if mask is None else mask, np.uintp)
    out = np.zeros((sl.size, nu, nu), np.float64)
    orc().orc_fdk_bp64(_p(filtered), _sz(nu), _sz(nv), _sz(nproj), _p(maps, ctypes.POINTER(ctypes.c_double)), _p(m, _SZ),
                       _p(sl, ctypes.POINTER(ctypes.c_int)), _sz(sl.size), _p(out, ctypes.POINTER(ctypes.c_double)))
    return out


def bp_geometry(angles, nu, center, direction=0):
    a = _f32(angles)
    s, c, su = (np.empty_like(a) for _ in range(3))
    orc().orc_bp_geometry(_p(a), _sz(a.size), _sz(nu), _f(center), int(direction), _p(s), _p(c), _p(su))
    return s, c, su


def circle_mask(nx, ny, correcttilt=False, tiltangle=0.0, nslices=0) -> np.ndarray:
    m = np.zeros(2 * ny, np.uintp)
    orc().orc_circle_mask(_sz(nx), _sz(ny), int(correcttilt), _f(tiltangle), _sz(nslices), _p(m, _SZ))
    return m.astype(np.uint32)


# --------------------------------------------------------------------- MorphSpotClean

DETECT = {"holes": 0, "peaks": 1, "both": 2}


def morphspotclean(img, detect="holes", conn8=True, th=(0.1, 0.1), sigma=(0.01, 0.01), edge=9, clamp=False,
                   minlevel=-0.1, maxlevel=7.0, removeinfnan=False, use_ref=False) -> np.ndarray:
    """MorphSpotClean::process, MorphCleanReplace, on one image (nv, nu) or a stack (n, nv, nu)."""
    out = np.array(img, dtype=np.float32, copy=True, order="C")
    stack = out.reshape((-1,) + out.shape[-2:])
    t = np.asarray(th, np.float32)
    s = np.asarray(sigma, np.float32)
    h, w = stack.shape[1:]
    for im in stack:
        if use_ref:
            _check_ref(ref().ref_morphspotclean(_p(im), _sz(w), _sz(h), DETECT[detect], 0, int(conn8), _p(t), _p(s),
                                                int(edge), 100, int(clamp), _f(minlevel), _f(maxlevel),
                                                int(removeinfnan)))
        else:
            rc = orc().orc_morphspotclean(_p(im), _sz(w), _sz(h), DETECT[detect], int(conn8), _p(t), _p(s),
                                          _sz(edge), int(clamp), _f(minlevel), _f(maxlevel), int(removeinfnan))
            if rc != 0:
                raise RuntimeError("RecByDilation: f>g")
    return out


def ref_morphspotclean_module(proj, connectivity="conn4", detectionmethod="morphdetectpeaks", threshold="0.1 0.1",
                              sigma="0.01 0.01", edgesmooth=5, maxarea=30, removeinfnan=False, clampdata=False,
                              minlevel=-0.1, maxlevel=7.0, threading=False):
    """The reference MorphSpotCleanModule (morphcleanreplace) on a stack; threading selects its
    ProcessParallelStd path (one thread per projection, no clamp or inf/NaN removal)."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    nproj, nv, nu = out.shape
    _check_ref(ref().ref_morphspotclean_module(_p(out), _sz(nu), _sz(nv), _sz(nproj), connectivity.encode(),
                                               b"morphcleanreplace", detectionmethod.encode(), threshold.encode(),
                                               sigma.encode(), int(edgesmooth), int(maxarea), int(removeinfnan),
                                               int(clampdata), _f(minlevel), _f(maxlevel), int(threading)))
    return out


def fill_hole(img, conn8=True) -> np.ndarray:
    img = _f32(img)
    out = np.empty_like(img)
    orc().orc_fill_hole(_p(img), _sz(img.shape[1]), _sz(img.shape[0]), int(conn8), _p(out))
    return out


def fill_peaks(img, conn8=True) -> np.ndarray:
    img = _f32(img)
    out = np.empty_like(img)
    if orc().orc_fill_peaks(_p(img), _sz(img.shape[1]), _sz(img.shape[0]), int(conn8), _p(out)) != 0:
        raise RuntimeError("RecByDilation: f>g")
    return out


def fill_peaks_forward(img, conn8=True) -> np.ndarray:
    img = _f32(img)
    out = np.empty_like(img)
    orc().orc_fill_peaks_forward(_p(img), _sz(img.shape[1]), _sz(img.shape[0]), int(conn8), _p(out))
    return out


# ------------------------------------------------------------------------ StripeFilter

_DAUB = None


def daubechies(n: int) -> np.ndarray:
    """dbN scaling filter (float64) from the table of imagingsuite_b200/csrc/gen_daubechies.py
    (N <= 15 from the spectral factorisation, N >= 16 kipl's table values as float)."""
    global _DAUB
    if _DAUB is None:
        import re

        src = open(os.path.join(os.path.dirname(_HERE), "imagingsuite_b200", "csrc", "mr_daubechies.h")).read()
        _DAUB = [np.array([float(v) for v in row.split(",")]) for row in re.findall(r"\{([^{}]*)\},", src)]
    return _DAUB[n - 1]


def wavelet_kernel(name: str):
    """WaveletKernel<float>::CopyKernel (wavelets.hpp:387-405) for 'daubN': returns
    (begin, end, float32 array [4, K] = analysis H, analysis G, synthesis H, synthesis G).
    The reference's daub3 table has the sign of its fifth coefficient flipped; it is
    reproduced here."""
    if not name.startswith("daub"):
        raise ValueError(f"unsupported wavelet {name}")
    n = int(name[4:])
    if n == 28:
        raise ValueError("daub28: the reference's table is shorter than the filter (undefined kernel)")
    k = daubechies(n).copy()
    if n == 3:
        k[4] = -k[4]
    end = len(k) - 1
    tH = np.array([k[end - i] for i in range(len(k))])
    sgn = -1.0
    tG = np.empty_like(k)
    for i in range(len(k)):
        tG[i] = sgn * k[i]
        sgn = -sgn
    sH = k.copy()
    sG = np.array([tG[end - i] for i in range(len(k))])
    return 0, end, np.stack([tH, tG, sH, sG]).astype(np.float32)


def stripefilter(sino, wname="daub15", scale=2, sigma=0.05, use_ref=False) -> np.ndarray:
    """StripeFilter::process (VerticalComponentFFT) on one sinogram (ntheta, nu)."""
    out = np.array(sino, dtype=np.float32, copy=True, order="C")
    h, w = out.shape
    if use_ref:
        _check_ref(ref().ref_stripefilter(_p(out), _sz(w), _sz(h), wname.encode(), int(scale), _f(sigma), 1))
    else:
        b, e, k = wavelet_kernel(wname)
        k = np.ascontiguousarray(k)
        if orc().orc_stripefilter(_p(out), _sz(w), _sz(h), _p(k), b, e, int(scale), _f(sigma)) != 0:
            raise RuntimeError("Image smaller than wavelet kernel size")
    return out


def waveletringclean(proj, wname="daub15", decnum=2, sigma=0.05, use_ref=False) -> np.ndarray:
    """WaveletRingClean::ProcessSingle on projections (nproj, nv, nu): every detector row's
    sinogram through StripeFilter."""
    out = np.array(proj, dtype=np.float32, copy=True, order="C")
    nproj, nv, nu = out.shape
    if use_ref:
        _check_ref(ref().ref_waveletringclean(_p(out), _sz(nu), _sz(nv), _sz(nproj), wname.encode(), int(decnum),
                                              _f(sigma)))
        return out
    for j in range(nv):
        out[:, j, :] = stripefilter(out[:, j, :], wname, decnum, sigma)
    return out


# --------------------------------------------------------------------- Joseph projector pair

_DP = ctypes.POINTER(ctypes.c_double)


def joseph_forward64(vol, angles, nu, centre, tan_tilt=0.0, pivot=0.0, derivative=False):
    """FP64 Joseph forward projection of vol (nz, n, n); returns proj (nproj, nz, nu) and, with
    derivative=True, d proj / d centre."""
    vol = _f32(vol)
    nz, n, _ = vol.shape
    a = _f32(angles)
    proj = np.zeros((a.size, nz, nu), np.float64)
    d = np.zeros_like(proj) if derivative else None
    orc().orc_joseph_forward64(_p(vol), _sz(n), _sz(nz), _p(a), _sz(a.size), _sz(nu), ctypes.c_double(centre),
                               ctypes.c_double(tan_tilt), ctypes.c_double(pivot), _p(proj, _DP),
                               _p(d, _DP) if derivative else None)
    return (proj, d) if derivative else proj


def mbp_geometry(angles, n, nz, centre, tan_tilt=0.0, pivot=0.0, direction=0):
    """sin/cos [nproj][2] and per-slice start positions [nproj][nz] of the pair matched to the
    parallel-beam backprojector."""
    a = _f32(angles)
    sc = np.empty((a.size, 2), np.float32)
    su = np.empty((a.size, nz), np.float32)
    orc().orc_mbp_geometry(_p(a), _sz(a.size), _sz(n), _sz(nz), _f(centre), _f(tan_tilt), _f(pivot), int(direction),
                           _p(sc), _p(su))
    return sc, su


def mbp_adjoint(proj, angles, centre, tan_tilt=0.0, pivot=0.0, direction=0) -> np.ndarray:
    """The matched pair's backprojection (float, the reference's order). proj (nproj, nz, n);
    returns the volume (n [y], n [x], nz)."""
    proj = _f32(proj)
    nproj, nz, n = proj.shape
    sc, su = mbp_geometry(angles, n, nz, centre, tan_tilt, pivot, direction)
    m = np.ascontiguousarray(circle_mask(n, n), np.uintp)
    vol = np.empty((n, n, nz), np.float32)
    orc().orc_mbp_adjoint(_p(proj), _sz(n), _sz(nz), _p(sc), _p(su), _sz(nproj), _p(m, _SZ), _p(vol))
    return vol


def mbp_forward64(vol, angles, centre, tan_tilt=0.0, pivot=0.0, direction=0, float_u=True, derivative=False):
    """The matched pair's forward projection as the explicit transpose, FP64 accumulation.
    vol (n, n, nz) z fastest; returns proj (nproj, nz, n) [and d proj / d c_z]."""
    vol = _f32(vol)
    n, _, nz = vol.shape
    a = _f32(angles)
    m = np.ascontiguousarray(circle_mask(n, n), np.uintp)
    proj = np.empty((a.size, nz, n), np.float64)
    d = np.empty_like(proj) if derivative else None
    orc().orc_mbp_forward64(_p(vol), _sz(n), _sz(nz), _p(a), _sz(a.size), ctypes.c_double(centre),
                            ctypes.c_double(tan_tilt), ctypes.c_double(pivot), int(direction), _p(m, _SZ),
                            int(float_u), _p(proj, _D), None if d is None else _p(d, _D))
    return (proj, d) if derivative else proj


def joseph_adjoint64(proj, angles, n, centre, tan_tilt=0.0, pivot=0.0):
    """Exact transpose of joseph_forward64. proj (nproj, nz, nu) -> vol (nz, n, n) float64."""
    proj = np.ascontiguousarray(proj, np.float64)
    nproj, nz, nu = proj.shape
    a = _f32(angles)
    vol = np.zeros((nz, n, n), np.float64)
    orc().orc_joseph_adjoint64(_p(proj, _DP), _sz(n), _sz(nz), _p(a), _sz(nproj), _sz(nu), ctypes.c_double(centre),
                               ctypes.c_double(tan_tilt), ctypes.c_double(pivot), _p(vol, _DP))
    return vol


def ref_joseph_project(slice2d, angles) -> np.ndarray:
    """The reference LinearForwardProjector on one slice (n, n); returns (nangles, n)."""
    sl = _f32(slice2d)
    n = sl.shape[0]
    a = _f32(angles)
    out = np.zeros((a.size, n), np.float32)
    _check_ref(ref().ref_joseph_project(_p(sl), _sz(n), _p(a), _sz(a.size), _p(out)))
    return out



# ----------------------------------------------------------------- slice serialisation

_U16 = ctypes.POINTER(ctypes.c_uint16)


def _slices_args(vol, plane, first, count, roi):
    v = _f32(vol)  # numpy shape (d2, d1, d0): d0 fastest
    d2, d1, d0 = v.shape
    na, nb = (d0, d1) if plane == 1 else (d1, d2)
    if roi is None:
        w, h, r = na, nb, None
    else:
        x0, x1 = sorted((roi[0], roi[2]))
        y0, y1 = sorted((roi[1], roi[3]))
        w, h = x1 - x0 + 1, y1 - y0 + 1
        r = np.asarray(roi, np.uint64)
    return v, d0, d1, d2, w, h, r


def slices_u16(vol, plane: int, first: int, count: int, lo: float, hi: float, roi=None) -> np.ndarray:
    """Restated slice serialisation (orc_slices_u16): uint16 slices (count, h, w) of the volume
    (numpy (d2, d1, d0), d0 fastest), plane 1 = XY or 4 = YZ."""
    v, d0, d1, d2, w, h, r = _slices_args(vol, plane, first, count, roi)
    out = np.zeros((count, h, w), np.uint16)
    rc = orc().orc_slices_u16(_p(v), _sz(d0), _sz(d1), _sz(d2), ctypes.c_int(plane), _sz(first), _sz(count),
                              None if r is None else _p(r, _SZ), _f(lo), _f(hi), _p(out, _U16))
    if rc != 0:
        raise ValueError("orc_slices_u16: bad arguments")
    return out


def ref_slices_u16(vol, plane: int, first: int, count: int, lo: float, hi: float, roi=None) -> np.ndarray:
    """The reference's ExtractSlice + ImageCaster<unsigned short, float> on the same volume."""
    v, d0, d1, d2, w, h, r = _slices_args(vol, plane, first, count, roi)
    out = np.zeros((count, h, w), np.uint16)
    _check_ref(ref().ref_slices_u16(_p(v), _sz(d0), _sz(d1), _sz(d2), ctypes.c_int(plane), _sz(first), _sz(count),
                                    None if r is None else _p(r, _SZ), _f(lo), _f(hi), _p(out, _U16)))
    return out


# ------------------------------------------------------- alternative ring cleaners


def median_filter(img, kx: int, ky: int, use_ref: bool = False) -> np.ndarray:
    """kipl TMedianFilter<float,2> with a kx x ky window on one image (h, w): the restatement
    (orc_median_filter) or, with use_ref, the reference template itself."""
    a = _f32(img)
    h, w = a.shape
    out = np.empty_like(a)
    if use_ref:
        _check_ref(ref().ref_median_filter(_p(a), _sz(w), _sz(h), ctypes.c_int(kx), ctypes.c_int(ky), _p(out)))
    elif orc().orc_median_filter(_p(a), _sz(w), _sz(h), ctypes.c_int(kx), ctypes.c_int(ky), _p(out)) != 0:
        raise ValueError("orc_median_filter: unsupported size")
    return out


def basicringclean(proj, use_ref: bool = False) -> np.ndarray:
    """BasicRingClean on projections (n, h, w); returns the cleaned copy."""
    p = _f32(proj).copy()
    n, h, w = p.shape
    if use_ref:
        _check_ref(ref().ref_basicringclean(_p(p), _sz(w), _sz(h), _sz(n)))
    elif orc().orc_basicringclean(_p(p), _sz(w), _sz(h), _sz(n)) != 0:
        raise ValueError("orc_basicringclean: unsupported size")
    return p


def sigmoid_lut(length: int, lam: float, sigma: float, use_ref: bool = False):
    """kipl SigmoidLUT: (table, (lo, hi, slope, intercept))."""
    lut = np.empty(length, np.float32)
    param = np.empty(4, np.float32)
    if use_ref:
        _check_ref(ref().ref_sigmoid_lut(_sz(length), _f(lam), _f(sigma), _p(lut), _p(param)))
    else:
        orc().orc_sigmoid_lut(_sz(length), _f(lam), _f(sigma), _p(lut), _p(param))
    return lut, param


def medianmixringclean(proj, threshold: float = 0.025, width: float = 0.0025, use_ref: bool = False) -> np.ndarray:
    """MedianMixRingClean on projections (n, h, w); returns the cleaned copy."""
    p = _f32(proj).copy()
    n, h, w = p.shape
    if use_ref:
        _check_ref(ref().ref_medianmixringclean(_p(p), _sz(w), _sz(h), _sz(n), _f(threshold), _f(width)))
    elif orc().orc_medianmixringclean(_p(p), _sz(w), _sz(h), _sz(n), _f(threshold), _f(width)) != 0:
        raise ValueError("orc_medianmixringclean: unsupported size")
    return p


def ref_gammaspotclean(proj, threshold3=25.0, threshold5=100.0, threshold7=400.0, sigma=0.8, mediansize=3):
    """The reference's GammaSpotCleanModule on projections (n, h, w); returns its output."""
    p = _f32(proj).copy()
    n, h, w = p.shape
    _check_ref(ref().ref_gammaspotclean(_p(p), _sz(w), _sz(h), _sz(n), _f(threshold3), _f(threshold5),
                                        _f(threshold7), _f(sigma), ctypes.c_int(mediansize)))
    return p


SPOT_METHODS = {"stddev": 0, "ring": 1, "median": 2, "minmax": 3, "trikernel": 4}


def spotclean2(proj, method: str = "ring", gamma: float = 0.1, sigma: float = 0.001, iterations: int = 1,
               minlevel: float = -0.1, maxlevel: float = 5.0, maxarea: int = 20, use_ref: bool = False) -> np.ndarray:
    """SpotClean2 (ImagingAlgorithms::SpotClean) on projections (n, h, w); returns the cleaned copy."""
    p = _f32(proj).copy()
    n, h, w = p.shape
    if use_ref:
        _check_ref(ref().ref_spotclean2(_p(p), _sz(w), _sz(h), _sz(n), method.encode(), _f(gamma), _f(sigma),
                                        ctypes.c_int(iterations), _f(minlevel), _f(maxlevel), ctypes.c_int(maxarea)))
    else:
        rc = orc().orc_spotclean(_p(p), _sz(w), _sz(h), _sz(n), ctypes.c_int(SPOT_METHODS[method]), _f(gamma),
                                 _f(sigma), ctypes.c_int(iterations), _f(minlevel), _f(maxlevel), ctypes.c_int(maxarea))
        if rc != 0:
            raise ValueError(f"orc_spotclean failed ({rc})")
    return p


def compute_weights(angles, scanarc=(0.0, 360.0), golden=False, use_ref=False, use_lib=False):
    """ComputeWeights on projection angles in acquisition order: (angles, weights) of the
    resulting map, in its order. use_ref: the reference's function; use_lib: the library's
    host implementation (mr_compute_weights)."""
    a = _f32(angles)
    n = a.size
    oa = np.zeros(max(n, 1), np.float32)
    ow = np.zeros(max(n, 1), np.float32)
    if use_ref:
        m = ctypes.c_size_t(0)
        _check_ref(ref().ref_compute_weights(_p(a), _sz(n), _f(scanarc[0]), _f(scanarc[1]), int(golden), _p(oa), _p(ow),
                                             ctypes.byref(m)))
        m = m.value
    elif use_lib:
        from imagingsuite_b200 import _lib as L

        arc = np.asarray(scanarc, np.float32)
        m = ctypes.c_size_t(0)
        L.check(L.lib().mr_compute_weights(_p(a), n, _p(arc), int(golden), _p(oa), _p(ow), ctypes.byref(m)))
        m = m.value
    else:
        orc().orc_compute_weights.restype = ctypes.c_size_t
        m = orc().orc_compute_weights(_p(a), _sz(n), _f(scanarc[0]), _f(scanarc[1]), int(golden), _p(oa), _p(ow))
    return oa[:m].copy(), ow[:m].copy()


def ref_fdk_double(proj, angles, weights, geom: FdkGeom) -> np.ndarray:
    """The reference's FDKbp (double-precision geometry, fdkbp.cpp) through FdkReconBase::Process
    3D on the same inputs as fdk(). Returns the XYZ volume (nv, nu, nu)."""
    proj = _f32(proj)
    nproj, nv, nu = proj.shape
    angles, weights = _f32(angles), _f32(weights)
    vol = np.zeros((nv, nu, nu), np.float32)
    _check_ref(ref().ref_fdk_double(_p(proj), _sz(nu), _sz(nv), _sz(nproj), _p(angles), _p(weights),
                                    ctypes.byref(geom), _p(vol), None))
    return vol
