"""ctypes binding of the mrcuda C ABI (``include/mrcuda.h``).

The library is built in-tree by ``imagingsuite_b200.build``. Loading fails loudly when it
is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmrcuda.so")
CHECKED_LIB_PATH = os.path.join(_HERE, "libmrcuda_checked.so")

c_size = ctypes.c_size_t
c_int = ctypes.c_int
c_float = ctypes.c_float
c_void = ctypes.c_void_p
P_float = ctypes.POINTER(ctypes.c_float)
P_size = ctypes.POINTER(ctypes.c_size_t)
P_int = ctypes.POINTER(ctypes.c_int)
P_u32 = ctypes.POINTER(ctypes.c_uint32)
P_double = ctypes.POINTER(ctypes.c_double)

MR_OK, MR_ERR_ARGUMENT, MR_ERR_CUDA, MR_ERR_ALLOCATION, MR_ERR_UNSUPPORTED, MR_ERR_DEVICE = range(6)
MR_F32, MR_BF16, MR_F16, MR_U16 = 0, 1, 2, 3
MR_PLANE_XY, MR_PLANE_YZ = 1, 4
MR_BP_MULTIPROJ_PARALLEL, MR_BP_MULTIPROJ_SERIAL, MR_BP_NEAREST = 0, 1, 2


class FdkGeom(ctypes.Structure):
    """mr_fdk_geom: the ReconConfig fields FDKbp_single reads."""

    _fields_ = [("sod", c_float), ("sdd", c_float), ("ppoint", c_float * 2), ("center", c_float),
                ("resolution", c_float * 2), ("voxelsize", c_float * 3), ("direction", c_int),
                ("correcttilt", c_int), ("tiltangle", c_float), ("tiltpivot", c_float)]


# name -> (restype, argtypes)
_PROTOS = {
    "mr_version": (c_int, []),
    "mr_status_string": (ctypes.c_char_p, [c_int]),
    "mr_last_error": (ctypes.c_char_p, []),
    "mr_reference_average": (c_int, [c_void, c_size, c_size, c_size, c_int, c_void, c_void]),
    "mr_projection_dose": (c_int, [c_void, c_int, c_size, c_size, c_size, P_size, c_void, c_void]),
    "mr_lognorm_logflat": (c_int, [c_void, c_void, c_size, c_int, c_float, c_void, c_void]),
    "mr_lognorm_doselog": (c_int, [P_float, c_size, c_float, P_float]),
    "mr_lognorm_apply": (c_int, [c_void, c_int, c_size, c_size, c_void, c_void, c_void, c_size, c_int, c_int,
                                 c_void, c_void]),
    "mr_lognorm_apply_lut": (c_int, [c_void, c_int, c_size, c_size, c_void, c_void, c_void, c_size, c_int, c_int,
                                     c_void, c_void]),
    "mr_morphspotclean": (c_int, [c_void, c_size, c_size, c_size, c_int, c_int, P_float, P_float, c_int, c_int, c_float,
                                  c_float, c_int, c_void]),
    "mr_wavelet_kernel": (c_int, [ctypes.c_char_p, P_int, P_int, P_float]),
    "mr_stripefilter": (c_int, [c_void, c_size, c_size, c_size, ctypes.c_char_p, c_int, c_float, c_void]),
    "mr_waveletringclean": (c_int, [c_void, c_size, c_size, c_size, ctypes.c_char_p, c_int, c_float, c_void]),
    "mr_median_filter": (c_int, [c_void, c_size, c_size, c_size, c_int, c_int, c_void, c_void]),
    "mr_basicringclean": (c_int, [c_void, c_size, c_size, c_size, c_void]),
    "mr_medianmixringclean": (c_int, [c_void, c_size, c_size, c_size, c_float, c_float, c_void]),
    "mr_sigmoid_lut": (c_int, [c_size, c_float, c_float, P_float, P_float]),
    "mr_compute_weights": (c_int, [P_float, c_size, P_float, c_int, P_float, P_float, P_size]),
    "mr_spotclean2": (c_int, [c_void, c_size, c_size, c_size, c_int, c_float, c_float, c_int, c_float, c_float, c_int,
                              c_void]),
    "mr_projfilter_tables": (c_int, [c_size, ctypes.c_char_p, c_float, c_float, c_int, c_float, c_int, P_size, P_size,
                                     P_float, P_float]),
    "mr_projfilter_create": (c_int, [c_size, ctypes.c_char_p, c_float, c_float, c_int, c_float, c_int,
                                     ctypes.POINTER(c_void)]),
    "mr_projfilter_destroy": (c_int, [c_void]),
    "mr_projfilter_info": (c_int, [c_void, P_size, P_size, P_float, P_float]),
    "mr_projfilter_apply": (c_int, [c_void, c_void, c_void, c_size, c_void, c_size, c_void]),
    "mr_bp_parallel_geometry": (c_int, [P_float, c_size, c_size, c_float, c_int, P_float, P_float, P_float]),
    "mr_bp_circle_mask": (c_int, [c_size, c_size, c_int, c_float, c_size, P_u32]),
    "mr_bp_parallel_tilt": (c_int, [c_float, c_float, c_size, P_float, P_float]),
    "mr_bp_parallel": (c_int, [c_void, c_int, c_void, c_void, c_void, c_void, c_void, c_void, c_size, c_size, c_size,
                               c_void, c_int, c_float, c_float, c_void, c_void]),
    "mr_bp_parallel_staged": (c_int, [c_void, c_size, c_int, c_void, c_void, c_void, c_void, c_void, c_void, c_size,
                                      c_size, c_size, c_void, c_int, c_float, c_float, c_void, c_void]),
    "mr_bp_parallel_rows": (c_int, [c_void, c_size, c_int, c_void, c_void, c_void, c_void, c_void, c_void, c_size,
                                    c_size, c_size, c_void, c_int, c_float, c_float, c_size, c_size, c_void, c_void]),
    "mr_bp_parallel_variant": (c_int, [c_int, c_void, c_size, c_int, c_void, c_void, c_void, c_void, c_void, c_void,
                                       c_size, c_size, c_size, c_void, c_int, c_float, c_float, c_size, c_size, c_void,
                                       c_void]),
    "mr_quantize": (c_int, [c_void, c_size, c_size, c_int, c_void, c_void, c_void]),
    "mr_quantize_noalloc": (c_int, [c_void, c_size, c_size, c_int, c_void, c_void, c_void]),
    "mr_fdk_partials": (c_int, [ctypes.POINTER(FdkGeom), c_size, c_size, P_float, c_size, P_float, P_float, P_float,
                                P_float, P_float, P_int]),
    "mr_fdk_filter": (c_int, [c_void, c_size, c_size, c_size, c_void, c_float, c_float, c_int, c_void, c_void,
                              c_void]),
    "mr_fdk_filter_rows": (c_int, [c_void, c_size, c_size, c_size, c_size, c_size, c_void, c_float, c_float, c_int,
                                   c_void, c_void, c_void]),
    "mr_fdk_backproject": (c_int, [c_void, c_int, c_void, c_size, c_size, c_size, c_void, c_void, c_void, c_int,
                                   c_void, c_int, c_int, c_int, c_void, c_void]),
    "mr_fdk_backproject_slab": (c_int, [c_void, c_int, c_void, c_size, c_size, c_size, c_void, c_void, c_void, c_int,
                                        c_void, c_int, c_int, c_int, c_size, c_size, c_void, c_void]),
    "mr_fdk_box": (c_int, [P_float, P_float, P_float, c_size, c_size, c_size, c_int, P_int, P_int]),
    "mr_fdk_maps64": (c_int, [ctypes.POINTER(FdkGeom), c_size, c_size, P_float, c_size, P_double]),
    "mr_fdk_box_maps": (c_int, [P_double, c_size, c_size, c_size, c_int, P_int, P_int]),
    "mr_fdk_backproject_fast": (c_int, [c_void, c_int, c_void, c_size, c_size, c_size, c_void, c_void, c_int, c_int,
                                        c_int, c_void, c_void]),
    "mr_fdk_backproject_f64": (c_int, [c_void, c_size, c_size, c_size, c_void, c_void, c_void, c_size, c_void,
                                       c_void]),
    "mr_slices_u16": (c_int, [c_void, c_int, c_size, c_size, c_size, c_size, c_size, P_size, c_float, c_float, c_void,
                              c_void]),
    "mr_joseph_geometry": (c_int, [P_float, c_size, c_size, P_float]),
    "mr_joseph_forward": (c_int, [c_void, c_void, c_size, c_size, c_void, c_size, c_size, c_float, c_float, c_float,
                                  c_void, c_void, c_void]),
    "mr_joseph_adjoint": (c_int, [c_void, c_size, c_size, c_void, c_size, c_size, c_float, c_float, c_float, c_int,
                                  c_void, c_void]),
    "mr_slice_dot": (c_int, [c_void, c_void, c_size, c_size, c_size, c_void, c_void]),
    "mr_mbp_geometry": (c_int, [P_float, c_size, c_size, c_size, c_float, c_float, c_float, c_int, P_float, P_float]),
    "mr_mbp_adjoint": (c_int, [c_void, c_size, c_size, c_void, c_void, c_size, c_void, c_int, c_void, c_void]),
    "mr_mbp_forward": (c_int, [c_void, c_size, c_size, c_void, c_void, c_size, c_void, c_void, c_void, c_void]),
    "mr_device_status": (c_int, [P_int]),
    "mr_measure_smem": (c_int, [P_double, P_double]),
    "mr_data_validator": (c_int, [c_void, c_size, c_void, c_void]),
    "mr_set_wait_limit": (c_int, [c_int]),
    "mr_bounds_status": (c_int, [ctypes.POINTER(ctypes.c_ulonglong)]),
    "mr_debug_fail_allocation": (c_int, [ctypes.c_longlong]),
    "mr_trace_push": (c_int, [ctypes.c_char_p]),
    "mr_trace_pop": (c_int, []),
}

EXPORTED = tuple(_PROTOS)

_lib = None


class MrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status
        self.message = message


def load(path: str) -> ctypes.CDLL:
    """A build of the library at `path` with every prototype set (the bounds-checked build
    libmrcuda_checked.so has the same entry points)."""
    if not os.path.exists(path):
        raise RuntimeError(f"mrcuda library not built: {path} (python -m imagingsuite_b200.build)")
    l = ctypes.CDLL(path)
    for name, (res, args) in _PROTOS.items():
        f = getattr(l, name)
        f.restype = res
        f.argtypes = args
    return l


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load(LIB_PATH)
    return _lib


def check(status: int) -> None:
    if status != MR_OK:
        raise MrError(status, lib().mr_last_error().decode())


def check_device() -> None:
    """Reads (and clears) the device error word of the bounded waits; raises MrError with
    MR_ERR_DEVICE when a kernel reported one. Synchronizes the device."""
    word = ctypes.c_int(0)
    check(lib().mr_device_status(ctypes.byref(word)))
    if word.value:
        raise MrError(MR_ERR_DEVICE, f"a kernel reported device error word {word.value} (bounded wait expired)")
