"""The C-ABI library (include/mrcuda.h) on the CPU: it loads, exports every declared
symbol, and its host-only entry points (geometry, masks, filter tables, FDK partials)
reproduce the reference arithmetic exactly. No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from imagingsuite_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "mrcuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mr_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    lib = L.lib()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.EXPORTED)


def test_checked_build_exports_the_same_symbols():
    """libmrcuda_checked.so (the bounds-checked build) has every entry point of the header and
    answers mr_bounds_status without a device."""
    if not os.path.exists(L.CHECKED_LIB_PATH):
        pytest.skip("bounds-checked build not made (python -m imagingsuite_b200.build --bounds-check)")
    lib = L.load(L.CHECKED_LIB_PATH)
    for n in _declared():
        assert hasattr(lib, n), n


def test_version_and_status():
    lib = L.lib()
    assert lib.mr_version() >= 100
    assert lib.mr_status_string(0) == b"ok"
    assert lib.mr_status_string(1) == b"invalid argument"


def test_argument_errors_need_no_gpu():
    lib = L.lib()
    st = lib.mr_lognorm_apply(None, 0, 10, 1, None, None, None, 1, 1, 1, None, None)
    assert st == L.MR_ERR_ARGUMENT
    assert b"null" in lib.mr_last_error()
    st = lib.mr_projfilter_tables(64, b"nonsense", 0.5, 1.0, 1, 0.1, 2, None, None, None, None)
    assert st == L.MR_ERR_ARGUMENT
    assert lib.mr_last_error() == b"Could not convert filter string to enum."
    st = lib.mr_projfilter_tables(64, b"hanning", 0.75, 1.0, 1, 0.1, 2, None, None, None, None)
    assert st == L.MR_ERR_ARGUMENT and b"Cut off" in lib.mr_last_error()
    # slice range outside the volume: rejected before any device access (the pointers are
    # never dereferenced)
    fake = 256
    st = lib.mr_fdk_backproject_slab(fake, L.MR_F32, None, 64, 32, 4, fake, fake, fake, 1, fake, 0, 0, 0, 8, 40, fake,
                                     None)
    assert st == L.MR_ERR_ARGUMENT and b"slice range" in lib.mr_last_error()
    st = lib.mr_fdk_backproject_slab(fake, L.MR_F32, None, 64, 32, 4, fake, fake, fake, 1, fake, 0, 0, 0, 9, 8, fake,
                                     None)
    assert st == L.MR_ERR_ARGUMENT


@pytest.mark.parametrize("direction", [0, 1])
def test_bp_geometry_matches_oracle(direction):
    ang = np.linspace(0, 359.7, 1201).astype(np.float32)
    s, c, su = (np.empty_like(ang) for _ in range(3))
    L.check(L.lib().mr_bp_parallel_geometry(ang.ctypes.data_as(L.P_float), ang.size, 2048, 1023.7, direction,
                                            s.ctypes.data_as(L.P_float), c.ctypes.data_as(L.P_float),
                                            su.ctypes.data_as(L.P_float)))
    os_, oc, osu = O.bp_geometry(ang, 2048, 1023.7, direction)
    assert np.array_equal(s, os_) and np.array_equal(c, oc) and np.array_equal(su, osu)


@pytest.mark.parametrize("n,tilt", [(256, False), (255, False), (64, True), (2048, False)])
def test_circle_mask_matches_oracle(n, tilt):
    m = np.zeros(2 * n, np.uint32)
    L.check(L.lib().mr_bp_circle_mask(n, n, int(tilt), 0.8, 40, m.ctypes.data_as(L.P_u32)))
    assert np.array_equal(m, O.circle_mask(n, n, tilt, 0.8, 40))


@pytest.mark.parametrize("ftype", ["Ram-Lak", "shepp-logan", "Hanning", "hamming", "butterworth"])
@pytest.mark.parametrize("nu,pd", [(256, 2), (2048, 2), (100, 1)])
def test_filter_tables_match_oracle(ftype, nu, pd):
    nfft, ins = ctypes.c_size_t(), ctypes.c_size_t()
    lib = L.lib()
    L.check(lib.mr_projfilter_tables(nu, ftype.encode(), 0.45, 3.0, 1, 0.1, pd, ctypes.byref(nfft), ctypes.byref(ins),
                                     None, None))
    f = np.zeros(nfft.value // 2, np.float32)
    p = np.zeros(max(1, ins.value), np.float32)
    L.check(lib.mr_projfilter_tables(nu, ftype.encode(), 0.45, 3.0, 1, 0.1, pd, None, None,
                                     f.ctypes.data_as(L.P_float), p.ctypes.data_as(L.P_float)))
    plan = O.projfilter_plan(nu, ftype, 0.45, 3.0, True, 0.1, pd)
    assert nfft.value == plan.nfft and ins.value == plan.ninsert
    assert np.array_equal(f, plan.filter)
    assert np.array_equal(p[: ins.value], plan.pad)


def _partials(g, nu, nv, ang):
    n = ang.size
    xip = np.empty((n, nu, 3), np.float32)
    yip = np.empty((n, nu, 3), np.float32)
    zip_ = np.empty((n, nv, 3), np.float32)
    s2, sc, uni = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
    L.check(L.lib().mr_fdk_partials(ctypes.byref(g), nu, nv, ang.ctypes.data_as(L.P_float), n,
                                    xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                                    zip_.ctypes.data_as(L.P_float), ctypes.byref(s2), ctypes.byref(sc),
                                    ctypes.byref(uni)))
    return xip, yip, zip_, s2.value, sc.value, uni.value


def test_fdk_partials_projection_matrix():
    """xip/yip/zip rebuilt from the oracle's projection matrix agree bit for bit."""
    nu, nv = 64, 48
    ang = np.array([0.0, 33.3, 181.0], np.float32)
    g = L.FdkGeom()
    g.sod, g.sdd = 300.0, 600.0
    g.ppoint[0], g.ppoint[1] = 31.5, 23.5
    g.center = 31.5
    g.resolution[0] = g.resolution[1] = 0.2
    g.voxelsize[0] = g.voxelsize[1] = g.voxelsize[2] = 0.1
    xip, yip, zip_, s2, sc, uni = _partials(g, nu, nv, ang)
    assert uni == 1
    assert s2 == np.float32(np.float32(300.0 * 300.0) / np.float32(600.0 * 600.0))
    og = O.fdk_geom(300.0, 600.0, (31.5, 23.5), 31.5, (0.2, 0.2), (0.1, 0.1, 0.1))
    f = np.float32
    for p, a in enumerate(ang):
        pm = O.fdk_projmatrix(og, nu, float(a))
        U = f(nu)
        origin0 = f(f(-(U - f(31.5))) * f(0.1)) - f(f(0.1) / f(2))
        ic0, ic1 = f(31.5), f(23.5)
        for i in (0, 7, 63):
            x = f(origin0 + f(f(i) * f(0.1)))
            assert xip[p, i, 0] == f(x * f(pm[0] + f(ic0 * pm[8])))
            assert xip[p, i, 2] == f(x * pm[8])
        assert np.all(zip_[p, :, 2] == zip_[p, 0, 2])


def test_fdk_partials_tilt_not_uniform():
    g = L.FdkGeom()
    g.sod, g.sdd = 300.0, 600.0
    g.ppoint[0], g.ppoint[1] = 15.5, 11.5
    g.center = 15.5
    g.resolution[0] = g.resolution[1] = 0.2
    g.voxelsize[0] = g.voxelsize[1] = g.voxelsize[2] = 0.1
    g.correcttilt = 1
    g.tiltangle = 0.5
    g.tiltpivot = 5.0
    *_, uni = _partials(g, 32, 24, np.array([0.0, 90.0], np.float32))
    assert uni == 0


@pytest.mark.parametrize("n", [n for n in range(1, 31) if n != 28])
def test_wavelet_kernel_abi(n):
    b, e = ctypes.c_int(), ctypes.c_int()
    taps = np.zeros(4 * 60, np.float32)
    L.check(L.lib().mr_wavelet_kernel(f"daub{n}".encode(), ctypes.byref(b), ctypes.byref(e),
                                      taps.ctypes.data_as(L.P_float)))
    ob, oe, k = O.wavelet_kernel(f"daub{n}")
    K = oe - ob + 1
    assert (b.value, e.value) == (ob, oe)
    assert np.array_equal(taps[: 4 * K].reshape(4, K), k)


def test_wavelet_kernel_rejects_unknown():
    b, e = ctypes.c_int(), ctypes.c_int()
    assert L.lib().mr_wavelet_kernel(b"haar", ctypes.byref(b), ctypes.byref(e), None) == L.MR_ERR_UNSUPPORTED
    assert L.lib().mr_wavelet_kernel(b"daub31", ctypes.byref(b), ctypes.byref(e), None) == L.MR_ERR_UNSUPPORTED
    assert L.lib().mr_wavelet_kernel(b"daub28", ctypes.byref(b), ctypes.byref(e), None) == L.MR_ERR_UNSUPPORTED


@pytest.mark.parametrize("tilt", [0.0, 0.4])
@pytest.mark.parametrize("direction", [0, 1])
def test_fdk_maps64_match_oracle_and_partials(tilt, direction):
    """FP64 detector maps equal the oracle's restatement bit for bit and agree with the float
    partials of FDKbp_single to float rounding (1e-4 pixel)."""
    nu, nv = 40, 36
    ang = (np.arange(16) * 22.5 + 3.3).astype(np.float32)
    og = O.fdk_geom(300.0, 600.0, (20.3, 17.1), 19.7, (0.2, 0.2), (0.1, 0.1, 0.1), direction=direction,
                    correcttilt=bool(tilt), tiltangle=tilt, tiltpivot=3.0)
    g = L.FdkGeom()
    ctypes.memmove(ctypes.byref(g), ctypes.byref(og), ctypes.sizeof(g))
    m = np.zeros((ang.size, 12), np.float64)
    L.check(L.lib().mr_fdk_maps64(ctypes.byref(g), nu, nv, ang.ctypes.data_as(L.P_float), ang.size,
                                  m.ctypes.data_as(L.P_double)))
    assert np.array_equal(m, O.fdk_maps64(og, nu, nv, ang))
    xip, yip, zip_, *_ = _partials(g, nu, nv, ang)
    i, j, k = np.meshgrid(np.arange(0, nu, 7), np.arange(0, nu, 5), np.arange(0, nv, 6), indexing="ij")
    for p in range(ang.size):
        a = [zip_[p, k, e].astype(np.float64) + yip[p, j, e] + xip[p, i, e] for e in range(3)]
        M_ = m[p]
        u = M_[0] * i + M_[1] * j + M_[2] * k + M_[3]
        v = M_[4] * i + M_[5] * j + M_[6] * k + M_[7]
        w = M_[8] * i + M_[9] * j + M_[10] * k + M_[11]
        assert np.abs(a[0] / a[2] - u / w).max() < 1e-4
        assert np.abs(a[1] / a[2] - v / w).max() < 1e-4
        assert np.abs(a[2] / w - 1).max() < 1e-5
    if not tilt:
        assert np.all(m[:, 2] == 0) and np.all(m[:, 10] == 0)  # column and depth do not depend on the slice


def test_fdk_box_maps_covers_partials_box():
    nu, nv, n = 64, 48, 32
    ang = (np.arange(n) * 360.0 / n).astype(np.float32)
    og = O.fdk_geom(300.0, 600.0, (31.7, 23.2), 31.6, (0.2, 0.2), (0.1, 0.1, 0.1))
    g = L.FdkGeom()
    ctypes.memmove(ctypes.byref(g), ctypes.byref(og), ctypes.sizeof(g))
    xip, yip, zip_, *_ = _partials(g, nu, nv, ang)
    m = O.fdk_maps64(og, nu, nv, ang)
    a, b, c, d = (ctypes.c_int() for _ in range(4))
    L.check(L.lib().mr_fdk_box(xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                               zip_.ctypes.data_as(L.P_float), nu, nv, n, L.MR_BF16, ctypes.byref(a), ctypes.byref(b)))
    L.check(L.lib().mr_fdk_box_maps(m.ctypes.data_as(L.P_double), nu, nv, n, L.MR_BF16, ctypes.byref(c), ctypes.byref(d)))
    assert (a.value, b.value) == (c.value, d.value)
    assert c.value % 8 == 0 and c.value > 32 and d.value > 32


def test_fdk_bp64_oracle_close_to_float_path():
    """The FP64 oracle and the reference's float arithmetic differ only where a voxel centre
    projects within float rounding of a pixel boundary (nearest-neighbour ties)."""
    rng = np.random.default_rng(5)
    nu, nv, n = 48, 40, 24
    proj = rng.standard_normal((n, nv, nu)).astype(np.float32)
    ang = np.sort(rng.uniform(0, 360, n)).astype(np.float32)
    og = O.fdk_geom(300.0, 600.0, (23.37, 19.61), 23.71, (0.2, 0.2), (0.1, 0.1, 0.1))
    f32 = O.fdk_bp(proj, ang, og)
    sl = np.array([0, 5, 17, 39], np.int32)
    f64 = O.fdk_bp64(proj, O.fdk_maps64(og, nu, nv, ang), sl)
    d = np.abs(f32[sl] - f64)
    assert (d > 1e-4).sum() <= 10  # a handful of tie voxels out of 9216
    assert np.median(d) < 1e-6
