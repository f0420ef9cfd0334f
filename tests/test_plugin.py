"""The MuhRec module libraries (imagingsuite_b200/plugin): libB200PreprocModules.so (tag
"muhrec") and libB200BackProjectors.so (tag "muhrecbp"), loaded the way ReconEngine loads
module libraries - through the reference's own ModuleItem / BackProjItem (compiled from the
reference sources in oracle/_ref) - and compared with the reference's own modules driven
through the same Configure / SetROI / Process / GetSlice calls.

CPU: the factory functions (tags, names, GetModuleList against the reference modules'
defaults). GPU: every module on seeded data against the reference module of the same name.
"""
import os

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRE = os.path.join(ROOT, "imagingsuite_b200", "plugin", "libB200PreprocModules.so")
BP = os.path.join(ROOT, "imagingsuite_b200", "plugin", "libB200BackProjectors.so")

PRE_MODULES = ("FullLogNorm", "MorphSpotClean", "WaveletRingClean", "ProjectionFilterSingle")
BP_MODULES = ("MultiProjBPparallel", "MultiProjBP", "NearestNeighborBP", "FDKbp_single")


@pytest.fixture(scope="module")
def plugins(ref_lib):
    for p in (PRE, BP):
        if not os.path.exists(p):
            pytest.fail(f"module library not built: {p} (make -C imagingsuite_b200/plugin REF=...)")
    return PRE, BP


def test_module_lists_match_reference_defaults(plugins):
    rc, mods = O.ref_plugin_module_list(PRE, "muhrec")
    assert rc == 0 and set(mods) == set(PRE_MODULES)
    for name in PRE_MODULES:
        assert mods[name] == O.ref_module_parameters(name), name  # same keys, same default texts
    rc, mods = O.ref_plugin_module_list(BP, "muhrecbp")
    assert rc == 0 and set(mods) == set(BP_MODULES)
    for name in BP_MODULES:
        # the reference's FdkReconBase leaves its defaults uninitialised: keys only
        assert set(mods[name]) == set(O.ref_module_parameters(name, backprojector=True)), name


def test_factory_tags_and_names(plugins):
    assert O.ref_plugin_module_list(PRE, "muhrecbp")[0] == -1
    assert O.ref_plugin_module_list(BP, "muhrec")[0] == -1
    for name in PRE_MODULES + ("FullLogNormCUDA", "MorphSpotCleanCUDA", "WaveletRingCleanCUDA", "ProjectionFilterCUDA"):
        assert O.ref_plugin_has_module(PRE, "muhrec", name), name
        assert not O.ref_plugin_has_module(PRE, "muhrecbp", name), name
    for name in BP_MODULES + ("MultiProjBPCUDA", "FDKbpCUDA"):
        assert O.ref_plugin_has_module(BP, "muhrecbp", name), name
        assert not O.ref_plugin_has_module(BP, "muhrec", name), name
    assert not O.ref_plugin_has_module(PRE, "muhrec", "SinoSpotClean")


# ------------------------------------------------------------------------------- GPU


def _relrms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def _counts(seed, nproj, nv, nu):
    rng = np.random.default_rng(seed)
    flats = rng.normal(20000, 150, (5, nv, nu)).astype(np.float32).round()
    darks = rng.normal(100, 3, (4, nv, nu)).astype(np.float32).round()
    proj = (rng.uniform(0.05, 0.9, (nproj, nv, nu)) * 20000 + 100).astype(np.float32).round()
    proj[0, 0, :5] = 90  # I - D <= 0
    return proj, flats, darks


@pytest.mark.gpu
@pytest.mark.parametrize("average", ["ImageWeightedAverage", "ImageAverage"])
@pytest.mark.parametrize("usenorm", [True, False])
def test_fulllognorm_loads_reference_files(cuda, plugins, tmp_path, average, usenorm):
    """FullLogNorm through the engine's path: SetROI reads the dark and open-beam images from
    files with the framework's ProjectionReader (MATLAB files here), averages them and takes
    their doses over the dose ROI; Process 3D takes the projection doses from coeff."""
    nproj, nv, nu = 9, 24, 40
    proj, flats, darks = _counts(5, nproj, nv, nu)
    for i, f in enumerate(flats):
        O.ref_write_mat(f, str(tmp_path / f"ob_{i + 1:04d}.mat"))
    for i, d in enumerate(darks):
        O.ref_write_mat(d, str(tmp_path / f"dc_{i + 1:04d}.mat"))
    roi = (0, 0, nu, nv)
    dose_roi = (2, 3, 30, 20)
    doses = [O.frame_dose(p, dose_roi) for p in proj]
    kw = dict(params={"usenormregion": str(usenorm).lower(), "uselut": "false", "referenceaverage": average},
              coeff={"dose": " ".join("%.9g" % d for d in doses)}, refpath=str(tmp_path) + "/",
              obmask="ob_####.mat", nob=5, obfirst=1, dcmask="dc_####.mat", ndc=4, dcfirst=1, dose_roi=dose_roi,
              roi=roi)
    exp = O.ref_preproc_module(proj, "FullLogNorm", **kw)
    got = O.ref_preproc_module(proj, "FullLogNorm", sofile=PRE, **kw)
    # CUDA logf against glibc logf: 1 ulp of each log term
    tol = 2 * np.spacing(np.float32(np.abs(exp).max() + 12.0))
    assert np.abs(got.astype(np.float64) - exp).max() <= tol
    assert np.array_equal(got == 0, exp == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", ["0 0", "0.01 0.01"])
@pytest.mark.parametrize("threading", ["false", "true"])
def test_morphspotclean_module(cuda, plugins, sigma, threading):
    rng = np.random.default_rng(6)
    proj = (rng.standard_normal((7, 40, 56)) * 0.05 + 1.0).astype(np.float32)
    idx = rng.integers(0, proj.size, 60)
    proj.flat[idx] = rng.choice([0.0, 4.0], 60)
    params = {"connectivity": "conn8", "cleanmethod": "morphcleanreplace", "detectionmethod": "morphdetectboth",
              "threshold": "0.1 0.1", "sigma": sigma, "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false",
              "clampdata": "true", "minlevel": "0.5", "maxlevel": "1.2", "threading": threading}
    exp = O.ref_preproc_module(proj, "MorphSpotClean", params)
    got = O.ref_preproc_module(proj, "MorphSpotCleanCUDA", params, sofile=PRE)
    if sigma == "0 0":
        assert np.array_equal(got, exp)
    else:  # the sigmoid blend through CUDA's expf: a few ulp
        assert np.abs(got - exp).max() <= 8 * np.spacing(np.float32(np.abs(exp).max()))


@pytest.mark.gpu
def test_waveletringclean_module(cuda, plugins):
    """WaveletRingClean through the module library against the reference's stripe filter on
    every sinogram (the reference module itself crashes in its StripeFilter constructor, so the
    harness's equivalent drives the same filter)."""
    rng = np.random.default_rng(7)
    proj = (rng.standard_normal((90, 6, 64)) * 0.1 + 1.0).astype(np.float32)
    proj[:, :, 17] += 0.05
    params = {"wname": "daub7", "sigma": "0.1", "decnum": "2", "parallel": "false", "method": "verticalfft"}
    got = O.ref_preproc_module(proj, "WaveletRingClean", params, sofile=PRE)
    exp = O.waveletringclean(proj, "daub7", 2, 0.1, use_ref=True)
    assert _relrms(got, exp) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("ftype", ["Hanning", "ram-lak", "Butterworth"])
def test_projectionfilter_module(cuda, plugins, ftype):
    rng = np.random.default_rng(8)
    proj = rng.standard_normal((5, 12, 100)).astype(np.float32)
    params = {"filtertype": ftype, "cutoff": "0.45", "order": "2", "usebias": "true", "biasweight": "0.1",
              "paddingdoubler": "2"}
    roi = (0, 0, 100, 12)
    exp = O.ref_preproc_module(proj, "ProjectionFilterSingle", params, roi=roi)
    got = O.ref_preproc_module(proj, "ProjectionFilterCUDA", params, sofile=PRE, roi=roi)
    assert _relrms(got, exp) < 1e-5  # FP32 FFT against the reference build's FP64 FFT


def _bp_cfg(nu, nv, tilt=False, direction=0, cone=False, matrix_roi=None):
    c = O.RefBpConfig()
    c.center = (nu - 1) / 2.0 + 0.27
    c.direction = direction
    c.correcttilt = int(tilt)
    c.tiltangle, c.tiltpivot = 0.6, nv / 2.0
    c.cone = int(cone)
    c.sod, c.sdd = 300.0, 600.0
    c.ppoint[0], c.ppoint[1] = (nu - 1) / 2.0 + 0.13, (nv - 1) / 2.0 - 0.21
    c.resolution[0] = c.resolution[1] = 0.2
    c.voxelsize[0] = c.voxelsize[1] = c.voxelsize[2] = 0.1
    c.use_matrix_roi = int(matrix_roi is not None)
    for i, v in enumerate(matrix_roi or (0, 0, 0, 0)):
        c.matrix_roi[i] = v
    return c


BP_PARAMS = {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["MultiProjBPparallel", "MultiProjBP", "NearestNeighborBP"])
@pytest.mark.parametrize("tilt", [False, True])
@pytest.mark.parametrize("matrix_roi", [None, (9, 5, 50, 40)])
def test_parallel_backprojectors(cuda, plugins, name, tilt, matrix_roi):
    """Volume and GetSlice (with the matrix ROI's mask and crop) of the three parallel-beam
    backprojectors: bit for bit against the reference modules."""
    rng = np.random.default_rng(9)
    nproj, nv, nu = 40, 12, 64
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    cfg = _bp_cfg(nu, nv, tilt=tilt, direction=1, matrix_roi=matrix_roi)
    roi = (0, 3, nu, 3 + nv)
    ev, es = O.ref_bp_module(proj, ang, w, name, cfg, roi, BP_PARAMS)
    gv, gs = O.ref_bp_module(proj, ang, w, name, cfg, roi, BP_PARAMS, sofile=BP)
    assert np.array_equal(gv, ev)
    assert gs.shape == es.shape and np.array_equal(gs, es)


@pytest.mark.gpu
@pytest.mark.parametrize("matrix_roi", [None, (6, 4, 40, 50)])
def test_fdk_backprojector(cuda, plugins, matrix_roi):
    rng = np.random.default_rng(10)
    nproj, nv, nu = 24, 40, 64
    proj = (rng.standard_normal((nproj, nv, nu)) * 0.2 + 1.0).astype(np.float32)
    ang = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    w = np.full(nproj, np.float32(1.0 / nproj))
    cfg = _bp_cfg(nu, nv, cone=True, matrix_roi=matrix_roi)
    roi = (0, 0, nu, nv)
    ev, es = O.ref_bp_module(proj, ang, w, "FDKbp_single", cfg, roi, BP_PARAMS)
    gv, gs = O.ref_bp_module(proj, ang, w, "FDKbpCUDA", cfg, roi, BP_PARAMS, sofile=BP)
    assert _relrms(gv, ev) < 1e-5  # FP32 FFT ramp filter against the reference build's FP64 FFT
    assert gs.shape == es.shape and _relrms(gs, es) < 1e-5
