"""The C restatement (oracle/liboracle.so) against the reference's own modules compiled from
source (oracle/_ref/libmuhrec_ref.so), on seeded inputs. These pins are what make the
oracle trustworthy: every GPU parity test compares against the restatement."""
import numpy as np
import pytest

import oracle as O


def _rng(seed):
    return np.random.default_rng(seed)


@pytest.mark.parametrize("tilt", [False, True])
@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("buffersize", [16, 7])
def test_bp_parallel_bit_exact(ref_lib, tilt, direction, buffersize):
    rng = _rng(10 + buffersize)
    nproj, nv, nu = 37, 12, 48
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    kw = dict(direction=direction, buffersize=buffersize, correcttilt=tilt, tiltangle=0.6, tiltpivot=2.0, roi_y0=3)
    a = O.bp_parallel(proj, ang, w, 23.5, **kw)
    b = O.bp_parallel(proj, ang, w, 23.5, use_ref=True, **kw)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("buffersize", [16, 7])
def test_bp_serial_equals_parallel_without_tilt(ref_lib, direction, buffersize):
    """The reference's serial MultiProjectionBP (MultiProjBP.cpp) gives the parallel
    backprojector's volume bit for bit without tilt correction, so the module of that name runs
    the same kernels."""
    rng = _rng(20 + buffersize)
    nproj, nv, nu = 37, 12, 48
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    kw = dict(direction=direction, buffersize=buffersize, roi_y0=3)
    a = O.bp_parallel(proj, ang, w, 23.5, **kw)
    assert np.array_equal(a, O.bp_parallel(proj, ang, w, 23.5, use_ref=True, serial=True, **kw))


def test_bp_serial_tilt_shifts_once(ref_lib):
    """With tilt correction the serial version differs from the parallel one from the second
    group of 4 slices on (one shift of the interpolation weight per group instead of two); in
    the first group only by the order in which the centre offset is subtracted (rounding)."""
    rng = _rng(21)
    nproj, nv, nu = 37, 12, 48
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = np.ones(nproj, np.float32)
    kw = dict(direction=0, buffersize=16, correcttilt=True, tiltangle=0.6, tiltpivot=2.0, roi_y0=3)
    par = O.bp_parallel(proj, ang, w, 23.5, use_ref=True, **kw)
    ser = O.bp_parallel(proj, ang, w, 23.5, use_ref=True, serial=True, **kw)
    assert np.abs(par[:, :, :4] - ser[:, :, :4]).max() < 1e-3
    assert all(np.abs(par[:, :, z] - ser[:, :, z]).max() > 0.1 for z in range(4, 12))


@pytest.mark.parametrize("variant", ["serial", "nn"])
@pytest.mark.parametrize("tilt", [False, True])
@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("buffersize", [16, 7])
@pytest.mark.parametrize("nv", [12, 7, 10])
def test_bp_variants_bit_exact(ref_lib, variant, tilt, direction, buffersize, nv):
    """The factory's other parallel-beam backprojectors restated (orc_bp_parallel_variant): the
    serial MultiProjectionBP (one weight shift per slice group under tilt; with a slice count
    that is not a multiple of 4 its second sample comes from elsewhere in the padded buffer) and
    NearestNeighborBP (truncated position, no interpolation, constant tilt offset), against the
    compiled modules."""
    rng = _rng(30 + buffersize + 2 * direction + nv)
    nproj, nu = 37, 48
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    kw = dict(direction=direction, buffersize=buffersize, correcttilt=tilt, tiltangle=0.6, tiltpivot=2.0, roi_y0=3,
              serial=variant == "serial", nn=variant == "nn")
    assert np.array_equal(O.bp_parallel(proj, ang, w, 23.5, **kw), O.bp_parallel(proj, ang, w, 23.5, use_ref=True, **kw))


def test_bp_serial_ragged_differs_from_parallel(ref_lib):
    """Without tilt and with a slice count that is not a multiple of 4 the serial
    MultiProjectionBP no longer equals the parallel one (its column B stride), so the module
    runs its own sampling there."""
    rng = _rng(22)
    nproj, nv, nu = 19, 7, 40
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = np.ones(nproj, np.float32)
    par = O.bp_parallel(proj, ang, w, 19.5, use_ref=True)
    ser = O.bp_parallel(proj, ang, w, 19.5, use_ref=True, serial=True)
    assert np.abs(par - ser).max() > 0.1


def test_bp_parallel_ragged_sizes(ref_lib):
    # nv not a multiple of 4 (the reference only updates 4*(nv/4) slices), odd nu
    rng = _rng(3)
    nproj, nv, nu = 9, 7, 33
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 20.0).astype(np.float32)
    w = np.ones(nproj, np.float32)
    a = O.bp_parallel(proj, ang, w, 16.2, buffersize=16)
    b = O.bp_parallel(proj, ang, w, 16.2, buffersize=16, use_ref=True)
    assert np.array_equal(a, b)
    assert not a[:, :, 4:].any()


@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("pp", [(23.5, 19.5), (20.0, 30.2), (26.0, 4.0)])
def test_fdk_bit_exact(ref_lib, direction, pp):
    rng = _rng(20)
    nproj, nv, nu = 16, 36, 40
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    g = O.fdk_geom(300.0, 600.0, pp, 19.7, (0.2, 0.2), (0.1, 0.1, 0.1), direction=direction)
    a = O.fdk(proj, ang, w, g)
    b = O.fdk(proj, ang, w, g, use_ref=True)
    assert np.array_equal(a, b)


def test_fdk_prepare_then_bp_equals_fdk():
    rng = _rng(21)
    nproj, nv, nu = 8, 24, 32
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 45.0).astype(np.float32)
    w = rng.uniform(0.5, 1.5, nproj).astype(np.float32)
    g = O.fdk_geom(250.0, 500.0, (15.5, 11.5), 15.5, (0.2, 0.2), (0.1, 0.1, 0.1))
    a = O.fdk(proj, ang, w, g)
    b = O.fdk_bp(O.fdk_prepare(proj, w, g), ang, g)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("usenorm", [False, True])
@pytest.mark.parametrize("method", ["ImageAverage", "ImageSum", "ImageMedian", "ImageMin", "ImageMax",
                                    "ImageWeightedAverage"])
def test_fulllognorm_bit_exact(ref_lib, usenorm, method):
    rng = _rng(30)
    nproj, nv, nu = 11, 10, 24
    darks = np.round(rng.normal(100, 3, (4, nv, nu))).astype(np.float32)
    flats = (rng.poisson(30000, (5, nv, nu)) + darks[0]).astype(np.float32)
    proj = (rng.poisson(20000, (nproj, nv, nu)) + 100).astype(np.float32)
    proj[0, 0, :5] = 50  # I - D <= 0 branch
    roi = (2, 2, 20, 9)
    out_r, dark_r, lf_r, doses_r, (dd, fd) = O.ref_fulllognorm(proj, darks, flats, method, usenorm, roi)
    refs = O.lognorm_refs(darks, flats, method, usenorm, roi)
    assert np.array_equal(refs.dark, dark_r)
    assert np.array_equal(refs.logflat, lf_r)
    assert refs.darkdose == dd and refs.flatdose == fd
    if usenorm:
        doses = np.array([O.frame_dose(proj[i], roi) for i in range(nproj)], np.float32)
        assert np.array_equal(doses, doses_r)
        dl = O.lognorm_doselog(doses, refs.darkdose)
    else:
        dl = np.zeros(1, np.float32)
    out = O.lognorm_apply(proj, refs.dark, refs.logflat, dl)
    assert np.array_equal(out, out_r)


@pytest.mark.parametrize("usenorm", [False, True])
@pytest.mark.parametrize("refs_present", [(4, 5), (0, 5), (4, 0)])
@pytest.mark.parametrize("method", ["ImageAverage", "ImageWeightedAverage"])
def test_fulllognorm_lut_bit_exact(ref_lib, usenorm, refs_present, method):
    """FullLogNorm with uselut=true: LogLUT of I - D (values at or below 0, above 65535, and
    exactly half way between integers included), with and without darks or flats."""
    rng = _rng(31)
    ndark, nflat = refs_present
    nproj, nv, nu = 11, 10, 24
    darks = np.round(rng.normal(100, 3, (4, nv, nu))).astype(np.float32)[:ndark]
    flats = (rng.poisson(30000, (5, nv, nu)) + 100).astype(np.float32)[:nflat]
    proj = (rng.poisson(20000, (nproj, nv, nu)) + 100).astype(np.float32)
    proj[0, 0, :5] = 50
    proj[1, 1, :3] = 70000.0
    proj[2, 2, :4] = [100.5, 101.5, 102.25, 65635.5]
    roi = (2, 2, 20, 9)
    out_r, _, _, _, _ = O.ref_fulllognorm(proj, darks, flats, method, usenorm, roi, uselut=True)
    refs = O.lognorm_refs(darks, flats, method, usenorm, roi)
    if usenorm:
        doses = np.array([O.frame_dose(proj[i], roi) for i in range(nproj)], np.float32)
        dl = O.lognorm_doselog(doses, refs.darkdose)
    else:
        dl = np.zeros(1, np.float32)
    out = O.lognorm_apply(proj, refs.dark, refs.logflat, dl, ndc=ndark > 0, nob=nflat > 0, uselut=True)
    assert np.array_equal(out.view(np.uint32), out_r.view(np.uint32))


@pytest.mark.parametrize("ftype", ["ram-lak", "shepp-logan", "hanning", "hamming", "butterworth"])
@pytest.mark.parametrize("nu,pd,cutoff", [(64, 2, 0.5), (50, 1, 0.35), (33, 0, 0.2)])
def test_projfilter(ref_lib, ftype, nu, pd, cutoff):
    rng = _rng(40)
    proj = rng.standard_normal((3, 5, nu)).astype(np.float32)
    plan = O.projfilter_plan(nu, ftype, cutoff, 2.0, True, 0.1, pd)
    out_r, filt_r, nfft = O.ref_projfilter(proj, ftype, cutoff, 2.0, True, 0.1, pd)
    assert nfft == plan.nfft
    assert np.array_equal(plan.filter, filt_r)
    out = O.projfilter(proj, plan)
    rel = np.sqrt(np.mean((out - out_r) ** 2) / np.mean(out_r ** 2))
    assert rel < 1e-6


def test_projfilter_bad_cutoff(ref_lib):
    with pytest.raises(ValueError):
        O.projfilter_plan(64, "hanning", 0.7)
    with pytest.raises(RuntimeError):
        O.ref_projfilter(np.zeros((1, 2, 64), np.float32), "hanning", 0.7)


@pytest.mark.parametrize("method", ["ImageSum", "ImageAverage", "ImageMedian", "ImageMin", "ImageMax",
                                    "ImageWeightedAverage"])
@pytest.mark.parametrize("n", [1, 4, 5])
def test_average(ref_lib, method, n):
    rng = _rng(50 + n)
    stack = np.round(rng.normal(1000, 30, (n, 6, 9))).astype(np.float32)
    assert np.array_equal(O.average(stack, method), O.average(stack, method, use_ref=True))


@pytest.mark.parametrize("shape", [(1, 5, 5), (3, 6, 7), (10, 33, 41), (20, 64, 64)])
def test_weighted_average_bit_exact(ref_lib, shape):
    """ImageWeightedAverage, FullLogNorm's default: 5x5 StdDevFilter weights with EdgeMirror
    edges, flat patches (sigma 0: weight 1/number of pixels), a bright row."""
    rng = _rng(sum(shape))
    st = rng.poisson(1000, shape).astype(np.float32)
    st[:, 2:5, 1:4] = 700.0
    st[0, 0, :] = 1e4
    a = O.average(st, "ImageWeightedAverage")
    assert np.array_equal(a.view(np.uint32), O.average(st, "ImageWeightedAverage", use_ref=True).view(np.uint32))


def test_frame_dose(ref_lib):
    rng = _rng(60)
    frame = rng.uniform(0, 100, (20, 30)).astype(np.float32)
    for roi in [(3, 2, 25, 18), (1, 1, 30, 20), (5, 5, 6, 7), (0, 3, 10, 9)]:
        r = np.asarray(roi, np.uintp)
        ref = O.ref().ref_frame_dose(O._p(frame), O._sz(30), O._p(r, O._SZ))
        assert O.frame_dose(frame, roi) == pytest.approx(ref, abs=0) or O.frame_dose(frame, roi) == ref


@pytest.mark.parametrize("detect", ["holes", "peaks", "both"])
@pytest.mark.parametrize("conn8", [True, False])
@pytest.mark.parametrize("sigma", [(0.0, 0.0), (0.05, 0.02)])
def test_morphspotclean_bit_exact(ref_lib, detect, conn8, sigma):
    rng = _rng(70)
    for t in range(6):
        h, w = rng.integers(5, 40, 2)  # the reference reads outside images of fewer than 5 rows
        img = rng.standard_normal((h, w)).astype(np.float32)
        if t % 2:
            img = np.round(img * 3).astype(np.float32)  # plateaus and ties
        e = int(rng.choice([3, 5, 9]))
        a = O.morphspotclean(img, detect, conn8, (0.5, 0.4), sigma, edge=e)
        b = O.morphspotclean(img, detect, conn8, (0.5, 0.4), sigma, edge=e, use_ref=True)
        assert np.array_equal(a, b)


def test_morphspotclean_clamp_infnan(ref_lib):
    rng = _rng(71)
    img = rng.standard_normal((12, 20)).astype(np.float32) * 5
    img[3, 4] = np.inf
    img[7, 9] = np.nan
    a = O.morphspotclean(img, "peaks", True, (0.5, 0.5), (0.0, 0.0), clamp=True, minlevel=-2, maxlevel=3,
                         removeinfnan=True)
    b = O.morphspotclean(img, "peaks", True, (0.5, 0.5), (0.0, 0.0), clamp=True, minlevel=-2, maxlevel=3,
                         removeinfnan=True, use_ref=True)
    assert np.array_equal(a, b)


def test_morphspotclean_module_defaults(ref_lib):
    """MorphSpotCleanModule's single-threaded path uses the cleaner's edge length 9, whatever
    `edgesmooth` says (MorphSpotCleanModule.cpp:142-181)."""
    rng = _rng(72)
    proj = (rng.standard_normal((3, 16, 24)) * 0.2 + 1).astype(np.float32)
    proj[:, 5, 7] = 5.0
    a = O.ref_morphspotclean_module(proj, edgesmooth=5)
    b = O.morphspotclean(proj, "peaks", False, (0.1, 0.1), (0.01, 0.01), edge=9)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [n for n in range(1, 31) if n != 28])
def test_wavelet_kernels_match_reference(ref_lib, n):
    """The dbN table equals the reference's float kernels: N <= 15 from the spectral
    factorisation (daub3 with the reference's sign of h[4]), N >= 16 kipl's own table values
    (less accurate than float, and the results follow them). daub28 is refused: its reference
    table is shorter than the filter."""
    import ctypes

    b, e, k = O.wavelet_kernel(f"daub{n}")
    th = np.zeros(64, np.float32)
    tg, sh, sg = th.copy(), th.copy(), th.copy()
    rb, re_ = ctypes.c_int(), ctypes.c_int()
    assert ref_lib.ref_wavelet_kernel(f"daub{n}".encode(), ctypes.byref(rb), ctypes.byref(re_), O._p(th), O._p(tg),
                                      O._p(sh), O._p(sg)) == 0
    K = re_.value - rb.value + 1
    assert (rb.value, re_.value) == (b, e)
    for ours, theirs in zip(k, (th, tg, sh, sg)):
        assert np.array_equal(ours, theirs[:K])


def test_daub28_refused():
    import ctypes

    from imagingsuite_b200 import _lib as L

    taps = np.zeros(4 * 56, np.float32)
    b, e = ctypes.c_int(), ctypes.c_int()
    assert L.lib().mr_wavelet_kernel(b"daub28", ctypes.byref(b), ctypes.byref(e), O._p(taps)) == L.MR_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        O.wavelet_kernel("daub28")


@pytest.mark.parametrize("name,levels,sigma", [("daub2", 1, 0.05), ("daub3", 3, 0.02), ("daub7", 2, 0.1),
                                               ("daub15", 2, 0.05), ("daub5", 3, 0.2), ("daub20", 2, 0.05),
                                               ("daub30", 2, 0.1)])
def test_stripefilter_bit_exact(ref_lib, name, levels, sigma):
    rng = _rng(90)
    for _ in range(3):
        h, w = rng.integers(70, 140, 2)
        s = rng.standard_normal((h, w)).astype(np.float32)
        assert np.array_equal(O.stripefilter(s, name, levels, sigma), O.stripefilter(s, name, levels, sigma, use_ref=True))


def test_waveletringclean_bit_exact(ref_lib):
    rng = _rng(91)
    proj = rng.standard_normal((80, 3, 70)).astype(np.float32)
    assert np.array_equal(O.waveletringclean(proj, "daub7", 2, 0.1), O.waveletringclean(proj, "daub7", 2, 0.1, use_ref=True))


@pytest.mark.parametrize("plane", [1, 4])
@pytest.mark.parametrize("roi", [None, (2, 1, 9, 6), (9, 6, 2, 1)])
def test_slices_u16_matches_reference(ref_lib, plane, roi):
    """Slice serialisation (ExtractSlice + ImageCaster<unsigned short, float>) restated in C,
    against the reference's own templates: planes XY and YZ, ROIs (also reversed), the clamps
    at the gray interval, infinities and NaN."""
    rng = np.random.default_rng(plane * 7 + (0 if roi is None else 1))
    vol = (rng.standard_normal((12, 10, 14)) * 0.02).astype(np.float32)
    vol[0, 0, 0], vol[1, 2, 3], vol[2, 3, 4], vol[3, 4, 5] = np.inf, -np.inf, np.nan, 0.05
    nsl = 12 if plane == 1 else 14
    for lo, hi in ((-0.03, 0.04), (0.0, 1e-3), (-1.0, 1.0)):
        got = O.slices_u16(vol, plane, 1, nsl - 2, lo, hi, roi)
        exp = O.ref_slices_u16(vol, plane, 1, nsl - 2, lo, hi, roi)
        assert np.array_equal(got, exp)


def _weight_cases(trailing_repeats: bool):
    rng = _rng(70)
    cases = []
    for n in (1, 2, 3, 5, 10, 360, 375, 1125):
        cases.append((np.arange(n, dtype=np.float32) * np.float32(180.0 / n), (0, 180), False))
        cases.append((np.arange(n, dtype=np.float32) * np.float32(360.0 / n), (0, 360), False))
        cases.append((np.arange(n, dtype=np.float32) * np.float32(180.0 / max(n - 1, 1)), (0, 180), False))
    g = np.float32(0.5 * (1 + np.sqrt(5.0)))
    for n, arc in ((50, 180.0), (100, 360.0)):
        i = np.arange(n, dtype=np.float32)
        cases.append((np.fmod(i * g * np.float32(arc), np.float32(arc)).astype(np.float32), (0, arc), True))
    cases.append((np.linspace(0, 120, 40).astype(np.float32), (0, 120), False))  # short arc
    cases.append((rng.permutation(np.arange(37, dtype=np.float32) * np.float32(5.0)), (0, 180), False))
    cases.append((np.array([0, 0, 10, 20, 20, 20, 30, 190, 200], np.float32), (0, 360), False))  # repeats inside
    if trailing_repeats:
        # a run of repeated keys at the end of the list: the reference reads past the end of its
        # multimap there (its result depends on memory behind the container), the restatements
        # end the run at the list end
        cases.append((np.repeat(np.arange(20, dtype=np.float32) * 9.0, 3), (0, 180), False))
        cases.append((np.concatenate([np.arange(30, dtype=np.float32) * 6.0, np.full(3, 174.0, np.float32)]), (0, 180),
                      False))
    return cases


def test_compute_weights_matches_reference(ref_lib):
    """ComputeWeights (ReconHelpers.cpp:365-488): the oracle's restatement and the library's host
    function (mr_compute_weights) against the reference on uniform half and full arcs (with and
    without the end angle), golden-section scans, a short arc, unsorted and repeated angles."""
    for ang, arc, gold in _weight_cases(False):
        ra, rw = O.compute_weights(ang, arc, gold, use_ref=True)
        for lib in (False, True):
            oa, ow = O.compute_weights(ang, arc, gold, use_lib=lib)
            assert np.array_equal(oa.view(np.uint32), ra.view(np.uint32)), (len(ang), arc, gold, lib)
            assert np.array_equal(ow.view(np.uint32), rw.view(np.uint32)), (len(ang), arc, gold, lib)


def test_compute_weights_library_matches_oracle():
    for ang, arc, gold in _weight_cases(True):
        oa, ow = O.compute_weights(ang, arc, gold)
        la, lw = O.compute_weights(ang, arc, gold, use_lib=True)
        assert np.array_equal(oa.view(np.uint32), la.view(np.uint32)) and np.array_equal(ow.view(np.uint32),
                                                                                         lw.view(np.uint32))
    # one projection per degree over a full turn: the weights sum to 1
    _, w = O.compute_weights(np.arange(360, dtype=np.float32), (0, 360))
    assert abs(float(w.sum()) - 1.0) < 1e-3


def test_reference_fdkbp_double_row_window(ref_lib):
    """The factory's FDKbp (fdkbp.cpp) lowers its CBCT row window by 8 without the single
    version's zero check (`if (CBCT_roi[1]-8>=0)` on a size_t): for a window that starts within
    8 rows of the detector top the index wraps and every sample misses the detector, so the
    volume stays 0. With the window further down it reconstructs (its projection scale also
    carries 1/nproj). This pins why that module is not offered as a drop-in."""
    rng = _rng(80)
    nproj, nu = 8, 32
    ang = (np.arange(nproj) * 45.0).astype(np.float32)
    w = np.ones(nproj, np.float32)
    proj = (rng.random((nproj, 24, nu)) + 0.5).astype(np.float32)
    g = O.fdk_geom(250.0, 500.0, (15.5, 11.5), 15.5, (0.2, 0.2), (0.1, 0.1, 0.1))
    assert not O.ref_fdk_double(proj, ang, w, g).any() and O.fdk(proj, ang, w, g, use_ref=True).any()
    proj = (rng.random((nproj, 64, nu)) + 0.5).astype(np.float32)
    g = O.fdk_geom(250.0, 500.0, (15.5, 60.0), 15.5, (0.2, 0.2), (0.05, 0.05, 0.05))
    assert O.ref_fdk_double(proj, ang, w, g).any()


def test_projection_lists_format_like_the_stream(ref_lib):
    """The engine's angle / weight lists: float arithmetic, then the default ostream format of
    each value, which the module helper reproduces."""
    import ctypes

    from imagingsuite_b200 import modules as M

    rng = _rng(90)
    ang = np.concatenate([np.arange(375, dtype=np.float32) * np.float32(180.0 / 375),
                          rng.uniform(-1e-6, 1e6, 50).astype(np.float32), np.array([0.0, -0.0, 1e-5], np.float32)])
    w = rng.uniform(1e-4, 2.0, ang.size).astype(np.float32)
    lists = M.projection_lists(ang, w, rotation=0.25, resolution=0.139)
    buf = ctypes.create_string_buffer(64)
    f32 = np.float32
    rw = f32(1.0) / (f32(0.139) * f32(0.1))
    exp_a = []
    exp_w = []
    for a, b in zip(ang, w):
        ref_lib.ref_stream_float(ctypes.c_float(f32(a) + f32(0.25)), buf, ctypes.c_size_t(64))
        exp_a.append(buf.value.decode())
        ref_lib.ref_stream_float(ctypes.c_float(f32(b) * rw), buf, ctypes.c_size_t(64))
        exp_w.append(buf.value.decode())
    assert lists["angles"] == " ".join(exp_a) + " " and lists["weights"] == " ".join(exp_w) + " "


@pytest.mark.parametrize("method,expected", [("ImageSum", 15.0), ("ImageAverage", 3.0), ("ImageWeightedAverage", 3.0),
                                             ("ImageMedian", 3.0), ("ImageMin", 1.0), ("ImageMax", 5.0)])
def test_average_known_answers(method, expected):
    """The reference's AverageImage_Processing known answers (core/algorithms/UnitTests/
    tImagingAlgorithms/tst_testImagingAlgorithms.cpp:209-249): five constant 11x11 frames of
    1..5; the weighted average falls back to equal weights (sigma 0 everywhere)."""
    stack = np.repeat(np.arange(1, 6, dtype=np.float32)[:, None, None], 121, axis=1).reshape(5, 11, 11)
    out = O.average(stack, method)
    assert np.all(out == np.float32(expected))


def test_average_python_binding_cases():
    """testBindAverageImage.py (core/algorithms/UnitTests/python): average, min, max and median
    along the frame axis of x + 10 y + 100 z on an 11 x 10 x 12 grid are exact."""
    a, b, c = np.linspace(0, 9, 10), np.linspace(0, 10, 11), np.linspace(0, 11, 12)
    x, y, z = np.meshgrid(a, b, c)
    img = (x + y * 10 + z * 100).astype(np.float32)
    assert np.array_equal(O.average(img, "ImageAverage"), img.mean(axis=0, dtype=np.float64).astype(np.float32))
    assert np.array_equal(O.average(img, "ImageMin"), img.min(axis=0))
    assert np.array_equal(O.average(img, "ImageMax"), img.max(axis=0))
    assert np.array_equal(O.average(img, "ImageMedian"), np.median(img, axis=0).astype(np.float32))


@pytest.mark.parametrize("refs_present", [(0, 5), (4, 0)])
@pytest.mark.parametrize("usenorm", [False, True])
def test_fulllognorm_without_darks_or_flats(ref_lib, refs_present, usenorm):
    """The exact path's branches without darks (I alone) or without flats (-log(I - D) + dose,
    NormPlugins.cpp:482-540), restated bit for bit."""
    rng = _rng(32)
    ndark, nflat = refs_present
    nproj, nv, nu = 9, 10, 24
    darks = np.round(rng.normal(100, 3, (4, nv, nu))).astype(np.float32)[:ndark]
    flats = (rng.poisson(30000, (5, nv, nu)) + 100).astype(np.float32)[:nflat]
    proj = (rng.poisson(20000, (nproj, nv, nu)) + 100).astype(np.float32)
    proj[0, 0, :5] = 50
    roi = (2, 2, 20, 9)
    out_r, _, _, _, _ = O.ref_fulllognorm(proj, darks, flats, "ImageAverage", usenorm, roi)
    refs = O.lognorm_refs(darks, flats, "ImageAverage", usenorm, roi)
    if usenorm:
        doses = np.array([O.frame_dose(proj[i], roi) for i in range(nproj)], np.float32)
        dl = O.lognorm_doselog(doses, refs.darkdose)
    else:
        dl = np.zeros(1, np.float32)
    out = O.lognorm_apply(proj, refs.dark, refs.logflat, dl, ndc=ndark > 0, nob=nflat > 0)
    assert np.array_equal(out.view(np.uint32), out_r.view(np.uint32))
