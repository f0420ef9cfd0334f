"""The oracle restatement against golden outputs of the reference itself (tests/golden,
made by tests/golden/make_golden.py from the reference compiled from source) and against the
reference's own golden statistics. Runs without the reference library."""
import os

import numpy as np
import pytest

import oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.npz"))


def test_morphspotclean_python_test_statistics():
    # core/algorithms/UnitTests/python/testBindMorphSpotClean.py: Holes+Replace,
    # process(ci, 0.3, 0.01) -> mean 5.89322, std 22.368868 (rel 1e-4)
    out = O.morphspotclean(G["spot_input"], "holes", True, (0.3, 0.3), (0.01, 0.01), edge=9)
    assert np.isclose(out.mean(), 5.89322, rtol=1e-4)
    assert np.isclose(out.std(), 22.368868, rtol=1e-4)
    out2 = O.morphspotclean(G["spot_input"], "holes", True, (0.3, 0.2), (0.01, 0.0005), edge=9)
    assert np.isclose(out2.mean(), 5.89322, rtol=1e-4)
    assert np.isclose(out2.std(), 22.368868, rtol=1e-4)


@pytest.mark.parametrize("key,args", [
    ("spot_holes_03_001", ("holes", True, (0.3, 0.3), (0.01, 0.01))),
    ("spot_holes_03_02", ("holes", True, (0.3, 0.2), (0.01, 0.0005))),
    ("spot_peaks_conn4_thr", ("peaks", False, (0.1, 0.1), (0.0, 0.0))),
    ("spot_both_conn8_sig", ("both", True, (1.0, 1.0), (0.05, 0.05))),
])
def test_morphspotclean_golden(key, args):
    assert np.array_equal(O.morphspotclean(G["spot_input"], *args, edge=9), G[key])


def test_morphspotclean_kat_fixture():
    """The 7x7 fixture of tst_testImagingAlgorithms.cpp. The reference computes 1.6 (not the
    1.8 its QtTest expects for the peak): the mirrored padding rows and the median-smoothed
    padded border cap the reconstruction at 1.6. The restatement equals the reference."""
    for d in ("holes", "peaks", "both"):
        out = O.morphspotclean(G["kat_input"], d, True, (1.0, 1.0), (0.05, 0.05), edge=9)
        assert np.array_equal(out, G[f"kat_{d}"])
    assert abs(G["kat_holes"].flat[24] - 1.6) < 1e-4 and G["kat_holes"].flat[10] == 100.0
    assert G["kat_peaks"].flat[24] == 0.0 and abs(G["kat_peaks"].flat[10] - 1.6) < 1e-4


def test_lognorm_golden():
    refs = O.lognorm_refs(G["lognorm_darks"], G["lognorm_flats"], "ImageAverage", True, (2, 1, 30, 7))
    c = G["lognorm_counts"]
    doses = np.array([O.frame_dose(c[i], (2, 1, 30, 7)) for i in range(c.shape[0])], np.float32)
    out = O.lognorm_apply(c, refs.dark, refs.logflat, O.lognorm_doselog(doses, refs.darkdose))
    assert np.array_equal(out, G["lognorm_out"])


def test_projfilter_golden():
    p = G["filter_input"]
    out = O.projfilter(p, O.projfilter_plan(p.shape[2], "hanning", 0.5, 1.0, True, 0.1, 2))
    assert np.sqrt(np.mean((out - G["filter_hanning_out"]) ** 2) / np.mean(G["filter_hanning_out"] ** 2)) < 1e-6


def test_bp_parallel_golden():
    out = O.bp_parallel(G["filter_input"], G["bp_angles"], G["bp_weights"], 15.5, buffersize=5)
    assert np.array_equal(out, G["bp_out"])


def test_fdk_golden():
    g = O.fdk_geom(300.0, 600.0, (15.5, 11.5), 15.7, (0.2, 0.2), (0.1, 0.1, 0.1))
    assert np.array_equal(O.fdk(G["fdk_input"], G["fdk_angles"], G["fdk_weights"], g), G["fdk_out"])


def test_stripefilter_python_test_mse():
    # core/algorithms/UnitTests/python/testBindStripeFilter.py: daub7, 2 levels, sigma 0.1,
    # VerticalComponentFFT -> mse(sino, out) == 1.8129678e-05 (rel 1e-6)
    wood = G["wood_input"]
    out = O.stripefilter(wood, "daub7", 2, 0.1)
    mse = float(((wood - out) ** 2).mean())
    assert np.isclose(mse, 1.8129678e-05, rtol=1e-6)


def test_stripefilter_golden_crops():
    crop = G["wood_input"][100:260, 50:250]
    assert np.array_equal(O.stripefilter(crop, "daub15", 2, 0.05), G["wood_crop_daub15_2_005"])
    assert np.array_equal(O.stripefilter(crop, "daub3", 3, 0.02), G["wood_crop_daub3_3_002"])
