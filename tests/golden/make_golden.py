"""Generate the golden fixtures in tests/golden from the reference itself.

Runs the reference's own modules, compiled from the reference sources into
oracle/_ref/libmuhrec_ref.so (make -C oracle ref), on:

* the reference's test images core/algorithms/UnitTests/data/spotprojection_0001.tif and
  woodsino_0200.tif (read with PIL), with the settings of the reference's own python tests
  (core/algorithms/UnitTests/python/testBindMorphSpotClean.py, testBindStripeFilter.py);
* the 7x7 fixture of core/algorithms/UnitTests/tImagingAlgorithms/tst_testImagingAlgorithms.cpp:54-73;
* small seeded cases of FullLogNorm, ProjectionFilterSingle, MultiProjectionBPparallel, FDKbp_single
  and LinearForwardProjector (the Joseph projector).

usage: python tests/golden/make_golden.py <reference root>
   (or set MUHREC_REFERENCE to the reference checkout)
The fixtures are committed; the tests never read the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def tiff(path):
    from PIL import Image

    return np.array(Image.open(path)).astype(np.float32)


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("MUHREC_REFERENCE")
    if not ref_root or not os.path.isdir(ref_root):
        sys.exit("make_golden.py: give the reference checkout as the argument or in MUHREC_REFERENCE")
    data = os.path.join(ref_root, "core", "algorithms", "UnitTests", "data")
    out = {}

    # MorphSpotClean on the reference's spot projection (python test settings)
    spot = tiff(os.path.join(data, "spotprojection_0001.tif"))
    out["spot_input"] = spot
    out["spot_holes_03_001"] = O.morphspotclean(spot, "holes", True, (0.3, 0.3), (0.01, 0.01), edge=9, use_ref=True)
    out["spot_holes_03_02"] = O.morphspotclean(spot, "holes", True, (0.3, 0.2), (0.01, 0.0005), edge=9, use_ref=True)
    out["spot_peaks_conn4_thr"] = O.morphspotclean(spot, "peaks", False, (0.1, 0.1), (0.0, 0.0), edge=9, use_ref=True)
    out["spot_both_conn8_sig"] = O.morphspotclean(spot, "both", True, (1.0, 1.0), (0.05, 0.05), edge=9, use_ref=True)

    # StripeFilter on the reference's sinogram (testBindStripeFilter.py: daub7, 2 levels, sigma 0.1)
    wood = tiff(os.path.join(data, "woodsino_0200.tif"))
    out["wood_input"] = wood
    crop = wood[100:260, 50:250].copy()
    out["wood_crop_daub15_2_005"] = O.stripefilter(crop, "daub15", 2, 0.05, use_ref=True)
    out["wood_crop_daub3_3_002"] = O.stripefilter(crop, "daub3", 3, 0.02, use_ref=True)

    # the 7x7 KAT fixture
    holes = (np.arange(49, dtype=np.float32) / np.float32(10.0)).reshape(7, 7)
    holes.flat[24] = 0.0
    holes.flat[10] = 100.0
    out["kat_input"] = holes
    for d in ("holes", "peaks", "both"):
        out[f"kat_{d}"] = O.morphspotclean(holes, d, True, (1.0, 1.0), (0.05, 0.05), edge=9, use_ref=True)

    # seeded small cases of the other modules
    rng = np.random.default_rng(2024)
    nproj, nv, nu = 12, 8, 32
    darks = np.round(rng.normal(100, 3, (3, nv, nu))).astype(np.float32)
    flats = (rng.poisson(30000, (4, nv, nu)) + 100).astype(np.float32)
    counts = (rng.poisson(12000, (nproj, nv, nu)) + 100).astype(np.float32)
    out["lognorm_darks"], out["lognorm_flats"], out["lognorm_counts"] = darks, flats, counts
    out["lognorm_out"] = O.ref_fulllognorm(counts, darks, flats, "ImageAverage", True, (2, 1, 30, 7))[0]
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    out["filter_input"] = proj
    out["filter_hanning_out"] = O.ref_projfilter(proj, "hanning", 0.5, 1.0, True, 0.1, 2)[0]
    ang = (np.arange(nproj) * 15.0).astype(np.float32)
    w = np.full(nproj, np.float32(np.pi / nproj))
    out["bp_angles"], out["bp_weights"] = ang, w
    out["bp_out"] = O.bp_parallel(proj, ang, w, 15.5, buffersize=5, use_ref=True)
    fproj = rng.standard_normal((6, 24, 32)).astype(np.float32)
    fang = (np.arange(6) * 60.0).astype(np.float32)
    fw = np.full(6, np.float32(0.5))
    out["fdk_input"], out["fdk_angles"], out["fdk_weights"] = fproj, fang, fw
    g = O.fdk_geom(300.0, 600.0, (15.5, 11.5), 15.7, (0.2, 0.2), (0.1, 0.1, 0.1))
    out["fdk_out"] = O.fdk(fproj, fang, fw, g, use_ref=True)

    # LinearForwardProjector (Joseph) on a phantom slice and a random slice
    import torch

    from imagingsuite_b200 import phantom

    ph = phantom.voxelize_torch(phantom.ellipsoids(1005), 64, 1, "cpu", supersample=2)[0].numpy()
    jang = np.sort(rng.uniform(0, 180, 45)).astype(np.float32)
    out["joseph_slices"] = np.stack([ph, rng.standard_normal((64, 64)).astype(np.float32)])
    out["joseph_angles"] = jang
    out["joseph_ref"] = np.stack([O.ref_joseph_project(s_, jang) for s_ in out["joseph_slices"]])

    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_outputs.npz"), sum(v.nbytes for v in out.values()), "bytes raw")


if __name__ == "__main__":
    main(*sys.argv[1:])
