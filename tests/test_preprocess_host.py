"""Host-side helpers of the preprocessing drop-in (no GPU): blur width,
background files, enhancement, Gaussian weights -- against the oracle's
restatement of the reference (laue_index/preprocess.py)."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import preprocess_oracle as PO  # noqa: E402
from lauematching_b200 import preprocess as PP  # noqa: E402


def test_blur_width_matches_the_reference_formula():
    rng = np.random.default_rng(0)
    for n in (0, 1, 2, 3, 17, 500):
        for spacing in (0.5, 3.0, 40.0):
            pts = rng.random((n, 2)) * 2048
            if n > 3:
                pts[3] = pts[2]  # a duplicate centre: nearest distance 0
            centres = [[i + 1, (float(x), float(y)), 10] for i, (x, y) in enumerate(pts)]
            for px, dist, osp in ((0.2, 0.513, 0.4), (0.0004, 0.513, spacing), (0.0, 0.5, 0.4)):
                assert PP.calculate_gaussian_sigma(centres, px, dist, osp) == \
                    PO.gaussian_sigma(centres, px, dist, osp)


def test_gaussian_weights_are_the_oracle_weights():
    for sigma in (0.3, 1.0, 1.7, 3.0, 11.2):
        w, r = PP.gaussian_weights(sigma)
        wo, ro = PO.gaussian_kernel(sigma)
        assert r == ro and np.array_equal(w, wo)


def test_background_file_rules(tmp_path):
    ny, nx = 6, 5
    good = tmp_path / "bg.bin"
    arr = np.arange(ny * nx, dtype=np.float64).reshape(ny, nx)
    arr.tofile(good)
    assert np.array_equal(PP.load_background(str(good), nx, ny), arr)
    bad = tmp_path / "short.bin"
    arr[:2].tofile(bad)
    assert not PP.load_background(str(bad), nx, ny).any()
    assert not PP.load_background(str(tmp_path / "missing.bin"), nx, ny).any()
    assert not PP.load_background("", nx, ny).any()


def test_enhancement_is_the_identity_without_scikit_image():
    a = np.ones((3, 4))
    assert PP.enhance_image(a, denoise=True, contrast=True, edge=True) is a


def test_module_functions_follow_the_reference_names():
    names = {"compute_background", "load_background", "enhance_image", "find_connected_components",
             "filter_small_components", "calculate_gaussian_sigma", "preprocess_image",
             "Preprocessor"}
    assert names <= set(PP.__all__)


def test_zero_radius_background_needs_no_device():
    a = np.arange(12.0).reshape(3, 4)
    assert not PP.compute_background(a, 0, 1).any()
    assert not PP.compute_background(a, 101, 0).any()


def test_config_from_a_parameter_file_follows_the_image_server_rules():
    txt = ("NrPxX 1024\n# ThresholdMethod fixed\nP_Array 0 0 0.61  # metres\n"
           "ThresholdMethod Percentile\nThreshold 12.5\nThresholdPercentile 99\n"
           "MinArea bad\nFilterRadius 51\nNMeadianPasses 2\nOrientationSpacing 0.25\n"
           "PxX 0.0002\nBackgroundFile /tmp/bg.bin\nLatticeParameter 0.3 0.3 0.3 90 90 90\n")
    cfg = PP.config_from_params_text(txt)
    assert cfg["nr_px_x"] == 1024 and cfg["nr_px_y"] == 2048
    assert cfg["distance"] == 0.61 and cfg["px_x"] == 0.0002
    assert cfg["threshold_method"] == "percentile" and cfg["threshold_value"] == 12.5
    assert cfg["threshold_percentile"] == 99.0 and cfg["min_area"] == 10  # malformed: default
    assert cfg["filter_radius"] == 51 and cfg["median_passes"] == 2
    assert cfg["orientation_spacing"] == 0.25 and cfg["background_file"] == "/tmp/bg.bin"
    assert PP.config_from_params_text("")["threshold_method"] == "adaptive"
