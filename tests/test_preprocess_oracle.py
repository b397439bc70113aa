"""The preprocessing oracle against the reference's own outputs (golden
fixtures made by tests/golden/make_preprocess_golden.py) and the
third-party contracts it restates against the libraries themselves."""
from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import preprocess_oracle as PO  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "pp_*.npz")))


def load_case(path):
    z = np.load(path)
    cfg = json.loads(str(z["cfg"]))
    bg = z["background_in"]
    return z, cfg, (bg if bg.size else None), float(z["override_thresh"])


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[3:-4] for p in FIXTURES])
def test_oracle_matches_reference_golden(path):
    z, cfg, bg, ovt = load_case(path)
    r = PO.preprocess_image(z["raw"], cfg, background=bg, override_thresh=ovt)
    assert np.array_equal(bits(r["background"]), bits(z["background"]))
    assert np.array_equal(r["thresholded"], z["thresholded"])
    assert np.array_equal(r["labels_unfiltered"], z["labels_unfiltered"])
    assert np.array_equal(r["filt_img"], z["filt_img"])
    assert np.array_equal(r["filt_labels"], z["filt_labels"])
    cen = np.array([[c[0], c[1][0], c[1][1], c[2]] for c in r["centers"]], np.float64).reshape(-1, 4)
    assert np.array_equal(bits(cen), bits(z["centers"]))
    assert np.array_equal(bits(r["blurred"]), bits(z["blurred"]))


def test_fixture_set_covers_the_paths():
    names = {os.path.basename(p)[3:-4] for p in FIXTURES}
    assert {"adaptive_bgmedian", "percentile", "fixed_given_bg", "override", "no_components",
            "all_small", "one_centre", "u16_wrap", "many_values"} <= names


def test_median_restatement_matches_scipy():
    nd = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(0)
    for _ in range(25):
        ny, nx = (int(v) for v in rng.integers(1, 40, 2))
        s = int(rng.integers(1, 30))
        if (ny > 1 and s >= 8 * ny) or (nx > 1 and s >= 8 * nx):
            continue
        a = rng.integers(0, 40, (ny, nx)).astype(np.float64) + rng.random((ny, nx)) * (s % 2)
        assert np.array_equal(PO.median_filter(a, s), nd.median_filter(a, size=s))


def test_gaussian_restatement_matches_scipy_bitwise():
    nd = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(1)
    for _ in range(20):
        ny, nx = (int(v) for v in rng.integers(1, 70, 2))
        a = rng.integers(0, 65535, (ny, nx)).astype(np.float64) * (rng.random((ny, nx)) < 0.3)
        sigma = float(rng.choice([1.0, 1.3, 2.7, 0.6, 3.0, 5.5]))
        assert np.array_equal(bits(PO.gaussian_blur(a, sigma)), bits(nd.gaussian_filter(a, sigma)))


def test_label_order_matches_opencv():
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(2)
    for t in range(20):
        ny, nx = (int(v) for v in rng.integers(1, 200, 2)) if t < 18 else (1024, 1536)
        b = (rng.random((ny, nx)) < rng.choice([0.05, 0.3, 0.6])).astype(np.uint16) * 7
        n, lab, st, _ = cv2.connectedComponentsWithStats(
            cv2.threshold(b, 0, 255, cv2.THRESH_BINARY)[1].astype(np.uint8), 8, cv2.CV_32S)
        labels, bboxes, areas, nl = PO.connected_components(b)
        assert nl == n
        assert np.array_equal(labels, lab)
        assert np.array_equal(areas, st[1:, cv2.CC_STAT_AREA])
        assert np.array_equal(bboxes, st[1:, :cv2.CC_STAT_HEIGHT + 1])


def test_u16_cast_matches_numpy():
    v = np.array([2147483647.5, 2147483648.0, 3e9, -2147483648.0, -2147483649.0, np.nan, np.inf,
                  -np.inf, 65535.999, 131071.5, -0.0, -0.7, 70000.7, 65536.0, 12.9])
    with np.errstate(invalid="ignore"):
        assert np.array_equal(PO.u16_cast(v), v.astype(np.uint16))


def test_threshold_statistics_match_numpy():
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 10, 1001, 4096):
        a = np.maximum(rng.normal(3, 4, n), 0.0)
        for pct in (0.0, 12.5, 50.0, 90.0, 99.2, 100.0):
            assert PO.percentile_linear(a, pct) == float(np.percentile(a, pct))
        nz = a[a > 0]
        if nz.size:
            med = float(np.median(nz))
            want = max(med + 4.0 * (1.4826 * float(np.median(np.abs(nz - med)))), 1.0)
            assert PO.noise_floor(a) == want
