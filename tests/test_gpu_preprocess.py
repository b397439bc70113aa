"""Device preprocessing against the reference's own outputs (golden fixtures
from tests/golden/make_preprocess_golden.py) and the oracle restatement."""
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

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "pp_*.npz")))


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def centres_array(centers):
    return np.array([[c[0], c[1][0], c[1][1], c[2]] for c in centers], np.float64).reshape(-1, 4)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[3:-4] for p in FIXTURES])
def test_preprocess_image_is_the_reference_bit_for_bit(path):
    from lauematching_b200 import preprocess as PP
    z = np.load(path)
    cfg = json.loads(str(z["cfg"]))
    bg = z["background_in"] if z["background_in"].size else None
    r = PP.preprocess_image(z["raw"], cfg, background=bg, override_thresh=float(z["override_thresh"]),
                            return_intermediates=True)
    assert np.array_equal(bits(r["background"]), bits(z["background"]))
    assert np.array_equal(r["thresholded"], z["thresholded"])
    assert np.array_equal(r["labels_unfiltered"], z["labels_unfiltered"])
    assert np.array_equal(r["filt_img"], z["filt_img"])
    assert np.array_equal(r["filt_labels"], z["filt_labels"])
    assert np.array_equal(bits(centres_array(r["centers"])), bits(z["centers"]))
    assert np.array_equal(bits(r["blurred"]), bits(z["blurred"]))
    # the four-tuple form returns the same arrays
    b, fi, fl, cen = PP.preprocess_image(z["raw"], cfg, background=bg,
                                         override_thresh=float(z["override_thresh"]))
    assert np.array_equal(bits(b), bits(z["blurred"]))
    assert np.array_equal(fi, z["filt_img"]) and np.array_equal(fl, z["filt_labels"])
    assert np.array_equal(bits(centres_array(cen)), bits(z["centers"]))


@pytest.mark.parametrize("shape,size,kind", [
    ((64, 48), 7, "int"), ((50, 61), 8, "float"), ((33, 40), 15, "wide"),
    ((300, 290), 5, "float"), ((7, 9), 31, "int"), ((1, 40), 5, "int"), ((40, 1), 6, "float"),
    ((128, 128), 1, "float"),
])
def test_median_is_exact_for_every_rank_depth(shape, size, kind):
    """Ranks of one, two and three 8-bit digits (up to 87000 distinct values),
    even and odd windows, windows wider than the frame, single rows/columns."""
    from lauematching_b200 import preprocess as PP
    rng = np.random.default_rng(sum(shape) * 31 + size)
    if kind == "int":
        a = rng.integers(0, 40, shape).astype(np.float64)
    elif kind == "wide":
        a = rng.integers(0, 100000, shape).astype(np.float64)
    else:
        a = rng.random(shape) * 1000.0
    got = PP.compute_background(a, size, 1)
    assert np.array_equal(bits(got), bits(PO.median_filter(a, size)))


def test_median_two_passes_and_input_types():
    from lauematching_b200 import preprocess as PP
    rng = np.random.default_rng(5)
    a = rng.integers(0, 3000, (96, 80)).astype(np.uint16)
    want = PO.compute_background(a, 9, 2)
    for arr in (a, a.astype(np.float32), a.astype(np.float64), a.astype(np.int32)):
        assert np.array_equal(bits(PP.compute_background(arr, 9, 2)), bits(want))
    assert not PP.compute_background(a, 0, 1).any()


def test_median_refuses_windows_of_eight_frame_sides():
    from lauematching_b200 import preprocess as PP
    from lauematching_b200._lib import LmbError
    with pytest.raises(LmbError):
        PP.compute_background(np.ones((4, 30)), 32, 1)


def test_full_size_median_radius_101_on_sampled_pixels():
    """2048^2 detector frame, the reference's default window (101): each
    sampled pixel equals the exact median of its mirrored window."""
    from lauematching_b200 import preprocess as PP, synth
    rng = np.random.default_rng(11)
    raw = synth.raw_frame(2048, 2048, rng, n_spots=400)
    bg = PP.compute_background(raw, 101, 1)
    s, lo = 101, 50
    pad = np.pad(raw, lo, mode="symmetric")
    ys = np.concatenate([rng.integers(0, 2048, 150), [0, 2047, 0, 2047, 49, 50, 1998]])
    xs = np.concatenate([rng.integers(0, 2048, 150), [0, 2047, 2047, 0, 1998, 51, 49]])
    for y, x in zip(ys, xs):
        w = pad[y:y + s, x:x + s].ravel()
        assert bg[y, x] == np.partition(w, (s * s) // 2)[(s * s) // 2], (y, x)


@pytest.mark.parametrize("method,extra,integer", [
    ("adaptive", {}, True), ("percentile", {"threshold_percentile": 99.5}, True),
    ("fixed", {"threshold_value": 40.0}, False), ("otsu", {}, True),
    # fractional values: the radix selection instead of the value histogram
    ("adaptive", {}, False), ("percentile", {"threshold_percentile": 97.25}, False)])
def test_full_size_frame_against_the_oracle(method, extra, integer):
    """2048^2 frames with a given background (the image server's flow)."""
    from lauematching_b200 import preprocess as PP, synth
    rng = np.random.default_rng(sum(map(ord, method)) + int(integer))
    raw = synth.raw_frame(2048, 2048, rng, n_spots=600, integer=integer)
    yy, xx = np.mgrid[0:2048, 0:2048]
    bg = 100.0 + 0.02 * yy + 0.01 * xx
    if integer:  # integer frames minus an integer background: the value-histogram path
        bg = np.rint(bg)
    cfg = dict(nr_px_x=2048, nr_px_y=2048, filter_radius=101, median_passes=1,
               threshold_method=method, threshold_value=0.0, threshold_percentile=90.0,
               min_area=10, px_x=0.2, distance=0.513, orientation_spacing=0.4)
    cfg.update(extra)
    got = PP.preprocess_image(raw, cfg, background=bg, return_intermediates=True)
    want = PO.preprocess_image(raw, cfg, background=bg)
    assert np.array_equal(got["thresholded"], want["thresholded"])
    assert np.array_equal(got["labels_unfiltered"], want["labels_unfiltered"])
    assert np.array_equal(got["filt_labels"], want["filt_labels"])
    assert np.array_equal(got["filt_img"], want["filt_img"])
    assert np.array_equal(bits(centres_array(got["centers"])), bits(centres_array(want["centers"])))
    assert np.array_equal(bits(got["blurred"]), bits(want["blurred"]))
    assert len(got["centers"]) > 50


def test_components_and_filter_helpers_match_opencv_order():
    from lauematching_b200 import preprocess as PP
    rng = np.random.default_rng(7)
    for shape in ((1, 1), (1, 57), (64, 1), (301, 257), (1024, 1536)):
        t = ((rng.random(shape) < 0.4) * rng.integers(1, 900, shape)).astype(np.uint16)
        labels, bboxes, areas, n = PP.find_connected_components(t)
        wl, wb, wa, wn = PO.connected_components(t)
        assert n == wn and np.array_equal(labels, wl)
        assert np.array_equal(bboxes, wb) and np.array_equal(areas, wa)
        fi, fl, cen = PP.filter_small_components(t, labels, bboxes, areas, n, min_area=3)
        wfi, wfl, wcen = PO.filter_small_components(t, wl, wb, wa, wn, min_area=3)
        assert np.array_equal(fi, wfi) and np.array_equal(fl, wfl)
        assert np.array_equal(bits(centres_array(cen)), bits(centres_array(wcen)))


def test_blur_width_from_the_closest_pair():
    """Many centres, some closer than the cell grid's side and some not."""
    from lauematching_b200 import preprocess as PP
    rng = np.random.default_rng(9)
    for spacing in (3, 40, 300):
        t = np.zeros((1024, 1024), np.uint16)
        pts = rng.integers(2, 1020 // spacing, (60, 2)) * spacing
        for y, x in pts:
            t[y:y + 2, x:x + 2] = rng.integers(1, 500)
        cfg = dict(nr_px_x=1024, nr_px_y=1024, filter_radius=0, median_passes=1,
                   threshold_method="fixed", threshold_value=0.0, threshold_percentile=90.0,
                   min_area=1, px_x=0.0001, distance=0.513, orientation_spacing=4.0)
        got = PP.preprocess_image(t.astype(np.float64), cfg, return_intermediates=True)
        want = PO.preprocess_image(t.astype(np.float64), cfg, background=np.zeros((1024, 1024)))
        assert np.array_equal(bits(got["blurred"]), bits(want["blurred"]))


def test_preprocessor_keeps_its_background_and_float32_output():
    from lauematching_b200 import preprocess as PP, synth
    z = np.load(os.path.join(HERE, "golden", "pp_fixed_given_bg.npz"))
    cfg = json.loads(str(z["cfg"]))
    pre = PP.Preprocessor(cfg, z["background_in"], blur_dtype=np.float32)
    for _ in range(2):
        b, fi, fl, cen = pre(z["raw"])
        assert b.dtype == np.float32
        assert np.array_equal(b, z["blurred"].astype(np.float32))
        assert np.array_equal(fl, z["filt_labels"])
    pre.close()


def test_reused_page_locked_outputs_hold_the_same_frames():
    from lauematching_b200 import preprocess as PP
    from lauematching_b200.engine import PinnedBuffer
    z = np.load(os.path.join(HERE, "golden", "pp_adaptive_bgmedian.npz"))
    cfg = json.loads(str(z["cfg"]))
    pre = PP.Preprocessor(cfg, z["background"], reuse_outputs=True)
    src = PinnedBuffer(z["raw"].shape, np.float64)
    src.array[...] = z["raw"]
    for _ in range(3):
        b, fi, fl, cen = pre(src.array)
        assert np.array_equal(bits(b), bits(z["blurred"]))
        assert np.array_equal(fi, z["filt_img"]) and np.array_equal(fl, z["filt_labels"])
        assert np.array_equal(bits(centres_array(cen)), bits(z["centers"]))
    b2 = pre(src.array)[0]
    assert b2.ctypes.data == b.ctypes.data  # the same buffer, refilled
    pre.close()


@pytest.mark.parametrize("frame_dtype", [np.float32, np.float64])
def test_raw_frames_straight_into_engine_slots(frame_dtype):
    """Preprocessing into a slot matches exactly as loading the reference's
    blurred frame (as float32 from the image server, or float64 from RunImage)
    from the host does."""
    from lauematching_b200 import params as P, preprocess as PP, synth
    from lauematching_b200.engine import Engine
    names = ["adaptive_bgmedian", "override", "fixed_given_bg", "no_components"]
    zs = [np.load(os.path.join(HERE, "golden", f"pp_{n}.npz")) for n in names]
    by_shape = {}
    for n, z in zip(names, zs):
        by_shape.setdefault(z["raw"].shape, []).append((n, z))
    for shape, cases in by_shape.items():
        ny, nx = shape
        txt = synth.params_text(nr_px=(nx, ny), px=0.0002 * 2048 / max(nx, ny),
                                min_nr_spots=2, min_intensity=5.0)
        p = P.parse_params_text(txt)
        with Engine(p) as e:
            e.build_db_synthetic(3, 60000, synth.hkls_cubic(6))
            for n, z in cases:
                cfg = json.loads(str(z["cfg"]))
                bg = z["background_in"] if z["background_in"].size else None
                pre = PP.Preprocessor(cfg, bg)
                got = pre.to_slot(e, 0, z["raw"], override_thresh=float(z["override_thresh"]),
                                  frame_dtype=frame_dtype)
                if z["centers"].shape[0] == 0:
                    assert got is None
                    pre.close()
                    continue
                assert got == z["centers"].shape[0]
                e.load_image(1, z["blurred"].astype(frame_dtype))
                e.match([0, 1], p.min_nr_spots, p.min_intensity)
                a, na = e.results(0)
                b, nb = e.results(1)
                assert na == nb and np.array_equal(a, b), n
                assert na > 0, n
                pre.close()


def test_pool_loads_the_same_slots_as_one_frame_at_a_time():
    from lauematching_b200 import params as P, preprocess as PP, synth
    from lauematching_b200.engine import Engine
    z = np.load(os.path.join(HERE, "golden", "pp_many_values.npz"))
    cfg = json.loads(str(z["cfg"]))
    ny, nx = z["raw"].shape
    txt = synth.params_text(nr_px=(nx, ny), px=0.0002 * 2048 / max(nx, ny), min_nr_spots=2,
                            min_intensity=5.0)
    p = P.parse_params_text(txt)
    rng = np.random.default_rng(4)
    frames = [z["raw"]] + [synth.raw_frame(ny, nx, rng, n_spots=40, integer=bool(i % 2))
                           for i in range(7)]
    with Engine(p) as e:
        e.build_db_synthetic(5, 60000, synth.hkls_cubic(6))
        pool = PP.PreprocessPool(cfg, z["background"], workers=3)
        got = pool.to_slots(e, list(range(8)), frames)
        pre = PP.Preprocessor(cfg, z["background"])
        for k, f in enumerate(frames):
            assert pre.to_slot(e, 8 + k, f) == got[k]
        slots = [k for k in range(8) if got[k] is not None]
        e.match(slots + [8 + k for k in slots], p.min_nr_spots, p.min_intensity)
        for k in slots:
            a, na = e.results(k)
            b, nb = e.results(8 + k)
            assert na == nb and np.array_equal(a, b)
        pool.close()
        pre.close()


@pytest.mark.parametrize("shape", [(100, 70), (33, 65), (5, 3), (1, 40)])
def test_blur_every_kernel_radius_against_scipy_order(shape):
    """Radii 1-8 (register kernels), 9-32 (shared-memory tile), above (two
    passes), on frames that are not multiples of the tile and on frames
    narrower than the window (mirrored periodically)."""
    from lauematching_b200 import preprocess as PP
    rng = np.random.default_rng(sum(shape))
    t = ((rng.random(shape) < 0.3) * rng.integers(1, 60000, shape)).astype(np.uint16)
    h = PP.DevicePreprocessor(*shape)
    h.segment_thresholded(t, 1)
    for sigma in (0.3, 0.5, 0.7, 1.0, 1.2, 1.4, 1.7, 1.9, 2.5, 5.0, 8.0, 9.0):
        w, r = PP.gaussian_weights(sigma)
        want = PO.gaussian_blur(t, sigma)
        got = h.blur(w, r, np.float64)
        assert np.array_equal(bits(got), bits(want)), (sigma, r)
        got32 = h.blur(w, r, np.float32)
        assert np.array_equal(got32, want.astype(np.float32)), (sigma, r)
    h.close()
