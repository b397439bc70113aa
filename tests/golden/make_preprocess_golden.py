"""Generate the frame-preprocessing golden fixtures from the REFERENCE itself.

Imports the reference's ``laue_index.preprocess.preprocess_image`` (in an
environment with numpy, scipy and OpenCV but without diplib and
scikit-image, like this one) and runs it with ``return_intermediates=True``
on seeded synthetic frames.  Each case is stored as ``pp_<case>.npz``: the
raw frame, the background passed in (or none), the config keys used, the
override threshold, and the reference's background, thresholded image,
unfiltered and filtered labels, filtered image, centres and blurred image.

Usage (in a checkout where the reference tree exists):
    python tests/golden/make_preprocess_golden.py [reference_root]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lauematching_b200 import synth  # noqa: E402

BASE_CFG = dict(filter_radius=101, median_passes=1, threshold_method="adaptive",
                threshold_value=0.0, threshold_percentile=90.0, min_area=10, px_x=0.2,
                distance=0.513, orientation_spacing=0.4)

# name: (ny, nx, seed, frame kwargs, cfg overrides, background kind, override threshold)
CASES = {
    "adaptive_bgmedian": (96, 128, 1, dict(n_spots=40), dict(filter_radius=15), None, 0.0),
    "even_radius_two_passes": (80, 72, 2, dict(n_spots=25), dict(filter_radius=8, median_passes=2),
                               None, 0.0),
    "percentile": (120, 100, 3, dict(n_spots=30), dict(filter_radius=11,
                   threshold_method="percentile", threshold_percentile=99.2), None, 0.0),
    "fixed_given_bg": (110, 130, 4, dict(n_spots=35, integer=False),
                       dict(threshold_method="fixed", threshold_value=20.5, min_area=4),
                       "smooth", 0.0),
    "override": (90, 90, 5, dict(n_spots=30), dict(filter_radius=21), None, 30.0),
    "otsu_falls_back": (64, 96, 6, dict(n_spots=20), dict(filter_radius=9,
                        threshold_method="otsu"), None, 0.0),
    "many_values": (300, 300, 7, dict(n_spots=60, integer=False), dict(filter_radius=11), None, 0.0),
    "wide_sigma": (100, 100, 8, dict(n_spots=12), dict(filter_radius=13, px_x=0.0004,
                   orientation_spacing=2.0), None, 0.0),
    "no_components": (64, 64, 9, dict(n_spots=3), dict(filter_radius=7), "equal", 0.0),
    "all_small": (70, 70, 10, dict(n_spots=6, sigma=0.3), dict(filter_radius=9, min_area=50),
                  None, 0.0),
    "one_centre": (60, 60, 11, dict(n_spots=1, amp_lo=3000.0), dict(filter_radius=9), None, 0.0),
    "u16_wrap": (64, 64, 12, dict(n_spots=8, amp_lo=70000.0, amp_hi=140000.0),
                 dict(threshold_method="fixed", threshold_value=50.0), "flat", 0.0),
    "window_wider_than_frame": (9, 7, 13, dict(n_spots=2, sigma=0.8), dict(filter_radius=25,
                                min_area=1), None, 0.0),
    "border_spots": (50, 60, 14, dict(n_spots=0), dict(filter_radius=9, min_area=3), "spots@edges",
                     0.0),
}


def make_frame(ny, nx, seed, kw, bg_kind):
    rng = np.random.default_rng(seed)
    raw = synth.raw_frame(ny, nx, rng, **kw)
    bg = None
    if bg_kind == "smooth":
        yy, xx = np.mgrid[0:ny, 0:nx]
        bg = 100.0 + 30.0 * np.sin(yy / 17.0) * np.cos(xx / 23.0) + 0.37 * xx
    elif bg_kind == "equal":
        bg = raw.copy()
    elif bg_kind == "flat":
        bg = np.full((ny, nx), 100.0)
    elif bg_kind == "spots@edges":
        bg = np.full((ny, nx), 100.0)
        for (y, x) in ((0, 0), (0, nx - 2), (ny - 2, 0), (ny - 1, nx - 1), (ny // 2, 0), (0, nx // 2)):
            raw[max(0, y - 1):y + 2, max(0, x - 1):x + 2] += 900.0
    return raw, bg


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LAUE_REFERENCE_ROOT")
    if not ref_root:
        sys.exit("give the reference tree as the argument or in LAUE_REFERENCE_ROOT")
    sys.path.insert(0, ref_root)
    from laue_index import preprocess as RP
    for name, (ny, nx, seed, kw, over, bg_kind, ovt) in CASES.items():
        cfg = dict(BASE_CFG, nr_px_x=nx, nr_px_y=ny, **over)
        raw, bg = make_frame(ny, nx, seed, kw, bg_kind)
        r = RP.preprocess_image(raw, cfg, background=bg, override_thresh=ovt,
                                return_intermediates=True)
        cen = np.array([[c[0], c[1][0], c[1][1], c[2]] for c in r["centers"]],
                       np.float64).reshape(-1, 4)
        out = os.path.join(HERE, f"pp_{name}.npz")
        np.savez_compressed(
            out, raw=raw, background_in=bg if bg is not None else np.zeros((0, 0)),
            cfg=json.dumps(cfg), override_thresh=ovt,
            background=r["background"], thresholded=r["thresholded"],
            labels_unfiltered=r["labels_unfiltered"], filt_img=r["filt_img"],
            filt_labels=r["filt_labels"], blurred=r["blurred"], centers=cen)
        print(f"{name}: {ny}x{nx}, {cen.shape[0]} centres, "
              f"{int(r['labels_unfiltered'].max())} components -> {os.path.basename(out)}")


if __name__ == "__main__":
    main()
