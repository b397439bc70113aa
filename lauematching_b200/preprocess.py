"""Frame preprocessing on the device, with the API of ``laue_index.preprocess``.

Drop-in for ``laue_index/preprocess.py`` (background median, subtraction,
threshold, connected components, small-component filter, blur width,
Gaussian blur; ``preprocess_image`` at :221-338), returning the same arrays
as the reference does where numpy, scipy and OpenCV are installed and diplib
and scikit-image are not (this image): the background is scipy's square
median, enhancement is the identity and the "otsu" method falls back to the
adaptive noise floor (``laue_index/thresholds.py:92-110``).

The image server (``scripts/laue_image_server.py:66-80``) and ``RunImage``
call ``preprocess_image`` once per frame; here every step runs on the GPU
through ``liblmb200.so`` and only the frames and the centre list cross the
host link.  A :class:`Preprocessor` keeps one device handle and the uploaded
background across frames; the module functions share a handle per thread
and frame size.
"""
from __future__ import annotations

import ctypes as C
import logging
import math
import os
import threading
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib

logger = logging.getLogger("LaueStream")

__all__ = [
    "compute_background", "load_background", "enhance_image",
    "find_connected_components", "filter_small_components",
    "calculate_gaussian_sigma", "gaussian_weights", "preprocess_image", "Preprocessor",
    "DevicePreprocessor", "PreprocessPool", "config_from_params_text",
]

_DTYPES = {np.dtype(np.float64): _lib.LMB_F64, np.dtype(np.float32): _lib.LMB_F32,
           np.dtype(np.uint16): _lib.LMB_U16, np.dtype(np.uint8): _lib.LMB_U8}


def _frame(a: np.ndarray):
    a = np.ascontiguousarray(a)
    if a.dtype not in _DTYPES:
        a = np.ascontiguousarray(a, dtype=np.float64)
    return a, _DTYPES[a.dtype]


class DevicePreprocessor:
    """One device handle for frames of ``(nr_px_y, nr_px_x)`` pixels."""

    def __init__(self, nr_px_y: int, nr_px_x: int, device: int = 0):
        self.shape = (int(nr_px_y), int(nr_px_x))
        self.device = int(device)
        h = C.c_void_p()
        check(lib().lmb_pre_create(self.device, self.shape[0], self.shape[1], C.byref(h)))
        self._h = h
        self._bg_token = None

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().lmb_pre_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_shape(self, a):
        if tuple(a.shape) != self.shape:
            raise ValueError(f"frame of shape {a.shape}, expected {self.shape}")

    # -- background ---------------------------------------------------------
    def median(self, frame: np.ndarray, size: int, passes: int = 1,
               want: bool = True) -> Optional[np.ndarray]:
        """Median background of ``frame``; it becomes the handle's background."""
        a, dt = _frame(frame)
        self._check_shape(a)
        out = np.empty(self.shape, np.float64) if want else None
        check(lib().lmb_pre_median(self._h, a.ctypes.data, dt, int(size), int(passes),
                                   out.ctypes.data if want else None))
        self._bg_token = ("median", id(frame))
        return out

    def set_background(self, background: Optional[np.ndarray], token=None) -> None:
        if token is not None and token == self._bg_token:
            return
        if background is None:
            check(lib().lmb_pre_set_background(self._h, None))
        else:
            bg = np.ascontiguousarray(background, dtype=np.float64)
            self._check_shape(bg)
            check(lib().lmb_pre_set_background(self._h, bg.ctypes.data))
        self._bg_token = token

    def background(self) -> np.ndarray:
        out = np.empty(self.shape, np.float64)
        check(lib().lmb_pre_get_background(self._h, out.ctypes.data))
        return out

    STAGES = ("upload", "threshold", "components", "blur", "blur_download", "median_upload",
              "median_ranks", "median")

    def timings(self) -> dict:
        """Device milliseconds of the stages of the last calls."""
        ms = (C.c_float * _lib.LMB_PRE_STAGES)()
        check(lib().lmb_pre_timings(self._h, ms, _lib.LMB_PRE_STAGES))
        return dict(zip(self.STAGES, [round(float(v), 4) for v in ms]))

    # -- segmentation ---------------------------------------------------------
    def segment(self, frame: np.ndarray, method: str = "adaptive", threshold_value: float = 0.0,
                threshold_percentile: float = 90.0, min_area: int = 10,
                override_thresh: float = 0.0) -> _lib.LmbPreCounts:
        a, dt = _frame(frame)
        self._check_shape(a)
        prm = _lib.LmbPreParams()
        prm.threshold_method = (_lib.LMB_THR_PERCENTILE if method == "percentile" else
                                _lib.LMB_THR_FIXED if method == "fixed" else
                                _lib.LMB_THR_ADAPTIVE)
        prm.min_area = int(min_area)
        prm.threshold_value = float(threshold_value)
        prm.threshold_percentile = float(threshold_percentile)
        prm.override_thresh = float(override_thresh)
        cnt = _lib.LmbPreCounts()
        check(lib().lmb_pre_segment(self._h, a.ctypes.data, dt, C.byref(prm), C.byref(cnt)))
        return cnt

    def segment_thresholded(self, thresholded: np.ndarray, min_area: int) -> _lib.LmbPreCounts:
        t = np.ascontiguousarray(thresholded, dtype=np.uint16)
        self._check_shape(t)
        cnt = _lib.LmbPreCounts()
        check(lib().lmb_pre_segment_thresholded(self._h, t.ctypes.data, int(min_area),
                                                C.byref(cnt)))
        return cnt

    def centres(self, n: int) -> List:
        rows = np.empty((max(n, 1), 4), np.float64)
        check(lib().lmb_pre_centres(self._h, rows.ctypes.data, int(n)))
        return [[int(r[0]), (float(r[1]), float(r[2])), int(r[3])] for r in rows[:n]]

    def stats(self, n_labels: int) -> Tuple[np.ndarray, np.ndarray]:
        n = max(n_labels - 1, 0)
        st = np.empty((max(n, 1), 5), np.int32)
        check(lib().lmb_pre_stats(self._h, st.ctypes.data, n))
        return np.ascontiguousarray(st[:n, :4]), np.ascontiguousarray(st[:n, 4])

    def images(self, thresholded=False, labels=False, filt_img=False, filt_labels=False,
               outs: Optional[dict] = None):
        """The last segment's frames; ``outs`` may supply the arrays to fill."""
        out = {}
        ptr = {}
        for name, want, dt in (("thresholded", thresholded, np.uint16), ("labels", labels, np.int32),
                               ("filt_img", filt_img, np.uint16),
                               ("filt_labels", filt_labels, np.int32)):
            if want:
                a = outs.get(name) if outs else None
                if a is None or a.shape != self.shape or a.dtype != dt or \
                        not a.flags.c_contiguous:
                    a = np.empty(self.shape, dt)
                out[name] = a
                ptr[name] = a.ctypes.data
            else:
                ptr[name] = None
        check(lib().lmb_pre_images(self._h, ptr["thresholded"], ptr["labels"], ptr["filt_img"],
                                   ptr["filt_labels"]))
        return out

    def blur_to_slot(self, weights: np.ndarray, radius: int, engine, slot: int,
                     frame_dtype=np.float32) -> float:
        """The blurred frame straight into an engine slot on this device,
        quantised as if ``frame_dtype`` copies of it had been loaded from the
        host; returns the slot's imScale."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if w.shape != (2 * radius + 1,):
            raise ValueError("weights must have 2*radius+1 entries")
        dt = np.dtype(frame_dtype)
        sc = C.c_double(0.0)
        check(lib().lmb_pre_blur_to_slot(self._h, w.ctypes.data, int(radius), engine._h,
                                         int(slot),
                                         _lib.LMB_F64 if dt == np.float64 else _lib.LMB_F32,
                                         C.byref(sc)))
        return sc.value

    def blur(self, weights: np.ndarray, radius: int, dtype=np.float64,
             out: Optional[np.ndarray] = None) -> np.ndarray:
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if w.shape != (2 * radius + 1,):
            raise ValueError("weights must have 2*radius+1 entries")
        dt = np.dtype(dtype)
        if out is None or out.shape != self.shape or out.dtype != dt or \
                not out.flags.c_contiguous:
            out = np.empty(self.shape, dt)
        check(lib().lmb_pre_blur(self._h, w.ctypes.data, int(radius), out.ctypes.data,
                                 _lib.LMB_F64 if dt == np.float64 else _lib.LMB_F32))
        return out


_local = threading.local()


def _handle(shape, device: int = 0) -> DevicePreprocessor:
    cache = getattr(_local, "handles", None)
    if cache is None:
        cache = _local.handles = {}
    key = (int(device), int(shape[0]), int(shape[1]))
    h = cache.get(key)
    if h is None:
        h = cache[key] = DevicePreprocessor(shape[0], shape[1], device)
    return h


def compute_background(image: np.ndarray, filter_radius: int = 101, median_passes: int = 1,
                       *, device: int = 0) -> np.ndarray:
    """Median background (``laue_index/preprocess.py:42-65``, scipy branch)."""
    if filter_radius <= 0 or median_passes <= 0:
        return np.zeros_like(image, dtype=np.float64)
    return _handle(np.shape(image), device).median(image, filter_radius, median_passes)


def load_background(background_file: str, nr_px_x: int, nr_px_y: int) -> np.ndarray:
    """Pre-computed background from a raw float64 file
    (``laue_index/preprocess.py:68-86``)."""
    expected = nr_px_x * nr_px_y * np.dtype(np.float64).itemsize
    if background_file and os.path.exists(background_file):
        actual = os.path.getsize(background_file)
        if actual == expected:
            return np.fromfile(background_file, dtype=np.float64).reshape((nr_px_y, nr_px_x))
        logger.warning(f"Background file size mismatch (expected {expected}, got {actual}). "
                       "Ignoring.")
    return np.zeros((nr_px_y, nr_px_x), dtype=np.float64)


def enhance_image(image: np.ndarray, *, denoise: bool = False, denoise_strength: float = 1.0,
                  contrast: bool = False, edge: bool = False) -> np.ndarray:
    """The identity, as ``laue_index/preprocess.py:89-133`` is without
    scikit-image: its denoising, CLAHE and unsharp mask are not provided."""
    return image


def find_connected_components(image: np.ndarray, *, device: int = 0):
    """8-connected components of ``image > 0`` numbered as OpenCV numbers them
    (``laue_index/preprocess.py:136-151``): (labels, bboxes, areas, nlabels)."""
    img = np.asarray(image)
    if img.dtype == np.uint16:
        t = img
    else:
        with np.errstate(invalid="ignore"):
            t = (img > 0).astype(np.uint16)
    h = _handle(img.shape, device)
    cnt = h.segment_thresholded(t, 0)
    labels = h.images(labels=True)["labels"]
    bboxes, areas = h.stats(cnt.n_labels)
    return labels, bboxes, areas, int(cnt.n_labels)


def filter_small_components(image: np.ndarray, labels: np.ndarray, bboxes: np.ndarray,
                            areas: np.ndarray, nlabels: int, min_area: int = 10,
                            *, device: int = 0):
    """``laue_index/preprocess.py:154-188`` for a uint16 frame and its own
    components (as find_connected_components returns them):
    (filtered_image, filtered_labels, centers)."""
    img = np.asarray(image)
    if img.dtype != np.uint16:
        if not np.issubdtype(img.dtype, np.integer) or img.min(initial=0) < 0 or \
                img.max(initial=0) > 65535:
            raise ValueError("filter_small_components takes a uint16 frame")
        img = img.astype(np.uint16)
    h = _handle(img.shape, device)
    cnt = h.segment_thresholded(img, min_area)
    got = h.images(labels=True, filt_img=True, filt_labels=True)
    if int(cnt.n_labels) != int(nlabels) or not np.array_equal(got["labels"], labels):
        raise ValueError("labels are not this frame's 8-connected components")
    return got["filt_img"], got["filt_labels"], h.centres(int(cnt.n_centres))


def _sigma_from(n_centres: int, min_dist2: float, pixel_size: float, distance: float,
                orient_spacing: float) -> float:
    """``laue_index/preprocess.py:191-218`` given the closest pair's squared
    distance (the nearest-neighbour distance minimum)."""
    if n_centres < 2:
        return 3.0
    min_px_dist = float(math.sqrt(min_dist2))
    if pixel_size > 0 and distance > 0:
        delta = (distance * np.tan(np.radians(orient_spacing))) / pixel_size
    else:
        delta = min_px_dist
    sigma = 0.25 * min(min_px_dist, delta) if delta > 0 else 0.25 * min_px_dist
    return max(sigma, 1.0)


def calculate_gaussian_sigma(centers: List, pixel_size: float = 0.2, distance: float = 0.513,
                             orient_spacing: float = 0.4) -> float:
    """Blur width from the spot spacing (``laue_index/preprocess.py:191-218``)."""
    if not centers or len(centers) < 2:
        return 3.0
    c = np.array([cc[1] for cc in centers], dtype=np.float64)
    best = np.inf
    for i0 in range(0, c.shape[0], 1024):
        blk = c[i0:i0 + 1024]
        dx = blk[:, None, 0] - c[None, :, 0]
        dy = blk[:, None, 1] - c[None, :, 1]
        d2 = dx * dx + dy * dy
        d2[np.arange(blk.shape[0]), np.arange(i0, i0 + blk.shape[0])] = np.inf
        best = min(best, float(d2.min()))
    return _sigma_from(len(centers), best, pixel_size, distance, orient_spacing)


def gaussian_weights(sigma: float, truncate: float = 4.0) -> Tuple[np.ndarray, int]:
    """(weights, radius) of scipy.ndimage.gaussian_filter for ``sigma``."""
    sd = float(sigma)
    radius = int(truncate * sd + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return phi / phi.sum(), radius


# Preprocessing keys of a LaueMatching parameter file and their defaults, as
# the image server reads them (scripts/laue_stream_utils.py:89-220).
_CONFIG_DEFAULTS = {"nr_px_x": 2048, "nr_px_y": 2048, "px_x": 0.2, "px_y": 0.2,
                    "distance": 0.513, "threshold_method": "adaptive", "threshold_value": 0.0,
                    "threshold_percentile": 90.0, "min_area": 10, "filter_radius": 101,
                    "median_passes": 1, "orientation_spacing": 0.4, "background_file": ""}


def config_from_params_text(text: str) -> Dict[str, Any]:
    """The preprocessing configuration of a parameter file's text, with the
    rules of ``scripts/laue_stream_utils.py:parse_config`` (141-220): ``#``
    comments, the first token is the key, malformed values are skipped."""
    cfg = dict(_CONFIG_DEFAULTS)
    conv = {"NrPxX": ("nr_px_x", int), "NrPxY": ("nr_px_y", int), "PxX": ("px_x", float),
            "PxY": ("px_y", float), "ThresholdMethod": ("threshold_method", str.lower),
            "Threshold": ("threshold_value", float),
            "ThresholdPercentile": ("threshold_percentile", float),
            "MinArea": ("min_area", int), "FilterRadius": ("filter_radius", int),
            "NMeadianPasses": ("median_passes", int),
            "OrientationSpacing": ("orientation_spacing", float),
            "BackgroundFile": ("background_file", str)}
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        if "#" in line:
            line = line[: line.index("#")].strip()
        parts = line.split()
        if len(parts) < 2:
            continue
        key, rest = parts[0], parts[1:]
        try:
            if key == "P_Array" and len(rest) >= 3:
                cfg["distance"] = float(rest[2])
            elif key in conv:
                name, f = conv[key]
                cfg[name] = f(rest[0])
        except (ValueError, IndexError):
            logger.warning(f"Skipping malformed config line '{line}'")
    return cfg


def _threshold_method(cfg) -> str:
    m = cfg["threshold_method"]
    return m if m in ("percentile", "fixed") else "adaptive"


def _run(h: DevicePreprocessor, raw_image, cfg, override_thresh, return_intermediates,
         blur_dtype, outs=None):
    cnt = h.segment(raw_image, _threshold_method(cfg), cfg["threshold_value"],
                    cfg["threshold_percentile"], cfg["min_area"], override_thresh)
    shape = h.shape
    inter = return_intermediates
    if cnt.n_labels <= 1:
        im = h.images(thresholded=True, labels=True)
        blurred = np.zeros(shape, dtype=np.float64)
        if inter:
            return {"background": h.background(), "thresholded": im["thresholded"],
                    "labels_unfiltered": im["labels"], "filt_img": im["thresholded"],
                    "filt_labels": im["labels"], "blurred": blurred, "centers": []}
        return blurred, im["thresholded"], im["labels"], []
    im = h.images(thresholded=inter, labels=inter, filt_img=True, filt_labels=True, outs=outs)
    centers = h.centres(int(cnt.n_centres))
    if not centers:
        blurred = np.zeros(shape, dtype=np.float64)
    else:
        sigma = _sigma_from(len(centers), cnt.min_dist2, cfg["px_x"], cfg["distance"],
                            cfg["orientation_spacing"])
        w, r = gaussian_weights(sigma)
        blurred = h.blur(w, r, blur_dtype, out=outs.get("blurred") if outs else None)
    if inter:
        return {"background": h.background(), "thresholded": im["thresholded"],
                "labels_unfiltered": im["labels"], "filt_img": im["filt_img"],
                "filt_labels": im["filt_labels"], "blurred": blurred, "centers": centers}
    return blurred, im["filt_img"], im["filt_labels"], centers


def _prepare_background(h: DevicePreprocessor, raw_image, cfg, background):
    if background is None:
        bg = load_background(cfg.get("background_file", ""), cfg["nr_px_x"], cfg["nr_px_y"])
        if np.count_nonzero(bg) == 0:
            if cfg["filter_radius"] <= 0 or cfg["median_passes"] <= 0:
                h.set_background(None, token=("zeros",))
            else:
                h.median(raw_image, cfg["filter_radius"], cfg["median_passes"], want=False)
        else:
            h.set_background(bg, token=None)
    else:
        h.set_background(background, token=None)


def preprocess_image(raw_image: np.ndarray, cfg: Dict[str, Any],
                     background: Optional[np.ndarray] = None, override_thresh: float = 0.0,
                     return_intermediates: bool = False, *, device: int = 0,
                     blur_dtype=np.float64):
    """``laue_index/preprocess.py:221-338`` on the device: returns
    (blurred, filtered_thresholded_image, filtered_labels, centers), or the
    dict of intermediates.  ``blur_dtype=np.float32`` delivers the blurred
    frame as the image server sends it (``laue_image_server.py:79``)."""
    raw = np.asarray(raw_image)
    if raw.shape != (cfg["nr_px_y"], cfg["nr_px_x"]):
        raise ValueError(f"frame of shape {raw.shape}, config says "
                         f"({cfg['nr_px_y']}, {cfg['nr_px_x']})")
    h = _handle(raw.shape, device)
    _prepare_background(h, raw, cfg, background)
    return _run(h, raw, cfg, override_thresh, return_intermediates, blur_dtype)


class Preprocessor:
    """Config-driven wrapper (``laue_index/preprocess.py:341-353``) holding
    one device handle and the background uploaded once."""

    def __init__(self, cfg: Dict[str, Any], background: Optional[np.ndarray] = None,
                 *, device: int = 0, blur_dtype=np.float64, reuse_outputs: bool = False):
        """``reuse_outputs``: the returned blurred frame, filtered frame and
        filtered labels are views of page-locked buffers owned by this object
        and overwritten by the next call (no page faults on fresh arrays,
        full-speed copies); by default every call returns new arrays, as the
        reference does."""
        self.cfg = cfg
        self.background = background
        self.blur_dtype = blur_dtype
        self._h = DevicePreprocessor(cfg["nr_px_y"], cfg["nr_px_x"], device)
        self._outs = None
        if reuse_outputs:
            from .engine import PinnedBuffer
            shape = self._h.shape
            self._pinned = [PinnedBuffer(shape, blur_dtype), PinnedBuffer(shape, np.uint16),
                            PinnedBuffer(shape, np.int32)]
            self._outs = {"blurred": self._pinned[0].array, "filt_img": self._pinned[1].array,
                          "filt_labels": self._pinned[2].array}
        if background is not None:
            self._h.set_background(background, token=("fixed",))

    def __call__(self, raw_image: np.ndarray, *, override_thresh: float = 0.0,
                 return_intermediates: bool = False):
        raw = np.asarray(raw_image)
        if raw.shape != self._h.shape:
            raise ValueError(f"frame of shape {raw.shape}, expected {self._h.shape}")
        if self.background is None:
            _prepare_background(self._h, raw, self.cfg, None)
        return _run(self._h, raw, self.cfg, override_thresh, return_intermediates,
                    self.blur_dtype, self._outs)

    def to_slot(self, engine, slot: int, raw_image: np.ndarray, *,
                override_thresh: float = 0.0, frame_dtype=np.float32, want_centres: bool = False):
        """Preprocess a raw frame straight into image slot ``slot`` of
        ``engine`` (same device, same frame size): the slot then holds what
        loading ``preprocess_image``'s blurred frame, as ``frame_dtype`` (float32:
        the image server's wire format; float64: RunImage's .bin), would give,
        without the frame leaving the GPU.  Returns the number of centres (or
        the centre list with ``want_centres``); ``None`` when the frame has no
        spots, as the image server then sends nothing (laue_image_server.py:76-77)
        and the slot is left untouched."""
        raw = np.asarray(raw_image)
        if raw.shape != self._h.shape:
            raise ValueError(f"frame of shape {raw.shape}, expected {self._h.shape}")
        if self.background is None:
            _prepare_background(self._h, raw, self.cfg, None)
        cfg = self.cfg
        cnt = self._h.segment(raw, _threshold_method(cfg), cfg["threshold_value"],
                              cfg["threshold_percentile"], cfg["min_area"], override_thresh)
        if cnt.n_labels <= 1 or cnt.n_centres == 0:
            return None
        sigma = _sigma_from(int(cnt.n_centres), cnt.min_dist2, cfg["px_x"], cfg["distance"],
                            cfg["orientation_spacing"])
        w, r = gaussian_weights(sigma)
        self._h.blur_to_slot(w, r, engine, slot, frame_dtype)
        return self._h.centres(int(cnt.n_centres)) if want_centres else int(cnt.n_centres)

    def close(self):
        self._h.close()


class PreprocessPool:
    """Several frames preprocessed at once into an engine's slots: one
    :class:`Preprocessor` (device handle and CUDA stream) per worker thread, so
    one frame's upload and host steps overlap another's kernels.  Calls into
    the engine are serialised (an engine is not re-entrant)."""

    def __init__(self, cfg: Dict[str, Any], background: Optional[np.ndarray] = None, *,
                 device: int = 0, workers: int = 3):
        from concurrent.futures import ThreadPoolExecutor
        self.cfg, self.background, self.device = cfg, background, device
        self._pres = [Preprocessor(cfg, background, device=device) for _ in range(workers)]
        self._free = list(range(workers))
        self._lock = threading.Lock()
        self._engine_lock = threading.Lock()
        self._pool = ThreadPoolExecutor(max_workers=workers)

    def _one(self, engine, slot, frame, frame_dtype, host_copy=False):
        with self._lock:
            w = self._free.pop()
        try:
            pre = self._pres[w]
            raw = np.asarray(frame)
            if pre.background is None:
                _prepare_background(pre._h, raw, self.cfg, None)
            cfg = self.cfg
            cnt = pre._h.segment(raw, _threshold_method(cfg), cfg["threshold_value"],
                                 cfg["threshold_percentile"], cfg["min_area"], 0.0)
            if cnt.n_labels <= 1 or cnt.n_centres == 0:
                return None
            sigma = _sigma_from(int(cnt.n_centres), cnt.min_dist2, cfg["px_x"], cfg["distance"],
                                cfg["orientation_spacing"])
            wts, r = gaussian_weights(sigma)
            with self._engine_lock:
                pre._h.blur_to_slot(wts, r, engine, slot, frame_dtype)
            if host_copy:  # the blurred frame as the matcher read it, for the post-stage
                return int(cnt.n_centres), pre._h.blur(wts, r, frame_dtype)
            return int(cnt.n_centres)
        finally:
            with self._lock:
                self._free.append(w)

    def to_slots(self, engine, slots, frames, frame_dtype=np.float32,
                 host_copy: bool = False) -> List:
        """Preprocess frames[i] into slots[i] (``Preprocessor.to_slot`` for
        each, several at a time); returns each frame's centre count (with
        ``host_copy``, the pair (count, blurred frame as ``frame_dtype`` in host
        memory)), ``None`` for frames without spots (their slots are left
        untouched)."""
        futs = [self._pool.submit(self._one, engine, s, f, frame_dtype, host_copy)
                for s, f in zip(slots, frames)]
        return [f.result() for f in futs]

    def close(self):
        self._pool.shutdown(wait=True)
        for p in self._pres:
            p.close()
