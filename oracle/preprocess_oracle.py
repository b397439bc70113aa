"""TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's frame
preprocessing (background median, subtraction, threshold, connected
components, small-component filter, blur width, Gaussian blur).

It follows ``laue_index/preprocess.py`` and ``laue_index/thresholds.py`` of
the reference as they run in an environment without diplib and scikit-image
(this one): the background is scipy's square median filter, enhancement is
the identity and the Otsu method falls back to the adaptive noise floor.
The third-party steps are restated from their observed contracts, each of
which the CPU tests pin against the library itself:

* scipy.ndimage.median_filter: the element of rank ``size*size // 2`` of the
  ``size x size`` window, window offsets ``-(size//2) .. size-1-size//2``,
  borders mirrored with the edge sample repeated (``d c b a | a b c d``),
  periodically for windows wider than the image (scipy departs from that
  once the window reaches 8x the image side; such sizes are refused);
* cv2.connectedComponentsWithStats (8-connectivity): components numbered
  1.. in the raster order of the first 2x2 pixel block each one touches;
* scipy.ndimage.gaussian_filter: weights ``exp(-x^2 / (2 sigma^2))``
  normalised by their sum over ``|x| <= int(4 sigma + 0.5)``, axis 0 then
  axis 1, each output ``w0*c + (l_r + r_r)*w_r + ... + (l_1 + r_1)*w_1``
  (outermost pair first), borders mirrored as above;
* numpy float64 -> uint16: truncate to int32 (values outside int32 give
  INT32_MIN), keep the low 16 bits.

Only tests/, __graft_entry__.smoke() and bench.py's baseline legs use this
module; the product never imports it.
"""
from __future__ import annotations

import numpy as np
from numpy.lib.stride_tricks import sliding_window_view

__all__ = ["median_filter", "compute_background", "u16_cast", "noise_floor",
           "percentile_linear", "threshold_value", "apply_threshold",
           "connected_components", "filter_small_components", "gaussian_sigma",
           "gaussian_kernel", "gaussian_blur", "preprocess_image"]


def _window(size: int):
    lo = size // 2
    return lo, size - 1 - lo


def median_filter(image: np.ndarray, size: int) -> np.ndarray:
    """scipy.ndimage.median_filter(image, size=size), mode 'reflect'
    (called by ``laue_index/preprocess.py:63-65``)."""
    a = np.asarray(image, dtype=np.float64)
    ny, nx = a.shape
    for n in (ny, nx):
        if n > 1 and size >= 8 * n:
            raise ValueError("median window reaches 8x the image side")
    lo, hi = _window(size)
    p = np.pad(a, ((lo, hi), (lo, hi)), mode="symmetric")
    k = (size * size) // 2
    out = np.empty_like(a)
    step = max(1, (1 << 22) // max(1, size * size * nx))
    for y0 in range(0, ny, step):
        y1 = min(ny, y0 + step)
        w = sliding_window_view(p[y0:y1 + size - 1], (size, size)).reshape(y1 - y0, nx, size * size)
        out[y0:y1] = np.partition(w, k, axis=-1)[..., k]
    return out


def compute_background(image, filter_radius: int = 101, median_passes: int = 1) -> np.ndarray:
    """``laue_index/preprocess.py:42-65`` (scipy branch)."""
    if filter_radius <= 0 or median_passes <= 0:
        return np.zeros_like(image, dtype=np.float64)
    bg = np.asarray(image).astype(np.float64)
    for _ in range(median_passes):
        bg = median_filter(bg, filter_radius)
    return bg


def u16_cast(x: np.ndarray) -> np.ndarray:
    """numpy's float64 -> uint16 conversion on x86-64."""
    x = np.asarray(x, dtype=np.float64)
    ok = (x > -2147483649.0) & (x < 2147483648.0)
    t = np.where(ok, np.trunc(np.where(ok, x, 0.0)), -2147483648.0).astype(np.int64)
    return (t & 0xFFFF).astype(np.uint16)


def _median_sorted(s: np.ndarray) -> float:
    n = s.shape[0]
    if n % 2:
        return float(s[n // 2])
    return float((s[n // 2 - 1] + s[n // 2]) / 2.0)


def noise_floor(image: np.ndarray, k: float = 4.0) -> float:
    """``laue_index/thresholds.py:35-45``: median(nz) + k*1.4826*MAD(nz), >= 1."""
    nz = np.sort(image[image > 0], kind="stable")
    if nz.size:
        med = _median_sorted(nz)
        mad = 1.4826 * _median_sorted(np.sort(np.abs(nz - med)))
        return max(med + k * mad, 1.0)
    return 1.0


def percentile_linear(values: np.ndarray, pct: float) -> float:
    """np.percentile(values, pct) with the default 'linear' method
    (``laue_index/thresholds.py:100``)."""
    v = np.sort(np.asarray(values, dtype=np.float64).ravel())
    n = v.shape[0]
    q = np.true_divide(np.float64(pct), np.float64(100))
    vi = np.float64(n - 1) * q
    if vi >= n - 1:
        return float(v[-1])
    if vi < 0:
        return float(v[0])
    lo = int(np.floor(vi))
    g = vi - np.float64(lo)
    a, b = v[lo], v[lo + 1]
    d = b - a
    r = a + d * g
    if g >= 0.5:
        r = b - d * (1 - g)
    return float(r)


def threshold_value(image, method="adaptive", fixed_value=0.0, percentile=90.0) -> float:
    """``laue_index/thresholds.py:92-110`` without scikit-image (otsu -> adaptive)."""
    if method == "percentile":
        return percentile_linear(image, percentile)
    if method == "fixed":
        return float(fixed_value)
    return noise_floor(image, k=4.0)


def apply_threshold(image, method="adaptive", fixed_value=0.0, percentile=90.0):
    """``laue_index/thresholds.py:29-32,92-110``."""
    t = threshold_value(image, method, fixed_value, percentile)
    out = image.copy()
    out[image <= t] = 0
    return out, float(t)


def connected_components(image: np.ndarray):
    """cv2.connectedComponentsWithStats(image > 0, 8, CV_32S) as used by
    ``laue_index/preprocess.py:136-151``: (labels int32, bboxes [x, y, w, h]
    of labels 1.., areas, nlabels)."""
    import scipy.ndimage as ndi
    b = np.asarray(image) > 0
    ny, nx = b.shape
    lab, n = ndi.label(b, structure=np.ones((3, 3), int))
    if n == 0:
        return np.zeros((ny, nx), np.int32), np.zeros((0, 4), np.int32), np.zeros(0, np.int32), 1
    yy, xx = np.nonzero(lab)
    ll = lab[yy, xx]
    blk = (yy // 2).astype(np.int64) * ((nx + 1) // 2) + (xx // 2)
    first = np.full(n + 1, np.iinfo(np.int64).max)
    np.minimum.at(first, ll, blk)
    order = np.argsort(first[1:], kind="stable") + 1
    remap = np.zeros(n + 1, np.int32)
    remap[order] = np.arange(1, n + 1, dtype=np.int32)
    labels = remap[lab].astype(np.int32)
    fl = remap[ll]
    x0 = np.full(n + 1, nx, np.int64); y0 = np.full(n + 1, ny, np.int64)
    x1 = np.full(n + 1, -1, np.int64); y1 = np.full(n + 1, -1, np.int64)
    np.minimum.at(x0, fl, xx); np.minimum.at(y0, fl, yy)
    np.maximum.at(x1, fl, xx); np.maximum.at(y1, fl, yy)
    areas = np.bincount(fl, minlength=n + 1)[1:].astype(np.int32)
    bboxes = np.stack([x0[1:], y0[1:], x1[1:] - x0[1:] + 1, y1[1:] - y0[1:] + 1], 1).astype(np.int32)
    return labels, bboxes, areas, n + 1


def filter_small_components(image, labels, bboxes, areas, nlabels, min_area=10):
    """``laue_index/preprocess.py:154-188``: components below ``min_area``
    are zeroed in the image and the labels; kept ones give
    ``[label, (cx, cy), area]`` with the intensity-weighted centre of mass
    taken over the component's own pixels inside its bounding box."""
    filt_img = image.copy()
    filt_lbl = labels.copy()
    small = np.zeros(nlabels, bool)
    small[1:] = areas < min_area
    m = small[labels]
    filt_img[m] = 0
    filt_lbl[m] = 0
    centers = []
    if nlabels > 1:
        yy, xx = np.nonzero(labels)
        ll = labels[yy, xx]
        w = image[yy, xx].astype(np.int64)
        sw = np.zeros(nlabels, np.int64); np.add.at(sw, ll, w)
        swx = np.zeros(nlabels, np.int64); np.add.at(swx, ll, w * xx)
        swy = np.zeros(nlabels, np.int64); np.add.at(swy, ll, w * yy)
        for lbl in range(1, nlabels):
            if small[lbl]:
                continue
            x, y = int(bboxes[lbl - 1][0]), int(bboxes[lbl - 1][1])
            s = int(sw[lbl])
            rx = float(int(swx[lbl]) - x * s)
            ry = float(int(swy[lbl]) - y * s)
            cx = np.float64(rx) / np.float64(s) + np.int32(x)
            cy = np.float64(ry) / np.float64(s) + np.int32(y)
            centers.append([lbl, (float(cx), float(cy)), int(areas[lbl - 1])])
    return filt_img, filt_lbl, centers


def gaussian_sigma(centers, pixel_size=0.2, distance=0.513, orient_spacing=0.4) -> float:
    """``laue_index/preprocess.py:191-218``; the nearest-neighbour distance
    of the closest pair of centres, sqrt(dx*dx + dy*dy)."""
    if not centers or len(centers) < 2:
        return 3.0
    c = np.array([cc[1] for cc in centers], dtype=np.float64)
    best = np.inf
    for i0 in range(0, c.shape[0], 2048):
        blk = c[i0:i0 + 2048]
        dx = blk[:, None, 0] - c[None, :, 0]
        dy = blk[:, None, 1] - c[None, :, 1]
        d2 = dx * dx + dy * dy
        idx = np.arange(i0, i0 + blk.shape[0])
        d2[np.arange(blk.shape[0]), idx] = np.inf
        best = min(best, float(d2.min()))
    min_px_dist = float(np.sqrt(best))
    if pixel_size > 0 and distance > 0:
        delta = (distance * np.tan(np.radians(orient_spacing))) / pixel_size
    else:
        delta = min_px_dist
    sigma = 0.25 * min(min_px_dist, delta) if delta > 0 else 0.25 * min_px_dist
    return max(sigma, 1.0)


def gaussian_kernel(sigma: float, truncate: float = 4.0):
    """(weights, radius) as scipy.ndimage.gaussian_filter builds them."""
    sd = float(sigma)
    r = int(truncate * sd + 0.5)
    x = np.arange(-r, r + 1)
    phi = np.exp(-0.5 / (sd * sd) * x ** 2)
    return phi / phi.sum(), r


def _corr_axis(a, w, r, axis):
    pw = [(0, 0), (0, 0)]
    pw[axis] = (r, r)
    p = np.pad(a, pw, mode="symmetric")
    n = a.shape[axis]

    def sl(off):
        idx = [slice(None), slice(None)]
        idx[axis] = slice(r + off, r + off + n)
        return p[tuple(idx)]
    out = sl(0) * w[r]
    for j in range(r, 0, -1):
        out = out + (sl(-j) + sl(j)) * w[r - j]
    return out


def gaussian_blur(image, sigma: float) -> np.ndarray:
    """scipy.ndimage.gaussian_filter(image.astype(float64), sigma)
    (``laue_index/preprocess.py:329``)."""
    w, r = gaussian_kernel(sigma)
    a = np.asarray(image, dtype=np.float64)
    return _corr_axis(_corr_axis(a, w, r, 0), w, r, 1)


def preprocess_image(raw_image, cfg, background=None, override_thresh=0.0) -> dict:
    """``laue_index/preprocess.py:221-338`` with every intermediate."""
    if background is None:
        background = compute_background(raw_image, cfg["filter_radius"], cfg["median_passes"])
    bg_sub = np.maximum(raw_image - background, 0.0)
    if override_thresh > 0:
        thr, t = apply_threshold(bg_sub, "fixed", override_thresh)
    else:
        thr, t = apply_threshold(bg_sub, cfg["threshold_method"], cfg["threshold_value"],
                                 cfg["threshold_percentile"])
    t16 = u16_cast(thr)
    labels, bboxes, areas, nlabels = connected_components(t16)
    out = {"background": background, "threshold": t, "thresholded": t16,
           "labels_unfiltered": labels}
    if nlabels <= 1:
        out.update(filt_img=t16, filt_labels=labels, centers=[], sigma=None,
                   blurred=np.zeros(raw_image.shape, np.float64))
        return out
    filt_img, filt_labels, centers = filter_small_components(t16, labels, bboxes, areas, nlabels,
                                                             cfg["min_area"])
    out.update(filt_img=filt_img, filt_labels=filt_labels, centers=centers)
    if not centers:
        out.update(sigma=None, blurred=np.zeros(raw_image.shape, np.float64))
        return out
    sigma = gaussian_sigma(centers, cfg["px_x"], cfg["distance"], cfg["orientation_spacing"])
    out.update(sigma=sigma, blurred=gaussian_blur(filt_img, sigma))
    return out
