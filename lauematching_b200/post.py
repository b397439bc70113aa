"""Post-stage after the compare pass: merge, refinement objective, output text.

Wraps ``lmb_post_process`` (host C++ in liblmb200).  Output headers are the
reference's (single image: LaueMatchingCPU.c:755-770; daemon:
LaueMatchingGPUStream.cu:1088-1104).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import check, lib
from .params import LaueParams

SOLUTIONS_HEADER = (
    "%GrainNr\tNumberOfSolutions\tIntensity\tNMatches*Intensity\tNMatches*sqrt(Intensity)\t"
    "NMatches\tNSpotsCalc\t"
    "Recip1\tRecip2\tRecip3\tRecip4\tRecip5\tRecip6\tRecip7\tRecip8\tRecip9\t"
    "LatticeParameterFit[a]\tLatticeParameterFit[b]\tLatticeParameterFit[c]\t"
    "LatticeParameterFit[alpha]\tLatticeParameterFit[beta]\tLatticeParameterFit[gamma]\t"
    "OrientMatrix0\tOrientMatrix1\tOrientMatrix2\tOrientMatrix3\tOrientMatrix4\tOrientMatrix5\t"
    "OrientMatrix6\tOrientMatrix7\tOrientMatrix8\t"
    "CoarseNMatches*sqrt(Intensity)\tmisOrientationPostRefinement[degrees]\torientationRowNr\n")
SPOTS_HEADER = "%GrainNr\tSpotNr\th\tk\tl\tX\tY\tQhat[0]\tQhat[1]\tQhat[2]\tIntensity\n"
STREAM_SOLUTIONS_HEADER = "%ImageNr\t" + SOLUTIONS_HEADER[1:]
STREAM_SPOTS_HEADER = "%ImageNr\t" + SPOTS_HEADER[1:]


def make_post_params(params: LaueParams, min_nr_spots: int | None = None,
                     num_threads: int | None = None) -> _lib.LmbPostParams:
    """The post-stage's crystal and merge parameters from a parameter file."""
    pp = _lib.LmbPostParams()
    for i in range(6):
        pp.lattice[i] = params.lattice[i]
        pp.tol_latc[i] = params.tol_latc[i]
    pp.space_group = int(params.space_group)
    pp.max_nr_spots = int(params.max_nr_spots)
    pp.tol_c_over_a = float(params.tol_c_over_a)
    pp.max_angle = float(params.max_angle)
    pp.min_nr_spots = int(params.min_nr_spots if min_nr_spots is None else min_nr_spots)
    pp.num_threads = int(num_threads or os.cpu_count() or 1)
    # "Optimizer NelderMead" in the parameter file: this library's bounded
    # Nelder-Mead (NLopt is not available); BOBYQA, the reference's default,
    # needs NLopt and is run as the evaluate-once stand-in
    pp.optimizer = 1 if params.optimizer == "NelderMead" else 0
    return pp


def post_process(params: LaueParams, geometry, orients: np.ndarray, ids: np.ndarray,
                 scores: np.ndarray, image_f32: np.ndarray, hkls: np.ndarray,
                 min_nr_spots: int | None = None, image_num: int = 0,
                 num_threads: int | None = None, max_results: int = 0,
                 merge_device: int | None = None, optimizer: str | None = None):
    """Return (solutions_text, spots_text, n_unique) for one image.

    ``ids``/``scores`` are the image's collected matches in the reference's
    collection order (ascending orientation ID).  ``max_results`` > 0 keeps
    only that many top-scored candidates for the merge (the reference's own
    cap path, LaueMatchingHeaders.h:976-997, with its cap of 50000 lowered).
    ``merge_device`` (a CUDA device index) runs the duplicate merge of 1024 or
    more candidates on that device (same clusters); None keeps it on the host.
    ``optimizer`` ("once" or "nelder-mead") overrides the parameter file's
    Optimizer (NelderMead: this library's Nelder-Mead; otherwise once)."""
    pp = make_post_params(params, min_nr_spots, num_threads)
    if optimizer is not None:
        pp.optimizer = {"once": 0, "nelder-mead": 1}[optimizer]
    pp.image_num = int(image_num)
    pp.max_results = int(max_results)  # 0: the reference's 50000
    pp.merge_on_device = 0 if merge_device is None else int(merge_device) + 1
    om = np.ascontiguousarray(orients, dtype=np.float64).reshape(-1, 9)
    idv = np.ascontiguousarray(ids, dtype=np.uint64)
    scv = np.ascontiguousarray(scores, dtype=np.float64)
    img = np.ascontiguousarray(image_f32, dtype=np.float32)
    hk = np.ascontiguousarray(hkls, dtype=np.int32).reshape(-1, 3)
    out = _lib.LmbPostOutput()
    check(lib().lmb_post_process(C.byref(geometry), C.byref(pp), om.ctypes.data, om.shape[0],
                                 idv.ctypes.data, scv.ctypes.data, idv.shape[0], img.ctypes.data,
                                 hk.ctypes.data, hk.shape[0], C.byref(out)))
    try:
        sol = C.string_at(out.solutions, out.solutions_len).decode("latin-1")
        spt = C.string_at(out.spots, out.spots_len).decode("latin-1")
        n_unique = int(out.n_unique)
    finally:
        lib().lmb_post_free(C.byref(out))
    return sol, spt, n_unique


def last_refine_stats() -> dict:
    """What this thread's last post_process refined: ``device`` -2 (nothing),
    -1 (host threads) or the device ordinal; points, rounds and the
    objective kernel's time."""
    d, pts, rnd, km = C.c_int32(0), C.c_int64(0), C.c_int32(0), C.c_float(0)
    check(lib().lmb_post_last_refine_stats(C.byref(d), C.byref(pts), C.byref(rnd), C.byref(km)))
    return {"device": d.value, "points": pts.value, "rounds": rnd.value,
            "kernel_ms": float(km.value)}


def collected_matches(survivors, n_pass: int):
    """(ids, scores) as the reference hands them to the merge: survivors in
    ascending ID, followed by one (0, 0.0) entry for each orientation that
    passed both thresholds with a zero score (LaueMatchingCPU.c:773-788 sizes
    the arrays by nrResults but fills only the non-zero scores)."""
    ids = np.asarray(survivors["id"], dtype=np.uint64)
    sc = np.asarray(survivors["score"], dtype=np.float64)
    extra = int(n_pass) - ids.shape[0]
    if extra > 0:
        ids = np.concatenate([ids, np.zeros(extra, np.uint64)])
        sc = np.concatenate([sc, np.zeros(extra, np.float64)])
    return ids, sc


def merge_clusters(space_group: int, max_angle: float, orients: np.ndarray, rows, scores,
                   device: int | None = None, host_band: float = 0.0,
                   num_threads: int | None = None):
    """The duplicate merge alone: (best_rows, best_scores, counts) per cluster,
    in the reference's cluster order.  ``device`` runs it on that CUDA device
    (1024 or more candidates), None on the host."""
    om = np.ascontiguousarray(orients, dtype=np.float64).reshape(-1, 9)
    rv = np.ascontiguousarray(rows, dtype=np.uint64)
    sv = np.ascontiguousarray(scores, dtype=np.float64)
    n = rv.shape[0]
    br = np.zeros(max(n, 1), np.uint64)
    bs = np.zeros(max(n, 1), np.float64)
    cn = np.zeros(max(n, 1), np.int32)
    nc = C.c_int32(0)
    check(lib().lmb_merge_clusters(-1 if device is None else int(device), int(space_group),
                                   float(max_angle), float(host_band), om.ctypes.data,
                                   om.shape[0], rv.ctypes.data, sv.ctypes.data, n,
                                   int(num_threads or os.cpu_count() or 1), C.byref(nc),
                                   br.ctypes.data, bs.ctypes.data, cn.ctypes.data))
    k = nc.value
    return br[:k].copy(), bs[:k].copy(), cn[:k].copy()

