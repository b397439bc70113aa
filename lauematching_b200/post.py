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


def post_process(params: LaueParams, geometry, orients: np.ndarray, ids: np.ndarray,
                 scores: np.ndarray, image_f32: np.ndarray, hkls: np.ndarray,
                 min_nr_spots: int | None = None, image_num: int = 0,
                 num_threads: int | None = None, max_results: int = 0):
    """Return (solutions_text, spots_text, n_unique) for one image.

    ``ids``/``scores`` are the image's collected matches in the reference's
    collection order (ascending orientation ID).  ``max_results`` > 0 keeps
    only that many top-scored candidates for the merge (the reference's own
    cap path, LaueMatchingHeaders.h:976-997, with its cap of 50000 lowered)."""
    pp = _lib.LmbPostParams()
    for i in range(6):
        pp.lattice[i] = params.lattice[i]
        pp.tol_latc[i] = params.tol_latc[i]
    pp.space_group = int(params.space_group)
    pp.max_nr_spots = int(params.max_nr_spots)
    pp.tol_c_over_a = float(params.tol_c_over_a)
    pp.max_angle = float(params.max_angle)
    pp.min_nr_spots = int(params.min_nr_spots if min_nr_spots is None else min_nr_spots)
    pp.image_num = int(image_num)
    pp.num_threads = int(num_threads or os.cpu_count() or 1)
    pp.optimizer = 0
    pp.max_results = int(max_results)  # 0: the reference's 50000
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
