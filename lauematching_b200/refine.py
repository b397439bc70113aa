"""Batched orientation refinement (FitOrientation over many grains at once).

Wraps the ``lmb_refine_*`` entry points of liblmb200.  The reference refines
each grain on its own host thread with NLopt, evaluating problem_function
(LaueMatchingHeaders.h:640-694 with calcOverlapFiltered :564-636) up to 200
times; fitAndWriteOrientations (:1072-1153) sets each fit up from the grain's
coarse orientation matrix (OrientMat2Euler, prefilterHKLs :513-561, the start
point and box of FitOrientation :718-743).  Here a :class:`Refiner` holds the
frames of a batch and the grains of all of them; objective evaluations of all
grains run together on a CUDA device, one launch per optimiser round, with
values bit-identical to the host's (``device=None`` evaluates on host threads
with the same arithmetic).

Optimisers: ``"once"`` evaluates at the start point and keeps it (the
reference built with an evaluate-once NLopt stand-in gives the same
numbers); ``"nelder-mead"`` is this library's own bounded Nelder-Mead, run in
lockstep over the grains.  NLopt is not available here, so the reference's
BOBYQA / NELDERMEAD trajectories are not reproduced.

    r = Refiner(params, geometry, hkls, device=0)
    r.set_images([frame0, frame1])                  # float32 (NrPxY, NrPxX)
    r.set_grains(orient_matrices, image_of_grain)   # coarse (g, 9) matrices
    x_fit, overlap, evals = r.fit("nelder-mead")
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .params import LaueParams
from .post import make_post_params

OPTIMIZERS = {"once": 0, "nelder-mead": 1}


class Refiner:
    def __init__(self, params: LaueParams, geometry, hkls: np.ndarray, device: int | None = 0,
                 num_threads: int | None = None):
        self._params = params
        self._geo = geometry
        self._pp = make_post_params(params, num_threads=num_threads)
        self._hkls = np.ascontiguousarray(hkls, dtype=np.int32).reshape(-1, 3)
        self.W, self.H = int(geometry.nr_px_x), int(geometry.nr_px_y)
        self.device = device
        h = C.c_void_p()
        check(lib().lmb_refine_create(-1 if device is None else int(device), C.byref(geometry),
                                      C.byref(self._pp), self._hkls.ctypes.data,
                                      self._hkls.shape[0], C.byref(h)))
        self._h = h
        n = C.c_int32()
        check(lib().lmb_refine_dims(self._h, C.byref(n)))
        self.dims = int(n.value)
        self.n_grains = 0

    def close(self):
        if self._h:
            lib().lmb_refine_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_images(self, frames):
        """Float frames of the batch, each (NrPxY, NrPxX) (the image the
        reference's post-stage refines against)."""
        fr = [np.ascontiguousarray(f, dtype=np.float32) for f in frames]
        for f in fr:
            if f.size != self.W * self.H:
                raise ValueError(f"frame of {f.size} pixels, expected {self.H}x{self.W}")
        ptrs = (C.c_void_p * max(1, len(fr)))(*[f.ctypes.data for f in fr])
        check(lib().lmb_refine_set_images(self._h, ptrs, len(fr)))
        self._frames = fr
        self.n_grains = 0

    def set_grains(self, orients: np.ndarray, image) -> np.ndarray:
        """Coarse orientation matrices (g, 9) and each grain's frame index;
        returns the prefiltered HKL count of every grain."""
        om = np.ascontiguousarray(orients, dtype=np.float64).reshape(-1, 9)
        im = np.ascontiguousarray(np.broadcast_to(np.asarray(image, np.int32), (om.shape[0],)))
        nv = np.zeros(max(1, om.shape[0]), np.int32)
        check(lib().lmb_refine_set_grains(self._h, om.ctypes.data, im.ctypes.data, om.shape[0],
                                          nv.ctypes.data))
        self.n_grains = om.shape[0]
        return nv[:self.n_grains].copy()

    def start(self):
        """(x0, lower, upper), each (n_grains, dims)."""
        shp = (self.n_grains, self.dims)
        x0, lo, hi = (np.zeros(shp) for _ in range(3))
        check(lib().lmb_refine_start(self._h, x0.ctypes.data, lo.ctypes.data, hi.ctypes.data))
        return x0, lo, hi

    def evaluate(self, grain, x) -> np.ndarray:
        """problem_function at points x (m, dims) of grains grain (m,)."""
        xv = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, self.dims)
        gv = np.ascontiguousarray(np.broadcast_to(np.asarray(grain, np.int32), (xv.shape[0],)))
        out = np.zeros(max(1, xv.shape[0]))
        check(lib().lmb_refine_evaluate(self._h, gv.ctypes.data, xv.ctypes.data, xv.shape[0],
                                        out.ctypes.data))
        return out[:xv.shape[0]].copy()

    def fit(self, optimizer: str = "once", max_eval: int = 200, init_step: float = 0.0):
        """(x_fit (g, dims), overlap (g,), evaluations (g,)).  init_step: the
        Nelder-Mead start simplex's step per coordinate as a fraction of its
        box width (0: the library's default, 0.02)."""
        g = self.n_grains
        x = np.zeros((max(1, g), self.dims))
        ov = np.zeros(max(1, g))
        ev = np.zeros(max(1, g), np.int32)
        check(lib().lmb_refine_fit(self._h, OPTIMIZERS[optimizer], int(max_eval),
                                   float(init_step), x.ctypes.data, ov.ctypes.data,
                                   ev.ctypes.data))
        return x[:g].copy(), ov[:g].copy(), ev[:g].copy()

    def last_stats(self) -> dict:
        p, r, ms = C.c_int64(), C.c_int32(), C.c_float()
        check(lib().lmb_refine_last_stats(self._h, C.byref(p), C.byref(r), C.byref(ms)))
        return {"points": int(p.value), "rounds": int(r.value), "kernel_ms": float(ms.value)}
