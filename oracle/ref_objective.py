"""Test infrastructure only: ctypes access to the reference's own refinement
objective (_ref/libref_objective.so, built by ``make -C oracle ref-objective``
from ref_objective.c and the reference tree's LaueMatchingHeaders.h).

Used by the refinement parity tests and by bench.py's CPU baseline of the
refinement leg; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_objective.so")


def available() -> bool:
    return os.path.exists(LIB)


class RefObjective:
    """problem_function / prefilterHKLs / OrientMat2Euler of the reference for
    one parameter set (params: lauematching_b200.params.LaueParams, geometry:
    its lmb_geometry)."""

    def __init__(self, params, geometry, hkls):
        self.L = C.CDLL(LIB)
        dp, vp, i32, dbl = C.POINTER(C.c_double), C.c_void_p, C.c_int, C.c_double
        self.L.refobj_set_crystal.argtypes = [vp, vp, dbl, i32]
        self.L.refobj_euler.argtypes = [vp, vp]
        self.L.refobj_prefilter.argtypes = [vp, i32, vp, vp, i32, i32, vp, vp, dbl, dbl, dbl, dbl,
                                            vp]
        self.L.refobj_prefilter.restype = i32
        self.L.refobj_problem.argtypes = [C.c_uint, vp, vp, vp, i32, i32, i32, vp, vp, i32, vp,
                                          vp, dbl, dbl, dbl, dbl, vp, i32]
        self.L.refobj_problem.restype = dbl
        self.lat = np.array(params.lattice, np.float64)
        tca = float(params.tol_c_over_a)
        self.tca = tca
        self.tol = np.zeros(6) if tca != 0 else np.array(params.tol_latc, np.float64)
        self.L.refobj_set_crystal(self.lat.ctypes.data, self.tol.ctypes.data, tca,
                                  int(params.space_group))
        self.n = 4 if tca != 0 else 3 + int(np.count_nonzero(self.tol))
        self.g = geometry
        self.recip = np.array(geometry.recip[:], np.float64)
        self.rt = np.array(geometry.rot_t[:], np.float64)
        self.p = np.array(geometry.p[:], np.float64)
        self.hkls = np.ascontiguousarray(hkls, dtype=np.int32).reshape(-1, 3)
        self.max_spots = 3 * int(geometry.max_nr_spots)

    def euler(self, om) -> np.ndarray:
        m = np.ascontiguousarray(om, np.float64).reshape(9)
        e = np.zeros(3)
        self.L.refobj_euler(m.ctypes.data, e.ctypes.data)
        return e

    def prefilter(self, euler) -> np.ndarray:
        e = np.ascontiguousarray(euler, np.float64)
        out = np.zeros(self.hkls.shape[0], np.int32)
        g = self.g
        k = self.L.refobj_prefilter(self.hkls.ctypes.data, self.hkls.shape[0], e.ctypes.data,
                                    self.recip.ctypes.data, g.nr_px_x, g.nr_px_y,
                                    self.rt.ctypes.data, self.p.ctypes.data, g.px_x, g.px_y,
                                    g.elo, g.ehi, out.ctypes.data)
        return out[:k].copy()

    def problem(self, x, image_f32, valid) -> float:
        xv = np.ascontiguousarray(x, np.float64)
        im = np.ascontiguousarray(image_f32, np.float32)
        va = np.ascontiguousarray(valid, np.int32)
        g = self.g
        return float(self.L.refobj_problem(
            len(xv), xv.ctypes.data, im.ctypes.data, self.hkls.ctypes.data, self.hkls.shape[0],
            g.nr_px_x, g.nr_px_y, self.lat.ctypes.data, self.recip.ctypes.data, self.max_spots,
            self.rt.ctypes.data, self.p.ctypes.data, g.px_x, g.px_y, g.elo, g.ehi,
            va.ctypes.data, va.shape[0]))

    def start(self, om) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """FitOrientation's x, xl, xu (LaueMatchingHeaders.h:718-743) at the
        coarse matrix om, as fitAndWriteOrientations calls it."""
        e = self.euler(om)
        tol = 3 * 0.0174532925199433
        x, lo, hi = list(e), [v - tol for v in e], [v + tol for v in e]
        for i in range(6):
            if self.tol[i] != 0:
                x.append(self.lat[i])
                lo.append(self.lat[i] * (1 - self.tol[i]))
                hi.append(self.lat[i] * (1 + self.tol[i]))
        if self.tca != 0:
            ca = self.lat[2] / self.lat[0]
            x.append(ca)
            lo.append(ca * (1 - self.tca))
            hi.append(ca * (1 + self.tca))
        return np.array(x), np.array(lo), np.array(hi)
