"""Python host API over the C ABI: one engine per (device, detector geometry).

An :class:`Engine` keeps the forward-simulated DB resident in HBM together
with up to 64 image slots; :meth:`Engine.match` runs one DB pass for any set
of loaded slots and :meth:`Engine.results` returns each slot's survivors in
ascending orientation ID, with the reference's integer and FP64 values.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .params import LaueParams

__all__ = ["SURVIVOR_DTYPE", "geometry_from_params", "Engine", "PinnedBuffer"]

SURVIVOR_DTYPE = np.dtype([("id", "<u8"), ("n_spots", "<i4"), ("sum_u8", "<i4"),
                           ("tot_int", "<f8"), ("score", "<f8")])
assert SURVIVOR_DTYPE.itemsize == C.sizeof(_lib.LmbSurvivor)

_DTYPES = {np.dtype(np.float64): _lib.LMB_F64, np.dtype(np.float32): _lib.LMB_F32,
           np.dtype(np.uint8): _lib.LMB_U8}


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def geometry_from_params(p: LaueParams) -> _lib.LmbGeometry:
    g = _lib.LmbGeometry()
    lat = np.asarray(p.lattice, np.float64)
    pa = np.asarray(p.p_array, np.float64)
    ra = np.asarray(p.r_array, np.float64)
    check(lib().lmb_geometry_init(_dptr(lat), int(p.space_group), _dptr(pa), _dptr(ra),
                                  float(p.px_x), float(p.px_y), int(p.nr_px_x), int(p.nr_px_y),
                                  float(p.elo), float(p.ehi), int(p.max_nr_spots), C.byref(g)))
    return g


class PinnedBuffer:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, shape, dtype):
        self.dtype = np.dtype(dtype)
        n = int(np.prod(shape)) * self.dtype.itemsize
        p = C.c_void_p()
        check(lib().lmb_host_alloc(n, C.byref(p)))
        self._p = p
        buf = (C.c_byte * max(n, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self._p is not None:
            self.array = None
            lib().lmb_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:  # interpreter shutdown
            pass


class Engine:
    def __init__(self, params: LaueParams, device: int = 0, survivor_capacity: int = 0):
        self.params = params
        self.device = int(device)
        self.geometry = geometry_from_params(params)
        self.S = int(params.max_nr_spots)
        self.R = 1 + 2 * self.S
        self.npx = int(params.nr_px_x) * int(params.nr_px_y)
        h = C.c_void_p()
        check(lib().lmb_engine_create(int(device), C.byref(self.geometry),
                                      int(survivor_capacity), C.byref(h)))
        self._h = h
        self.n_orient = 0
        self._pinned_shape = False
        self._shape_bucket = None

    # ---- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().lmb_engine_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(lib().lmb_engine_stream(self._h) or 0)

    TUNING_FIELDS = ("variant", "tile_sub", "stages", "consumers", "blocks_per_sm", "grid_mult",
                     "full_gather")

    def set_tuning(self, test_consumer_wait_us: int = 0, cell_consumers: int = 0,
                   cell_stages: int = 0, cell_queue: int = 0, **kw) -> None:
        """Pin the compare pass's launch shape (TUNING_FIELDS; variant 3 =
        automatic when not given; cell_consumers / cell_stages shape the
        cell-mask pass when the automatic variant picks it).
        test_consumer_wait_us is for tests only: the pass gives up after that
        wait and reports a timeout."""
        check(lib().lmb_engine_set_tuning(
            self._h, self._tuning_vals(kw, test_consumer_wait_us, cell_consumers, cell_stages,
                                       cell_queue), 11))
        self._pinned_shape = True

    def _tuning_vals(self, kw, test_wait=0, cell_consumers=0, cell_stages=0, cell_queue=0):
        vals = (C.c_int32 * 11)(*[int(kw.get(f, 0)) for f in self.TUNING_FIELDS],
                                int(test_wait), int(cell_consumers), int(cell_stages),
                                int(cell_queue))
        if "variant" not in kw:
            vals[0] = 3
        return vals

    def set_sparse_uploads(self, enable: bool) -> None:
        check(lib().lmb_engine_set_sparse_uploads(self._h, int(bool(enable))))

    def set_dense_share(self, share: float) -> None:
        """Share of the page-locked frames of a load_images call sent dense
        over the copy engine while the host scans the others."""
        check(lib().lmb_engine_set_dense_share(self._h, float(share)))

    def layout_info(self) -> dict:
        """State of the compact device layout (compare variant 2)."""
        st, nb = C.c_int32(0), C.c_uint64(0)
        tr, tb = C.c_int32(0), C.c_int32(0)
        check(lib().lmb_engine_layout_info(self._h, C.byref(st), C.byref(nb), C.byref(tr),
                                           C.byref(tb)))
        return {"compact": st.value, "bytes": int(nb.value), "tiles": tr.value,
                "tile_bytes": tb.value}

    def get_tuning(self) -> dict:
        """The shape set (variant 3 = automatic) and ``last_variant``, the
        variant the latest pass ran."""
        vals = (C.c_int32 * 8)()
        check(lib().lmb_engine_get_tuning(self._h, vals, 8))
        return dict(zip(self.TUNING_FIELDS + ("last_variant",), list(vals)))

    # ---- DB -------------------------------------------------------------------
    def upload_db(self, records: np.ndarray) -> None:
        rec = np.ascontiguousarray(records, dtype=np.uint16).reshape(-1, self.R)
        check(lib().lmb_db_upload(self._h, rec.ctypes.data, rec.shape[0]))
        self.n_orient = rec.shape[0]

    def build_db(self, orients: np.ndarray, hkls: np.ndarray, exact_fp64: bool = False) -> None:
        om = np.ascontiguousarray(orients, dtype=np.float64).reshape(-1, 9)
        hk = np.ascontiguousarray(hkls, dtype=np.int32).reshape(-1, 3)
        flags = _lib.LMB_BUILD_EXACT_FP64 if exact_fp64 else 0
        check(lib().lmb_db_build_ex(self._h, om.ctypes.data, om.shape[0], hk.ctypes.data,
                                    hk.shape[0], flags))
        self.n_orient = om.shape[0]

    def build_db_synthetic(self, seed: int, n: int, hkls: np.ndarray,
                           return_orients: bool = False, hex_fz: bool = False):
        """DB of n device-generated uniform rotations (seeded); ``hex_fz``
        reduces them to the hexagonal fundamental zone first."""
        hk = np.ascontiguousarray(hkls, dtype=np.int32).reshape(-1, 3)
        out = np.empty((n, 9), np.float64) if return_orients else None
        flags = _lib.LMB_BUILD_SYNTH_HEX_FZ if hex_fz else 0
        check(lib().lmb_db_build_synthetic_ex(self._h, int(seed), int(n), hk.ctypes.data,
                                              hk.shape[0],
                                              out.ctypes.data if out is not None else None, flags))
        self.n_orient = n
        self._synth_flags = flags
        return out

    def synth_orientations(self, seed: int, first: int, n: int,
                           hex_fz: bool | None = None) -> np.ndarray:
        """Matrices of the synthetic generator (those of the last synthetic
        build unless ``hex_fz`` says otherwise)."""
        flags = getattr(self, "_synth_flags", 0) if hex_fz is None else \
            (_lib.LMB_BUILD_SYNTH_HEX_FZ if hex_fz else 0)
        out = np.empty((n, 9), np.float64)
        check(lib().lmb_synth_orientations_ex(self._h, int(seed), int(first), int(n),
                                              out.ctypes.data, flags))
        return out

    def download_db(self, first: int = 0, count: int | None = None) -> np.ndarray:
        if count is None:
            count = self.n_orient - first
        out = np.empty((count, self.R), np.uint16)
        check(lib().lmb_db_download(self._h, first, count, out.ctypes.data))
        return out

    # ---- images ---------------------------------------------------------------
    def load_image(self, slot: int, pixels: np.ndarray, keep_f64: bool = False,
                   want_scale: bool = True):
        px = np.ascontiguousarray(pixels).ravel()
        if px.size != self.npx:
            raise ValueError(f"image has {px.size} pixels, detector has {self.npx}")
        dt = _DTYPES.get(px.dtype)
        if dt is None:
            px = px.astype(np.float64)
            dt = _lib.LMB_F64
        sc = C.c_double(0.0)
        check(lib().lmb_image_load(self._h, int(slot), px.ctypes.data, dt, int(bool(keep_f64)),
                                   C.byref(sc) if want_scale else None))
        return sc.value if want_scale else None

    def load_images(self, slots, frames, want_scales: bool = False):
        """Load several frames (one dtype) into distinct slots with one
        library call: each slot ends as after ``load_image(slot, frame)``.
        Returns the imScale of each frame when ``want_scales``."""
        sl = np.ascontiguousarray(list(slots), dtype=np.int32)
        n = sl.shape[0]
        if len(frames) != n:
            raise ValueError(f"{n} slots for {len(frames)} frames")
        pxs = []
        dt = None
        for f in frames:
            px = np.ascontiguousarray(f).ravel()
            if px.size != self.npx:
                raise ValueError(f"image has {px.size} pixels, detector has {self.npx}")
            if px.dtype not in _DTYPES:
                px = px.astype(np.float64)
            if dt is None:
                dt = px.dtype
            elif px.dtype != dt:
                raise ValueError("frames of one batch share a dtype")
            pxs.append(px)
        ptrs = (C.c_void_p * max(n, 1))(*[p.ctypes.data for p in pxs])
        sc = np.zeros(max(n, 1), np.float64)
        check(lib().lmb_image_load_batch(self._h, sl.ctypes.data, ptrs, n,
                                         _DTYPES[dt] if n else _lib.LMB_U8,
                                         _dptr(sc) if want_scales else None))
        return sc[:n].tolist() if want_scales else None

    # ---- passes ---------------------------------------------------------------
    def _apply_table_shape(self, k: int) -> None:
        """Use the autotuned launch shape for passes of k images, unless the
        caller fixed one with set_tuning."""
        if self._pinned_shape:
            return
        from .autotune import batch_bucket, lookup
        b = batch_bucket(k)
        if b != self._shape_bucket:
            shape = lookup(self.R, b)
            dense = lookup(self.R, b, dense=True) or {}
            if shape:
                check(lib().lmb_engine_set_tuning(
                    self._h, self._tuning_vals(shape, 0, dense.get("consumers", 0),
                                               dense.get("stages", 0),
                                               dense.get("cell_queue", 0)), 11))
            self._shape_bucket = b

    def match(self, slots, min_nr_spots: int, min_intensity: float, value_mode: int = 0) -> None:
        mask = 0
        n = 0
        for s in slots:
            mask |= 1 << int(s)
            n += 1
        self._apply_table_shape(n)
        check(lib().lmb_match(self._h, mask, int(min_nr_spots), float(min_intensity),
                              int(value_mode)))

    def results(self, slot: int):
        """(survivors structured array sorted by id, n_pass)."""
        n = C.c_uint64(0)
        npass = C.c_uint64(0)
        check(lib().lmb_results(self._h, int(slot), None, 0, C.byref(n), C.byref(npass)))
        out = np.empty(n.value, SURVIVOR_DTYPE)
        if n.value:
            check(lib().lmb_results(self._h, int(slot), out.ctypes.data, n.value, C.byref(n),
                                    C.byref(npass)))
        return out, int(npass.value)

    def results_batch(self, slots):
        """{slot: (survivors, n_pass)} for several slots with one library call
        per pass (a second one only when the survivors outgrow the buffer)."""
        sl = np.ascontiguousarray(list(slots), dtype=np.int32)
        n = sl.shape[0]
        counts = np.zeros(n, np.uint64)
        npass = np.zeros(n, np.uint64)
        cap = max(getattr(self, "_rb_cap", 4096), 1)
        while True:
            out = np.empty(cap, SURVIVOR_DTYPE)
            rc = lib().lmb_results_batch(self._h, sl.ctypes.data, n, out.ctypes.data, cap,
                                         counts.ctypes.data, npass.ctypes.data)
            total = int(counts.sum())
            if rc == _lib.LMB_ERR_OVERFLOW and total > cap:
                cap = total
                self._rb_cap = total
                continue
            check(rc)
            break
        res, off = {}, 0
        for i, s in enumerate(sl.tolist()):
            c = int(counts[i])
            res[s] = (out[off:off + c].copy(), int(npass[i]))
            off += c
        return res

    def last_pass_ms(self):
        a, b = C.c_float(0), C.c_float(0)
        check(lib().lmb_last_pass_ms(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def bytes_moved(self):
        """(host->device, device->host) bytes since the engine was created."""
        a, b = C.c_uint64(0), C.c_uint64(0)
        check(lib().lmb_engine_bytes(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)
