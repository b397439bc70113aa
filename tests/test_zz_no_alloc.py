"""Survivor ordering that allocates nothing (lmb_order_survivors_noalloc).

For callers that cannot call cudaMalloc but hold device buffers (memory from
another framework's pool, or a thread that must not synchronise the device
through an allocation): the entry point orders an unsorted survivor list with
a fixed device array inside the library as scratch.  Its output must equal
what the engine's own path delivers through lmb_results, bit for bit, on two
calls in a row (the scratch keeps the previous call's contents).

Collected last (file name) so that a failure here does not hide the others.
"""
import ctypes as C

import numpy as np
import pytest

from lauematching_b200 import synth, params as P
from lauematching_b200._lib import LMB_ERR_INVALID, LMB_NOALLOC_ORDER_MAX, check, lib
from lauematching_b200.engine import SURVIVOR_DTYPE, Engine

pytestmark = pytest.mark.gpu


def _engine_survivors():
    """Sorted survivors of one pass, from the existing entry point, large
    enough (> 8192) to need the scratch array."""
    txt = synth.params_text(nr_px=(256, 256), max_nr_spots=7, min_nr_spots=1,
                            min_intensity=1.0)
    p = P.parse_params_text(txt)
    rng = np.random.default_rng(21)
    n = 60000
    rec = np.zeros((n, 15), np.uint16)
    rec[:, 0] = rng.integers(0, 8, n)
    rec[:, 1::2] = rng.integers(0, 256, (n, 7))
    rec[:, 2::2] = rng.integers(0, 256, (n, 7))
    img = np.where(rng.random(256 * 256) < 0.4, rng.integers(1, 256, 256 * 256), 0)
    with Engine(p) as e:
        e.upload_db(rec)
        e.load_image(0, img.astype(np.float64) * 0.9)
        e.match([0], p.min_nr_spots, p.min_intensity)
        ref, _ = e.results(0)
    return ref


def _order_on_device(unsorted):
    import torch
    d_in = torch.from_numpy(unsorted.view(np.uint8).copy()).cuda()
    d_out = torch.zeros_like(d_in)
    stream = torch.cuda.current_stream().cuda_stream
    check(lib().lmb_order_survivors_noalloc(d_in.data_ptr(), unsorted.shape[0],
                                            d_out.data_ptr(), stream))
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(SURVIVOR_DTYPE)


def _expected_order(lst):
    """Ascending id, ties by position in the unsorted list."""
    return lst[np.lexsort((np.arange(lst.shape[0]), lst["id"]))]


def test_noalloc_order_equals_engine_order_twice():
    ref = _engine_survivors()
    assert ref.shape[0] > 8192  # large enough for the scratch array
    rng = np.random.default_rng(5)
    for _ in range(2):  # second call sees the first call's scratch contents
        got = _order_on_device(ref[rng.permutation(ref.shape[0])])
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_noalloc_order_small_list_and_limits():
    ref = _engine_survivors()[:3000]  # fits in shared memory
    rng = np.random.default_rng(6)
    for _ in range(2):
        got = _order_on_device(ref[rng.permutation(ref.shape[0])])
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    # sizes beyond the fixed scratch are rejected before any device work
    rc = lib().lmb_order_survivors_noalloc(C.c_void_p(16), LMB_NOALLOC_ORDER_MAX + 1,
                                           C.c_void_p(32), None)
    assert rc == LMB_ERR_INVALID
    assert b"LMB_NOALLOC_ORDER_MAX" in lib().lmb_last_error()
    assert lib().lmb_order_survivors_noalloc(None, 0, None, None) == 0


def test_noalloc_order_of_ids_beyond_40_bits():
    """Ids of 2^40 and above (which a packed id << 24 key cannot hold) and
    repeated ids are still ordered by (id, position), in shared memory and
    in the scratch array."""
    base = _engine_survivors()
    rng = np.random.default_rng(8)
    for n in (2500, 20000):
        lst = base[rng.permutation(base.shape[0])[:n]].copy()
        lst["id"][::3] += np.uint64(1) << np.uint64(41)
        lst["id"][1::7] = lst["id"][0]
        for _ in range(2):
            got = _order_on_device(lst)
            assert np.array_equal(got.view(np.uint8), _expected_order(lst).view(np.uint8))


def test_noalloc_order_rejects_overlapping_buffers():
    """The output may not overlap the input at all (the last step reads the
    input while writing the output): equal, partly overlapping either way."""
    import torch
    n = 100
    buf = torch.zeros(3 * n * SURVIVOR_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    b = buf.data_ptr()
    sz = SURVIVOR_DTYPE.itemsize
    for d_in, d_out in ((b, b), (b, b + 10 * sz), (b + 10 * sz, b), (b, b + (n - 1) * sz)):
        rc = lib().lmb_order_survivors_noalloc(C.c_void_p(d_in), n, C.c_void_p(d_out), None)
        assert rc == LMB_ERR_INVALID
        assert b"overlap" in lib().lmb_last_error()
    # adjacent ranges are fine
    check(lib().lmb_order_survivors_noalloc(C.c_void_p(b), n, C.c_void_p(b + n * sz), None))
    torch.cuda.synchronize()
