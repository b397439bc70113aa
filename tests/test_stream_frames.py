"""The daemon's receive buffers (stream.FramePool), on the host (no GPU).

Buffers are reused across messages per (pixel count, dtype); float32 wire
frames may be page-locked within a byte budget, and where page-locked memory
cannot be had (no device here) the pool falls back to ordinary memory and
keeps its budget.  Arrays the pool did not make are ignored on return.
"""
import numpy as np

from lauematching_b200.stream import FramePool


def test_buffers_are_reused_per_size_and_dtype():
    fp = FramePool(pinned_bytes=0)
    a = fp.get(64 * 64, np.float32)
    b = fp.get(64 * 64, np.uint8)
    assert a.dtype == np.float32 and a.size == 64 * 64 and b.dtype == np.uint8
    fp.put(a)
    fp.put(b)
    assert fp.get(64 * 64, np.float32) is a
    assert fp.get(64 * 64, np.uint8) is b
    c = fp.get(64 * 64, np.float32)  # the pool's only float32 buffer is out: a new one
    assert c is not a
    fp.put(np.empty(64 * 64, np.float32))  # not the pool's: ignored
    fp.put(c)
    assert fp.get(64 * 64, np.float32) is c
    fp.close()


def test_prefill_makes_buffers_once():
    fp = FramePool(pinned_bytes=0)
    fp.prefill(1000, np.float32, 5)
    got = [fp.get(1000, np.float32) for _ in range(5)]
    assert len({id(g) for g in got}) == 5
    for g in got:
        fp.put(g)
    fp.prefill(1000, np.float32, 5)  # already made: nothing new
    again = [fp.get(1000, np.float32) for _ in range(5)]
    assert {id(g) for g in again} == {id(g) for g in got}
    fp.close()


def test_page_locked_budget_falls_back_to_ordinary_memory_without_a_device():
    # 2 buffers' worth of budget; without a usable device the page-locked
    # allocation fails, the buffer is ordinary memory and the budget is kept
    fp = FramePool(pinned_bytes=2 * 4 * 256)
    bufs = [fp.get(256, np.float32) for _ in range(4)]
    assert all(b.size == 256 and b.dtype == np.float32 for b in bufs)
    for b in bufs:
        b[:] = 1.0  # writable
    u8 = fp.get(256, np.uint8)  # uint8 frames are never page-locked
    assert u8.dtype == np.uint8
    fp.close()
