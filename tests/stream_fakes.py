"""Host-side stand-in for the engine, for daemon tests that need no GPU.

FakeEngine takes the calls the stream daemon makes (load_images, match,
results_batch, close), records the frames it was given, and returns empty
survivor lists; ``pass_seconds`` keeps each pass "on the device" that long
before its results can be read, so a test can act while a pass is in flight.
"""
import threading
import time

import numpy as np

SURV = np.dtype([("id", "<u8"), ("n_spots", "<i4"), ("sum_u8", "<i4"),
                 ("tot_int", "<f8"), ("score", "<f8")])


class FakeEngine:
    geometry = None

    def __init__(self, pass_seconds=0.0, hold=None):
        self.pass_seconds = pass_seconds
        self.hold = hold  # threading.Event: results wait until it is set
        self.lock = threading.Lock()
        self.frames = []   # every loaded frame, in load order
        self.passes = []   # slots of every pass
        self.inflight = 0

    def set_dense_share(self, share):
        self.dense_share = share

    def load_images(self, slots, frames):
        with self.lock:
            self.frames += [np.array(f, copy=True) for f in frames]

    def match(self, slots, min_nr_spots, min_intensity, value_mode=0):
        with self.lock:
            self.passes.append(list(slots))
            self.inflight += 1

    def results_batch(self, slots):
        if self.hold is not None:
            self.hold.wait(30)
        if self.pass_seconds:
            time.sleep(self.pass_seconds)
        with self.lock:
            self.inflight -= 1
        return {s: (np.zeros(0, SURV), 0) for s in slots}

    def close(self):
        pass


def make_server(tmp_dir, port, ext_port, engine, nr_px=(64, 64), max_batch=4, max_queue=32):
    from lauematching_b200 import params as P, synth
    from lauematching_b200.stream import StreamServer
    p = P.parse_params_text(synth.params_text(nr_px=nr_px) + "MinGoodSpots 5\n", binary="stream")
    return StreamServer([p], np.zeros((1, 9)), np.zeros((1, 3), np.int32), ncpus=1,
                        max_batch=max_batch, result_dir=str(tmp_dir), port=port,
                        ext_port=ext_port, host="127.0.0.1", log=lambda *a: None,
                        engines=[engine], max_queue=max_queue, free_bytes=1 << 34,
                        pinned_bytes=0)
