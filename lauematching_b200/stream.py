"""``LaueMatchingGPUStream`` daemon, drop-in for the reference executable.

    LaueMatchingGPUStream <params.txt> <orientations.bin> <hkls.csv> <nCPUs>
        [--extra-params other_detector.txt ...] [--max-batch 64] [--device 0]

Wire protocol of the reference (LaueMatchingGPUStream.cu:42-46,295-383;
client scripts/laue_stream_utils.py:553-565): TCP port 60517, each message a
2-byte host-endian image number followed by NrPxX*NrPxY float32 pixels, many
messages per connection, no reply.  Results are appended, one image at a
time and flushed, to ``<cwd>/<ResultDir>/solutions.txt`` and ``spots.txt``
with the ImageNr column (LaueMatchingGPUStream.cu:1079-1104); the written
grains are gated by MinGoodSpots (:1173).  SIGINT/SIGTERM: stop accepting,
finish every received image, exit 0.

What changes (the serving side of the B200 design):

* continuous batching -- the reference runs one full DB pass per image with
  kernels serialised (gpu_gate, :1160-1165, :1196, :1248).  Here every image
  that arrives while a pass is running is uploaded into a free slot (the
  upload overlaps the pass on its own stream) and joins the next pass; one
  pass serves up to 64 images;
* admission by memory budget -- slots per geometry are limited by the free
  HBM after the DB is resident, and the per-pixel occupancy word keeps the
  L2-resident working set at 8 bytes per pixel whatever the batch;
* mixed detector sizes -- ``--extra-params`` adds further detector
  geometries, each with its own resident DB; frames for them arrive on port
  60518 with an extended header (``b"LMB2"``, uint16 image number, uint16
  width, uint16 height, uint8 dtype 0=float32/1=uint8/2=raw uint16, one pad
  byte);
* raw detector frames -- dtype 2 on the extended port is an unprocessed
  uint16 frame: the daemon runs the image server's preprocessing
  (``laue_index.preprocess.preprocess_image``, configured by the same keys
  of the parameter file, background from BackgroundFile or the median of
  the geometry's first raw frame, as ``scripts/laue_image_server.py:160-176``)
  on the device, straight into the frame's slot; the blurred frame the
  matcher read (float32, as the image server would have sent it) feeds the
  post-stage; a frame without spots is finished without lines (the image
  server does not send it, ``laue_image_server.py:76-77``);
* the post-stage (merge, refinement, text) runs on a writer thread, off the
  GPU loop; per-image latency (arrival -> lines written) is recorded and
  p50/p99 reported.
"""
from __future__ import annotations

import argparse
import collections
import os
import queue
import signal
import socket
import struct
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np

PORT = 60517
EXT_PORT = 60518
MAX_CONNECTIONS = 10
MAX_QUEUE = 32
EXT_MAGIC = b"LMB2"
RCVBUF = 32 << 20
PINNED_BYTES = 2 << 30  # page-locked receive buffers (the rest are ordinary memory)
EXT_HEADER = struct.Struct("<4sHHHBB")
_SURV_DTYPE = np.dtype([("id", "<u8"), ("n_spots", "<i4"), ("sum_u8", "<i4"),
                        ("tot_int", "<f8"), ("score", "<f8")])


@dataclass
class Request:
    image_num: int
    key: tuple  # (NrPxX, NrPxY)
    pixels: np.ndarray
    t_arrival: float
    raw: bool = False  # an unprocessed detector frame, preprocessed on the device


@dataclass
class Done:
    req: Request
    survivors: np.ndarray
    n_pass: int
    t_gpu_done: float


@dataclass
class Geometry:
    params: object
    engine: object
    free: list = field(default_factory=list)
    loaded: list = field(default_factory=list)  # (slot, Request) uploaded, waiting for a pass
    # passes on the device, oldest first, each a list of (slot, Request); a
    # second pass queues behind the running one while its results are read
    inflight: collections.deque = field(default_factory=collections.deque)
    pre_cfg: dict = None  # preprocessing configuration for raw frames
    pool: object = None   # PreprocessPool, made on the first raw frame


class FramePool:
    """Receive buffers reused across messages, per (pixel count, dtype): a
    fresh 16 MiB array per frame costs its page faults on every message.  A
    buffer goes back to the pool when its image is finished (or dropped);
    arrays the pool did not make are ignored on return.

    Up to ``pinned_bytes`` of the float32 buffers (the reference's wire
    frames, 16 MiB at 2048^2) are page-locked: the engine sends such frames to
    the device over the copy engine (its dense share) instead of scanning them
    on host threads, which leaves the host's cores to the socket receives.
    uint8 frames stay in ordinary memory: their host scan is cheap and sends
    only the positive pixels.  Buffers beyond the budget are ordinary memory."""

    def __init__(self, pinned_bytes=0, pin_dtypes=(np.float32,)):
        self._pin_dtypes = {np.dtype(d).str for d in pin_dtypes}
        self._lock = threading.Lock()
        self._free: dict = collections.defaultdict(list)
        self._mine: set = set()
        self._pinned_left = int(pinned_bytes)
        self._keep: list = []  # the page-locked allocations, alive as long as the pool
        self._made: dict = {}  # buffers made per (pixel count, dtype)

    def _alloc(self, n, dtype):
        nb = int(n) * np.dtype(dtype).itemsize
        with self._lock:
            pin = np.dtype(dtype).str in self._pin_dtypes and nb <= self._pinned_left
            if pin:
                self._pinned_left -= nb
        if pin:
            from .engine import PinnedBuffer
            try:
                pb = PinnedBuffer((int(n),), dtype)
            except Exception:  # no page-locked memory to be had: ordinary buffer
                with self._lock:
                    self._pinned_left += nb
            else:
                with self._lock:
                    self._keep.append(pb)
                return pb.array
        return np.empty(int(n), dtype)

    def prefill(self, n, dtype, count):
        """Make up to ``count`` buffers of n pixels of dtype ahead of the
        first frames (page-locking costs milliseconds per buffer)."""
        k = (int(n), np.dtype(dtype).str)
        with self._lock:
            have = self._made.get(k, 0)
        for _ in range(max(0, int(count) - have)):
            a = self._alloc(n, dtype)
            with self._lock:
                self._mine.add(id(a))
                self._made[k] = self._made.get(k, 0) + 1
                self._free[k].append(a)

    def get(self, n, dtype):
        k = (int(n), np.dtype(dtype).str)
        with self._lock:
            if self._free[k]:
                return self._free[k].pop()
        a = self._alloc(n, dtype)
        with self._lock:
            self._mine.add(id(a))
            self._made[k] = self._made.get(k, 0) + 1
        return a

    def close(self):
        """Free the page-locked buffers (after the last frame is finished)."""
        with self._lock:
            keep, self._keep = self._keep, []
            self._free.clear()
            self._mine.clear()
            self._made.clear()
        for pb in keep:
            pb.free()

    def put(self, a):
        if a is None:
            return
        with self._lock:
            if id(a) in self._mine:
                self._free[(a.size, a.dtype.str)].append(a)


def _recv_exact(sock, buf, running):
    view = memoryview(buf)
    got = 0
    while got < len(buf):
        try:
            n = sock.recv_into(view[got:])
        except (socket.timeout, BlockingIOError):  # the receive timeout ran out
            if not running():
                return False
            continue
        except InterruptedError:
            continue
        except OSError:
            return False
        if n == 0:
            return False
        got += n
    return True


class StreamServer:
    """The daemon, usable in-process (tests, benchmarks) or from the CLI.

    pinned_bytes: page-locked budget of the receive buffers (float32 frames);
    dense_share: the share of page-locked frames each engine sends over the
    copy engine (set on the engines, including engines passed in, for as long
    as they live); frame_pool: a FramePool kept across servers (its owner
    closes it), else the server makes and frees its own."""

    def __init__(self, params_list, orients, hkls, ncpus=1, max_batch=64, device=0,
                 result_dir=None, port=PORT, ext_port=EXT_PORT, host="0.0.0.0",
                 log=print, max_queue=MAX_QUEUE, engines=None, preprocess_cfgs=None,
                 free_bytes=None, pinned_bytes=PINNED_BYTES, dense_share=1.0,
                 frame_pool=None):
        from . import _lib, formats
        from .engine import Engine
        self.log = log
        self.device = int(device)
        self.ncpus = max(1, int(ncpus))
        # images are post-processed concurrently, each on few threads
        self.n_writers = max(1, min(8, self.ncpus))
        self.post_threads = max(1, self.ncpus // self.n_writers)
        self._out_lock = threading.Lock()
        self.orients = orients
        self.hkls = hkls
        self.primary = params_list[0]
        self.result_dir = result_dir if result_dir is not None else self.primary.result_dir
        self.geoms: dict = {}
        for i, p in enumerate(params_list):
            key = (int(p.nr_px_x), int(p.nr_px_y))
            if key in self.geoms:
                raise ValueError(f"two parameter files describe a {key} detector")
            pcfg = preprocess_cfgs[i] if preprocess_cfgs else None
            if engines is not None:  # DBs already resident (in-process use)
                self.geoms[key] = Geometry(p, engines[i], pre_cfg=pcfg)
                continue
            e = Engine(p, device=device)
            fwd = p.forward_file
            if p.do_fwd == 0 and fwd and os.path.exists(fwd):
                e.upload_db(formats.read_forward_cache(fwd, orients.shape[0], p.max_nr_spots))
                log(f"{fwd} file was found. Will not do forward simulation.")
            else:
                t0 = time.perf_counter()
                e.build_db(orients, hkls)
                log(f"Forward simulation on the device: {orients.shape[0]} orientations in "
                    f"{time.perf_counter() - t0:.2f} s")
                if fwd:
                    from .cli import _write_cache
                    try:
                        _write_cache(e, fwd, orients.shape[0])
                    except OSError as exc:
                        log(f"Could not write the forward simulation to {fwd}: {exc}")
            self.geoms[key] = Geometry(p, e, pre_cfg=pcfg)
        # admission: slots per geometry within the free HBM after the DBs
        # (free_bytes: the caller's figure, for engines it manages itself)
        free = _lib.device_info(device)["free"] if free_bytes is None else int(free_bytes)
        per_slot = max(int(k[0]) * int(k[1]) * 5 for k in self.geoms)  # u8 frame + wire staging
        budget = max(1, int(0.5 * free // per_slot))
        self.max_batch = int(min(max_batch, 64, budget))
        for g in self.geoms.values():
            g.free = list(range(self.max_batch))[::-1]
        self.queue: queue.Queue = queue.Queue(maxsize=max_queue)
        # receive buffers: page-locked up to pinned_bytes; that share of them
        # goes to the device over the copy engine (dense_share of the
        # engines), the others through the host scan
        # (frame_pool: a caller's pool, kept across servers; the caller closes it)
        self._own_frames = frame_pool is None
        self.frames = FramePool(pinned_bytes) if frame_pool is None else frame_pool
        for g in self.geoms.values():
            g.engine.set_dense_share(dense_share)
        self._backlog = collections.deque()
        self.done_q: queue.Queue = queue.Queue()
        self.running = False
        self.latencies_ms: list = []
        self.gpu_latencies_ms: list = []
        self.done_at: dict = {}  # image number -> time.monotonic() its lines were written
        self.passes = 0
        self.images_done = 0
        self.batch_sizes: list = []
        self._threads: list = []
        self._socks: list = []
        self.port, self.ext_port, self.host = port, ext_port, host
        self.t_first = None
        self.t_last = None
        os.makedirs(self.result_dir, exist_ok=True)
        from .post import STREAM_SOLUTIONS_HEADER, STREAM_SPOTS_HEADER
        self.sol_f = open(os.path.join(self.result_dir, "solutions.txt"), "w")
        self.spt_f = open(os.path.join(self.result_dir, "spots.txt"), "w")
        self.spt_f.write(STREAM_SPOTS_HEADER)
        self.sol_f.write(STREAM_SOLUTIONS_HEADER)
        self.sol_f.flush()
        self.spt_f.flush()

    # ---- network --------------------------------------------------------------
    def _listen(self, port):
        s = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
        s.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
        s.bind((self.host, port))
        s.listen(MAX_CONNECTIONS)
        s.settimeout(0.5)
        self._socks.append(s)
        return s

    def _accept_loop(self, srv, extended):
        try:
            while self.running:
                try:
                    c, _ = srv.accept()
                except socket.timeout:
                    continue
                except OSError:
                    break
                t = threading.Thread(target=self._client, args=(c, extended), daemon=True)
                t.start()
                self._threads.append(t)
        finally:
            srv.close()

    def _client(self, c, extended):
        # bounded receives so shutdown is seen: the kernel's SO_RCVTIMEO on a
        # blocking socket (as the reference, 5 s there, 0.5 s here) -- a Python
        # socket timeout would add a poll() before every receive
        c.settimeout(None)
        c.setsockopt(socket.SOL_SOCKET, socket.SO_RCVTIMEO, struct.pack("ll", 0, 500000))
        try:  # a larger receive buffer: fewer receives per 16 MiB frame
            c.setsockopt(socket.SOL_SOCKET, socket.SO_RCVBUF, RCVBUF)
        except OSError:
            pass
        run = lambda: self.running  # noqa: E731
        W, H = int(self.primary.nr_px_x), int(self.primary.nr_px_y)
        try:
            while self.running:
                if extended:
                    hb = bytearray(EXT_HEADER.size)
                    if not _recv_exact(c, hb, run):
                        break
                    magic, num, w, h, dt, _ = EXT_HEADER.unpack(hb)
                    if magic != EXT_MAGIC or dt not in (0, 1, 2):
                        self.log("bad extended header; closing connection")
                        break
                    key = (w, h)
                    dtype = (np.float32, np.uint8, np.uint16)[dt]
                else:
                    hb = bytearray(2)
                    if not _recv_exact(c, hb, run):
                        break
                    num = int.from_bytes(hb, sys.byteorder)  # host-endian, as memcpy
                    key, dtype = (W, H), np.float32
                    w, h = W, H
                payload = self.frames.get(w * h, dtype)
                if not _recv_exact(c, payload.view(np.uint8), run):
                    self.frames.put(payload)
                    break
                t = time.perf_counter()
                if key not in self.geoms:
                    self.log(f"image {num}: no DB for a {w}x{h} detector; dropped")
                    self.frames.put(payload)
                    continue
                # blocks while MAX_QUEUE images wait (back-pressure, as queue_push)
                queued = False
                while self.running:
                    try:
                        self.queue.put(Request(num, key, payload, t, raw=dtype == np.uint16),
                                       timeout=0.5)
                        queued = True
                        break
                    except queue.Full:
                        continue
                if not queued:
                    self.frames.put(payload)
        finally:
            c.close()

    # ---- GPU loop -------------------------------------------------------------
    def _gpu_loop(self):
        while True:
            idle = not any(g.loaded or g.inflight for g in self.geoms.values())
            if not self.running and idle and self.queue.empty() and not self._backlog:
                break
            # admit arrivals into free slots (uploads overlap the running pass)
            admitted = self._admit(block=idle)
            # start a pass over the uploaded images of every geometry; with one
            # pass already on the device the new one queues behind it
            for g in self.geoms.values():
                if g.loaded and len(g.inflight) < 2:
                    batch, g.loaded = g.loaded, []
                    p = g.params
                    g.engine.match([s for s, _ in batch], p.min_nr_spots, p.min_intensity)
                    g.inflight.append(batch)
                    self.passes += 1
                    self.batch_sizes.append(len(batch))
            if not admitted:
                self._admit(block=False)
            # collect the oldest pass of each geometry (waits for it; a pass
            # queued behind it keeps the device busy meanwhile), free its slots
            for g in self.geoms.values():
                if not g.inflight:
                    continue
                batch = g.inflight.popleft()
                res = g.engine.results_batch([s for s, _ in batch])
                t = time.perf_counter()
                for s, r in batch:
                    surv, npass = res[s]
                    self.done_q.put(Done(r, surv, npass, t))
                    g.free.append(s)
        self.done_q.put(None)

    def _admit(self, block):
        """Upload waiting images into free slots; images whose geometry has no
        free slot stay in the backlog (in arrival order) until a pass ends."""
        n = 0
        while len(self._backlog) < 4 * self.max_batch:
            try:
                r = self.queue.get(timeout=0.05) if (block and not self._backlog and n == 0) \
                    else self.queue.get_nowait()
            except queue.Empty:
                break
            self._backlog.append(r)
            block = False
        keep = collections.deque()
        admitted = {}
        while self._backlog:
            r = self._backlog.popleft()
            g = self.geoms[r.key]
            if not g.free:
                keep.append(r)
                continue
            admitted.setdefault(r.key, []).append((g.free.pop(), r))
            n += 1
        # one batched upload per geometry and pixel type; raw frames are
        # preprocessed on the device straight into their slots
        for key, items in admitted.items():
            g = self.geoms[key]
            raw = [(s, r) for s, r in items if r.raw]
            items = [(s, r) for s, r in items if not r.raw]
            if raw:
                items += self._preprocess_raw(g, raw)
            by_type = collections.defaultdict(list)
            for s, r in items:
                if not r.raw:
                    by_type[r.pixels.dtype].append((s, r))
            for its in by_type.values():
                g.engine.load_images([s for s, _ in its], [r.pixels for _, r in its])
            g.loaded.extend(items)
        self._backlog = keep
        return n

    def _preprocess_raw(self, g, raw):
        """Raw frames into their slots; returns the loaded (slot, request)
        pairs, each request now holding its blurred frame.  Frames without
        spots are finished at once without lines and free their slots."""
        from . import preprocess as PP
        if g.pool is None:
            cfg = dict(g.pre_cfg) if g.pre_cfg else PP.config_from_params_text("")
            cfg["nr_px_x"], cfg["nr_px_y"] = int(g.params.nr_px_x), int(g.params.nr_px_y)
            bg = PP.load_background(cfg.get("background_file", ""), cfg["nr_px_x"],
                                    cfg["nr_px_y"])
            if np.count_nonzero(bg) == 0:  # the image server: median of the first frame
                bg = PP.compute_background(raw[0][1].pixels.reshape(cfg["nr_px_y"],
                                                                    cfg["nr_px_x"]),
                                           cfg["filter_radius"], cfg["median_passes"],
                                           device=self.device)
            g.pool = PP.PreprocessPool(cfg, bg, device=self.device)
        shape = (int(g.params.nr_px_y), int(g.params.nr_px_x))
        res = g.pool.to_slots(g.engine, [s for s, _ in raw],
                              [r.pixels.reshape(shape) for _, r in raw], np.float32,
                              host_copy=True)
        loaded = []
        t = time.perf_counter()
        for (s, r), out in zip(raw, res):
            if out is None:
                g.free.append(s)
                self.done_q.put(Done(r, np.zeros(0, _SURV_DTYPE), 0, t))
                continue
            self.frames.put(r.pixels)  # the raw frame; the blurred one replaces it
            r.pixels = out[1].ravel()
            loaded.append((s, r))
        return loaded

    # ---- post-stage + output ----------------------------------------------------
    def _writer(self):
        """One of the writer threads: post-stage of finished images (the C
        post-stage releases the GIL), then an atomic append of the image's
        lines to both files."""
        from .post import collected_matches, post_process
        while True:
            d = self.done_q.get()
            if d is None:
                break
            g = self.geoms[d.req.key]
            p = g.params
            img = d.req.pixels.astype(np.float32, copy=False)
            sol = spt = ""
            if d.survivors.shape[0] or d.n_pass:
                ids, sc = collected_matches(d.survivors, d.n_pass)
                sol, spt, nu = post_process(p, g.engine.geometry, self.orients, ids, sc, img,
                                            self.hkls, min_nr_spots=p.min_good_spots,
                                            image_num=d.req.image_num,
                                            num_threads=self.post_threads,
                                            merge_device=self.device)
            with self._out_lock:
                if sol or spt:
                    self.sol_f.write(sol)
                    self.spt_f.write(spt)
                    self.sol_f.flush()
                    self.spt_f.flush()
                self.frames.put(d.req.pixels)
                t = time.perf_counter()
                self.done_at[d.req.image_num] = time.monotonic()
                self.latencies_ms.append((t - d.req.t_arrival) * 1e3)
                self.gpu_latencies_ms.append((d.t_gpu_done - d.req.t_arrival) * 1e3)
                self.images_done += 1
                self.t_first = self.t_first or d.req.t_arrival
                self.t_last = t

    # ---- lifecycle --------------------------------------------------------------
    def start(self, listen=True):
        # receive buffers of the primary detector's float32 wire frames made
        # before the first message: as many as can wait in the queue and in
        # two passes' slots (the page-locked budget caps it)
        W, H = int(self.primary.nr_px_x), int(self.primary.nr_px_y)
        self.frames.prefill(W * H, np.float32, self.queue.maxsize + 2 * self.max_batch)
        self.running = True
        if listen:
            self._accept_threads = [
                threading.Thread(target=self._accept_loop, args=(self._listen(self.port), False),
                                 daemon=True)]
            if len(self.geoms) > 1 or self.ext_port:
                self._accept_threads.append(threading.Thread(
                    target=self._accept_loop, args=(self._listen(self.ext_port), True),
                    daemon=True))
            for t in self._accept_threads:
                t.start()
        self._gpu = threading.Thread(target=self._gpu_loop, daemon=True)
        self._wr = [threading.Thread(target=self._writer, daemon=True)
                    for _ in range(self.n_writers)]
        self._gpu.start()
        for t in self._wr:
            t.start()
        return self

    def submit(self, image_num, pixels, key=None):
        """In-process submission (same path as a received message)."""
        key = key or (int(self.primary.nr_px_x), int(self.primary.nr_px_y))
        self.queue.put(Request(int(image_num), key, np.asarray(pixels), time.perf_counter()))

    def stop(self, drain_timeout=600.0, close_engines=True):
        """Stop accepting, finish every received image, close the files."""
        self.running = False
        for t in getattr(self, "_accept_threads", []):
            t.join(timeout=5.0)  # each closes its listening socket
        for t in self._threads:
            t.join(timeout=5.0)
        self._gpu.join(timeout=drain_timeout)
        for _ in range(len(self._wr) - 1):  # the GPU loop queued one end marker
            self.done_q.put(None)
        for t in self._wr:
            t.join(timeout=drain_timeout)
        self.sol_f.close()
        self.spt_f.close()
        for g in self.geoms.values():
            if g.pool is not None:
                g.pool.close()
        if self._gpu.is_alive() or any(t.is_alive() for t in self._wr):
            self.log("stop: images still in flight; receive buffers kept")
        elif self._own_frames:
            self.frames.close()
        if close_engines:
            for g in self.geoms.values():
                g.engine.close()
        return self.stats()

    def stats(self):
        lat = np.asarray(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        glat = np.asarray(self.gpu_latencies_ms) if self.gpu_latencies_ms else np.zeros(1)
        span = (self.t_last - self.t_first) if self.t_first and self.t_last else 0.0
        return {"images": self.images_done, "passes": self.passes,
                "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "gpu_p50_ms": float(np.percentile(glat, 50)),
                "gpu_p99_ms": float(np.percentile(glat, 99)),
                "images_per_s": self.images_done / span if span > 0 else 0.0,
                "max_batch": self.max_batch}


def main(argv=None) -> int:
    argv = sys.argv if argv is None else argv
    if len(argv) < 5:
        print("LaueMatchingGPUStream -- persistent GPU daemon (B200)\n\n"
              f"Usage: {argv[0] if argv else 'LaueMatchingGPUStream'} parameterFile "
              "orientationFile hklFile nCPUs\n\n"
              f"Listens on TCP port {PORT} for binary images.\n"
              "Wire protocol: uint16_t image_num + float[NrPxX*NrPxY]")
        return 0
    ap = argparse.ArgumentParser(add_help=False)
    ap.add_argument("--extra-params", action="append", default=[])
    ap.add_argument("--max-batch", type=int, default=64)
    ap.add_argument("--device", type=int, default=int(os.environ.get("LMB_DEVICE", "0")))
    ap.add_argument("--port", type=int, default=PORT)
    ap.add_argument("--ext-port", type=int, default=EXT_PORT)
    opts, rest = ap.parse_known_args(argv[5:])
    from . import formats
    from .params import ParamsError, read_params
    param_fn, orient_fn, hkl_fn, ncpu_s = argv[1:5]
    print("Reading parameter file", flush=True)
    try:
        plist = [read_params(param_fn, binary="stream")]
        plist += [read_params(x, binary="stream") for x in opts.extra_params]
    except (OSError, ParamsError) as exc:
        print(f"Could not open parameter file {param_fn}: {exc}")
        return 1
    print("Parameters read", flush=True)
    orients = formats.read_orientations(orient_fn)
    hkls = formats.read_hkls(hkl_fn)
    print(f"{orients.shape[0]} orientations, {len(hkls)} hkls", flush=True)
    from .preprocess import config_from_params_text
    pcfgs = []
    for fn in [param_fn] + opts.extra_params:
        with open(fn) as f:
            pcfgs.append(config_from_params_text(f.read()))
    srv = StreamServer(plist, orients, hkls, ncpus=int(ncpu_s), max_batch=opts.max_batch,
                       device=opts.device, port=opts.port, ext_port=opts.ext_port,
                       log=lambda *a: print(*a, flush=True), preprocess_cfgs=pcfgs)
    return serve_until_signalled(srv)


def serve_until_signalled(srv) -> int:
    """Run the daemon until SIGINT or SIGTERM (LaueMatchingGPUStream.cu:542-551):
    the first signal stops accepting and drains -- every image already
    received is matched and written -- then returns 0 (:1288); a second
    signal exits at once with status 1."""
    stop = threading.Event()

    def on_signal(signum, frame):
        if stop.is_set():
            os._exit(1)  # second signal: hard exit, as the reference
        stop.set()

    signal.signal(signal.SIGINT, on_signal)
    signal.signal(signal.SIGTERM, on_signal)
    srv.start()
    print(f"Listening on port {srv.port} (extended header on {srv.ext_port}); "
          f"up to {srv.max_batch} images per DB pass", flush=True)
    while not stop.wait(0.5):
        pass
    st = srv.stop()
    print(f"Processed {st['images']} images in {st['passes']} DB passes "
          f"(mean batch {st['mean_batch']:.1f}); latency p50 {st['p50_ms']:.1f} ms, "
          f"p99 {st['p99_ms']:.1f} ms", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
