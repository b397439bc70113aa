"""The serving daemon end to end on the GPU.

* the reference's TCP protocol (2-byte host-endian image number + float32
  frame) from two concurrent connections;
* each image's lines in results/solutions.txt and spots.txt equal the
  expectation computed from the oracle's survivors for that image alone, and
  equal the lines a one-image-per-pass daemon writes (same result alone and
  in the mix);
* a second detector geometry (1024x1024) on the extended-header port, with
  its own resident DB, mixed with 2048x2048 frames.
"""
import os
import socket
import struct
import sys
import threading
import time

import numpy as np
import pytest

import oracle as O
from conftest import golden_case
from lauematching_b200 import params as P, post, synth
from lauematching_b200.engine import geometry_from_params

pytestmark = pytest.mark.gpu


def _params_text(c):
    """The case's params without its (generation-time) ForwardFile path."""
    return "".join(ln for ln in c.params_text.splitlines(keepends=True)
                   if not ln.startswith("ForwardFile")) + "MinGoodSpots 4\n"


def _ports():
    base = 41000 + (os.getpid() % 500) * 4
    return base, base + 1


def _frames(c, n, seed):
    rng = np.random.default_rng(seed)
    p = c.params
    out = []
    for _ in range(n):
        g = synth.pick_grains(c.records, int(rng.integers(1, 5)), 8, rng)
        out.append(synth.render_image(c.records[g], p.nr_px_x, p.nr_px_y, rng).astype(np.float32))
    return out


def _send(port, msgs, extended=False):
    s = socket.create_connection(("127.0.0.1", port))
    for m in msgs:
        if extended:
            num, w, h, arr = m
            dt = 0 if arr.dtype == np.float32 else 1
            s.sendall(struct.pack("<4sHHHBB", b"LMB2", num, w, h, dt, 0))
            s.sendall(arr.tobytes())
        else:
            num, arr = m
            s.sendall(struct.pack("=H", num))
            s.sendall(arr.astype(np.float32).tobytes())
    s.close()


def _wait_done(srv, n, timeout=120):
    t0 = time.time()
    while srv.images_done < n and time.time() - t0 < timeout:
        time.sleep(0.05)
    assert srv.images_done == n


def _lines_by_image(path):
    out = {}
    for ln in open(path).read().splitlines()[1:]:
        out.setdefault(int(ln.split("\t")[0]), []).append(ln)
    return out


def _expected(c_params, orients, hkls, img_f32, num):
    p = c_params
    rec = _expected.records[(p.nr_px_x, p.nr_px_y)]
    s = O.compare(rec, p.max_nr_spots, img_f32.astype(np.float64), p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity)
    if len(s.ids) == 0 and s.n_pass == 0:
        return [], []
    surv = np.zeros(len(s.ids), [("id", "<u8"), ("score", "<f8")])
    surv["id"], surv["score"] = s.ids, s.score
    ids, sc = post.collected_matches(surv, s.n_pass)
    sol, spt, _ = post.post_process(p, geometry_from_params(p), orients, ids, sc, img_f32, hkls,
                                    min_nr_spots=p.min_good_spots, image_num=num)
    return sol.splitlines(), spt.splitlines()


def _server(plist, orients, hkls, tmp, max_batch, ports, preprocess_cfgs=None):
    from lauematching_b200.stream import StreamServer
    return StreamServer(plist, orients, hkls, ncpus=4, max_batch=max_batch,
                        result_dir=str(tmp), port=ports[0], ext_port=ports[1],
                        host="127.0.0.1", log=lambda *a: None,
                        preprocess_cfgs=preprocess_cfgs).start()


def test_stream_mix_equals_alone_equals_oracle(tmp_path):
    c = golden_case("tilted_fcc")
    p = P.parse_params_text(_params_text(c), binary="stream")
    frames = _frames(c, 8, seed=1)
    ports = _ports()
    srv = _server([p], c.orients, c.hkls, tmp_path / "mix", 64, ports)
    try:
        time.sleep(0.3)
        t1 = threading.Thread(target=_send, args=(ports[0], [(i + 1, frames[i]) for i in range(0, 8, 2)]))
        t2 = threading.Thread(target=_send, args=(ports[0], [(i + 1, frames[i]) for i in range(1, 8, 2)]))
        t1.start(), t2.start(), t1.join(), t2.join()
        _wait_done(srv, 8)
    finally:
        st = srv.stop()
    assert st["images"] == 8
    mix_sol = _lines_by_image(tmp_path / "mix" / "solutions.txt")
    mix_spt = _lines_by_image(tmp_path / "mix" / "spots.txt")
    # one image per pass, sequentially
    srv1 = _server([p], c.orients, c.hkls, tmp_path / "alone", 1, ports)
    try:
        time.sleep(0.3)
        for i in range(8):
            _send(ports[0], [(i + 1, frames[i])])
            _wait_done(srv1, i + 1)
    finally:
        srv1.stop()
    one_sol = _lines_by_image(tmp_path / "alone" / "solutions.txt")
    one_spt = _lines_by_image(tmp_path / "alone" / "spots.txt")
    _expected.records = {(p.nr_px_x, p.nr_px_y): c.records}
    for i in range(8):
        es, ep = _expected(p, c.orients, c.hkls, frames[i], i + 1)
        assert mix_sol.get(i + 1, []) == one_sol.get(i + 1, []) == es
        assert mix_spt.get(i + 1, []) == one_spt.get(i + 1, []) == ep
    assert sum(len(v) for v in mix_sol.values()) > 0


def test_stream_mixed_detector_sizes(tmp_path):
    c = golden_case("tilted_fcc")
    p2 = P.parse_params_text(_params_text(c), binary="stream")
    txt1 = _params_text(c).replace("NrPxX 2048", "NrPxX 1024").replace("NrPxY 2048", "NrPxY 1024")
    txt1 = txt1.replace("PxX 0.0002", "PxX 0.0004").replace("PxY 0.0002", "PxY 0.0004")
    p1 = P.parse_params_text(txt1, binary="stream")
    assert (p1.nr_px_x, p1.px_x) == (1024, 0.0004)
    rec1 = O.forward(p1, c.orients, c.hkls)
    rng = np.random.default_rng(3)
    f2 = _frames(c, 4, seed=2)
    f1 = []
    for _ in range(4):
        g = synth.pick_grains(rec1, 3, 6, rng)
        f1.append(synth.render_image(rec1[g], 1024, 1024, rng).astype(np.uint8))
    ports = _ports()
    srv = _server([p2, p1], c.orients, c.hkls, tmp_path / "mixed", 64, ports)
    try:
        time.sleep(0.3)
        msgs = []
        for i in range(4):
            msgs.append((10 + i, 2048, 2048, f2[i]))
            msgs.append((20 + i, 1024, 1024, f1[i]))
        _send(ports[1], msgs, extended=True)
        _wait_done(srv, 8)
    finally:
        srv.stop()
    sol = _lines_by_image(tmp_path / "mixed" / "solutions.txt")
    _expected.records = {(2048, 2048): c.records, (1024, 1024): rec1}
    for i in range(4):
        assert sol.get(10 + i, []) == _expected(p2, c.orients, c.hkls, f2[i], 10 + i)[0]
        assert sol.get(20 + i, []) == _expected(p1, c.orients, c.hkls,
                                                f1[i].astype(np.float32), 20 + i)[0]


def test_stream_raw_frames_preprocessed_on_the_device(tmp_path):
    """Raw uint16 detector frames (extended header, dtype 2) are preprocessed
    on the device into their slots: each image's lines equal those of the
    blurred frame preprocess_image makes (as float32, what the image server
    sends), and a frame without spots is finished without lines."""
    from lauematching_b200 import preprocess as PP
    c = golden_case("tilted_fcc")
    p = P.parse_params_text(_params_text(c), binary="stream")
    ny, nx = p.nr_px_y, p.nr_px_x
    yy, xx = np.mgrid[0:ny, 0:nx]
    bg = np.rint(100.0 + 0.01 * yy + 0.02 * xx)
    bg_path = tmp_path / "background.bin"
    bg.tofile(bg_path)
    cfg = PP.config_from_params_text(_params_text(c) + f"BackgroundFile {bg_path}\nMinArea 5\n")
    assert cfg["background_file"] == str(bg_path) and cfg["min_area"] == 5
    rng = np.random.default_rng(5)
    raws = []
    for _ in range(5):
        g = synth.pick_grains(c.records, int(rng.integers(1, 5)), 8, rng)
        f = synth.raw_frame(ny, nx, rng, spot_records=c.records[g], sigma=1.2, amp_lo=300.0,
                            amp_hi=4000.0)
        raws.append(np.clip(f, 0, 65535).astype(np.uint16))
    raws.append(bg.astype(np.uint16))  # nothing above the background: no spots
    ports = _ports()
    srv = _server([p], c.orients, c.hkls, tmp_path / "raw", 64, ports, preprocess_cfgs=[cfg])
    try:
        time.sleep(0.3)
        sock = socket.create_connection(("127.0.0.1", ports[1]))
        for i, f in enumerate(raws):
            sock.sendall(struct.pack("<4sHHHBB", b"LMB2", 30 + i, nx, ny, 2, 0))
            sock.sendall(f.tobytes())
        sock.close()
        _wait_done(srv, len(raws))
    finally:
        srv.stop()
    sol = _lines_by_image(tmp_path / "raw" / "solutions.txt")
    spt = _lines_by_image(tmp_path / "raw" / "spots.txt")
    _expected.records = {(nx, ny): c.records}
    n_lines = 0
    for i, f in enumerate(raws[:-1]):
        blurred = PP.preprocess_image(f, cfg, background=bg)[0].astype(np.float32)
        es, ep = _expected(p, c.orients, c.hkls, blurred, 30 + i)
        assert sol.get(30 + i, []) == es
        assert spt.get(30 + i, []) == ep
        n_lines += len(es)
    assert 30 + len(raws) - 1 not in sol
    assert n_lines > 0


@pytest.mark.parametrize("name", ["tilted_fcc", "tilted_dense", "tilted_hex"])
def test_stream_lines_are_the_reference_binarys_lines_with_the_image_number(name, tmp_path):
    """With MinGoodSpots equal to MinNrSpots (the batch executables gate the
    written grains by MinNrSpots, LaueMatchingCPU.c:809; the daemon by
    MinGoodSpots, LaueMatchingGPUStream.cu:1173), the daemon's lines for a
    golden frame sent in the reference's message are the reference binary's
    own solutions/spots lines for that frame (tests/golden, written by
    LaueMatchingCPU) with the image number as the first column
    (LaueMatchingHeaders.h:1070-1071,1132-1133,888-899)."""
    c = golden_case(name)
    txt = "".join(ln for ln in c.params_text.splitlines(keepends=True)
                  if not ln.startswith("ForwardFile"))
    p = P.parse_params_text(txt + f"MinGoodSpots {c.params.min_nr_spots}\n", binary="stream")
    ports = _ports()
    srv = _server([p], c.orients, c.hkls, tmp_path, 64, ports)
    try:
        time.sleep(0.3)
        _send(ports[0], [(7, c.image.astype(np.float32)), (9, c.image.astype(np.float32))])
        _wait_done(srv, 2)
    finally:
        srv.stop()
    sol = _lines_by_image(str(tmp_path / "solutions.txt"))
    spt = _lines_by_image(str(tmp_path / "spots.txt"))
    want_sol = c.cmp_solutions.splitlines()[1:]
    want_spt = c.cmp_spots.splitlines()[1:]
    assert want_sol and want_spt
    for num in (7, 9):
        assert sol[num] == [f"{num}\t{ln}" for ln in want_sol]
        assert spt[num] == [f"{num}\t{ln}" for ln in want_spt]
