"""Fault paths of the streaming daemon, on the host (no GPU): the engine is a
stand-in (tests/stream_fakes.py), the sockets are real.

The reference daemon hardens the same paths: a receive timeout that retries
while running (LaueMatchingGPUStream.cu:302-358), a bounded queue that blocks
the receiving thread when full (:199-292), connections that end in the middle
of a message, and SIGINT/SIGTERM that stop accepting, drain what was
received and exit 0 (:542-551, :1288).
"""
import os
import signal
import socket
import struct
import subprocess
import sys
import threading
import time

import numpy as np
import pytest

from conftest import ROOT
from stream_fakes import FakeEngine, make_server

W = H = 64


def _free_ports(n):
    socks = [socket.socket() for _ in range(n)]
    for s in socks:
        s.bind(("127.0.0.1", 0))
    ports = [s.getsockname()[1] for s in socks]
    for s in socks:
        s.close()
    return ports


def _frame(num, dtype=np.float32):
    f = np.zeros(W * H, dtype)
    f[0] = num
    return f


def _plain(num):
    return num.to_bytes(2, sys.byteorder) + _frame(num).tobytes()


def _ext(num, dt=0, magic=b"LMB2", w=W, h=H):
    body = _frame(num, (np.float32, np.uint8, np.uint16)[dt] if dt in (0, 1, 2) else np.uint8)
    return struct.pack("<4sHHHBB", magic, num, w, h, dt, 0) + body.tobytes()


def _send(port, data, close=True, pause=None):
    s = socket.create_connection(("127.0.0.1", port))
    if pause is None:
        s.sendall(data)
    else:
        cut, secs = pause
        s.sendall(data[:cut])
        time.sleep(secs)
        s.sendall(data[cut:])
    if close:
        s.close()
    return s


def _wait(cond, secs=20.0):
    t0 = time.time()
    while not cond():
        if time.time() - t0 > secs:
            return False
        time.sleep(0.02)
    return True


def _received(eng):
    with eng.lock:
        return [int(f[0]) for f in eng.frames]


@pytest.fixture
def server(tmp_path):
    port, ext = _free_ports(2)
    eng = FakeEngine()
    srv = make_server(tmp_path, port, ext, eng).start()
    yield srv, eng, port, ext
    srv.stop()


def test_short_header_and_disconnect_mid_payload_drop_only_that_message(server):
    srv, eng, port, ext = server
    _send(port, b"\x01")                            # 1 of the 2 header bytes
    _send(port, _plain(7)[: 2 + 1000])              # header + part of the payload
    _send(ext, _ext(8)[:5])                         # part of an extended header
    _send(ext, _ext(9)[: 12 + 100])                 # extended header + part of the payload
    _send(port, _plain(3) + _plain(4))              # complete messages still served
    _send(ext, _ext(5))
    assert _wait(lambda: srv.images_done == 3)
    time.sleep(0.3)
    assert sorted(_received(eng)) == [3, 4, 5] and srv.images_done == 3


def test_bad_extended_header_closes_that_connection_only(server):
    srv, eng, port, ext = server
    _send(ext, _ext(11, magic=b"XXXX") + _ext(12))  # bad magic: connection dropped
    _send(ext, _ext(13, dt=7))                      # unknown pixel type: dropped
    _send(ext, _ext(14, w=32, h=32))                # no DB for this detector: message skipped
    _send(ext, _ext(15) + _ext(16, dt=1))           # float32 then uint8 frames
    assert _wait(lambda: srv.images_done == 2)
    time.sleep(0.3)
    assert sorted(_received(eng)) == [15, 16]


def test_receive_timeout_retries_while_running(server):
    """A sender that pauses longer than the receive timeout (0.5 s here, 5 s
    in the reference) in the middle of a message is waited for."""
    srv, eng, port, ext = server
    _send(port, _plain(21), pause=(2 + 4000, 1.3))
    _send(port, _plain(22), pause=(1, 1.3))
    assert _wait(lambda: srv.images_done == 2)
    assert sorted(_received(eng)) == [21, 22]


def test_full_queue_blocks_the_receiver_and_loses_nothing(tmp_path):
    """Queue of 2 and one slot, passes held on the device: the receiving
    thread blocks (back-pressure) instead of dropping frames; when the
    passes finish every frame is matched, in the order sent."""
    port, ext = _free_ports(2)
    hold = threading.Event()
    eng = FakeEngine(hold=hold)
    srv = make_server(tmp_path, port, ext, eng, max_batch=1, max_queue=2).start()
    try:
        s = socket.create_connection(("127.0.0.1", port))
        sender = threading.Thread(target=lambda: s.sendall(b"".join(_plain(i) for i in range(1, 41))))
        sender.start()
        time.sleep(1.5)
        assert srv.queue.qsize() <= 2
        assert len(_received(eng)) <= 4 and srv.images_done == 0
        hold.set()
        sender.join(30)
        s.close()
        assert _wait(lambda: srv.images_done == 40)
        assert _received(eng) == list(range(1, 41))
    finally:
        hold.set()
        srv.stop()


_DAEMON = r"""
import sys, threading
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
from stream_fakes import FakeEngine, make_server
from lauematching_b200 import stream
eng = FakeEngine(pass_seconds={secs})
srv = make_server({tmp!r}, {port}, {ext}, eng, max_batch=2)
sys.exit(stream.serve_until_signalled(srv))
"""


def _daemon(tmp_path, secs):
    port, ext = _free_ports(2)
    code = _DAEMON.format(root=ROOT, tests=os.path.join(ROOT, "tests"), secs=secs,
                          tmp=str(tmp_path), port=port, ext=ext)
    proc = subprocess.Popen([sys.executable, "-c", code], stdout=subprocess.PIPE,
                            stderr=subprocess.STDOUT, text=True)
    line = proc.stdout.readline()
    assert "Listening on port" in line, line
    return proc, port


def test_sigterm_during_a_pass_drains_received_frames_and_exits_0(tmp_path):
    proc, port = _daemon(tmp_path, secs=0.8)
    try:
        _send(port, b"".join(_plain(i) for i in range(1, 6)))
        time.sleep(0.5)  # the first pass is on the "device"
        proc.send_signal(signal.SIGTERM)
        out, _ = proc.communicate(timeout=60)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 0, out
    assert "Processed 5 images" in out, out
    # the listening socket is closed: new connections are refused
    with pytest.raises(OSError):
        socket.create_connection(("127.0.0.1", port), timeout=2).close()


def test_second_signal_exits_at_once_with_status_1(tmp_path):
    proc, port = _daemon(tmp_path, secs=5.0)
    try:
        _send(port, b"".join(_plain(i) for i in range(1, 6)))
        time.sleep(0.5)
        proc.send_signal(signal.SIGINT)
        time.sleep(0.3)
        proc.send_signal(signal.SIGINT)
        out, _ = proc.communicate(timeout=30)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 1, out
    assert "Processed" not in out
