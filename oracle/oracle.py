"""TEST INFRASTRUCTURE ONLY: Python access to the oracle.

* ``liblmoracle.so`` -- our FP64 C restatement of the reference CPU algorithm
  (lm_oracle.c), loaded with ctypes;
* ``_ref/LaueMatchingCPU`` -- the reference's own CPU executable compiled from
  its sources by oracle/Makefile (NLopt replaced by an evaluate-once
  stand-in), driven through its 5-argument command line;
* ``_ref/LaueMatchingGPU`` -- the reference's single-image GPU executable
  compiled from its sources for sm_100a, the plain one-pass-per-image GPU
  baseline (same command line).

Only tests/, __graft_entry__.smoke() and bench.py's baseline legs (the CPU
baseline and the reference arms) use this module; the product never imports
it.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblmoracle.so")
REF_BIN = os.path.join(HERE, "_ref", "LaueMatchingCPU")
REF_GPU_BIN = os.path.join(HERE, "_ref", "LaueMatchingGPU")
REF_STREAM_BIN = os.path.join(HERE, "_ref", "LaueMatchingGPUStream")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, os.path.join(HERE, "liblmoracle.so")],
                           check=True, capture_output=True)
        L = C.CDLL(LIB_PATH)
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        lp = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        up = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
        bp = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        L.orc_detector_rot_t.argtypes = [dp, dp]
        L.orc_recip.argtypes = [dp, C.c_int, dp]
        L.orc_forward.argtypes = [dp, C.c_int64, ip, C.c_int, dp, dp, dp, C.c_double,
                                  C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                  C.c_int, up, C.c_int]
        L.orc_quantize.argtypes = [dp, C.c_int64, bp]
        L.orc_quantize.restype = C.c_double
        L.orc_compare.argtypes = [up, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                                  lp, ip, ip, dp, dp, C.c_int64,
                                  C.POINTER(C.c_int64), C.c_int]
        L.orc_compare.restype = C.c_int64
        _lib = L
    return _lib


def geometry(p):
    """(rot_t[9], recip[9]) from a LaueParams, exactly as the reference."""
    rt = np.zeros(9)
    rc = np.zeros(9)
    lib().orc_detector_rot_t(np.asarray(p.r_array, np.float64), rt)
    lib().orc_recip(np.asarray(p.lattice, np.float64), int(p.space_group), rc)
    return rt, rc


def forward(p, orients, hkls, nthreads=os.cpu_count()):
    """Forward-cache records uint16[n, 1+2S] for the given orientations."""
    om = np.ascontiguousarray(orients, np.float64).reshape(-1, 9)
    hk = np.ascontiguousarray(hkls, np.int32).reshape(-1, 3)
    S = int(p.max_nr_spots)
    out = np.zeros((om.shape[0], 1 + 2 * S), np.uint16)
    rt, rc = geometry(p)
    lib().orc_forward(om, om.shape[0], hk, hk.shape[0], rc, rt,
                      np.asarray(p.p_array, np.float64), p.px_x, p.px_y,
                      p.nr_px_x, p.nr_px_y, p.elo, p.ehi, S, out, int(nthreads))
    return out


def quantize(img):
    im = np.ascontiguousarray(img, np.float64).ravel()
    out = np.zeros(im.size, np.uint8)
    scale = lib().orc_quantize(im, im.size, out)
    return out, scale


@dataclass
class Survivors:
    ids: np.ndarray
    n_spots: np.ndarray
    sum_u8: np.ndarray
    tot_int: np.ndarray
    score: np.ndarray
    n_pass: int


def compare(records, S, img_f64, nr_px_x, nr_px_y, min_nr_spots, min_intensity,
            mode=0, nthreads=os.cpu_count(), cap=1 << 22):
    """Survivors in ascending ID.  mode 0 = uint8 path (DoFwd 0), 1 = float64
    image path (DoFwd 1)."""
    rec = np.ascontiguousarray(records, np.uint16).reshape(-1, 1 + 2 * S)
    im = np.ascontiguousarray(img_f64, np.float64).ravel()
    u8, scale = quantize(im)
    while True:
        ids = np.zeros(cap, np.int64)
        ns = np.zeros(cap, np.int32)
        su = np.zeros(cap, np.int32)
        ti = np.zeros(cap, np.float64)
        sc = np.zeros(cap, np.float64)
        npass = C.c_int64(0)
        r = lib().orc_compare(rec, rec.shape[0], S, mode, u8.ctypes.data,
                              im.ctypes.data, scale, nr_px_x, nr_px_y,
                              min_nr_spots, min_intensity, ids, ns, su, ti, sc,
                              cap, C.byref(npass), int(nthreads))
        if r >= 0:
            return Survivors(ids[:r], ns[:r], su[:r], ti[:r], sc[:r], npass.value)
        cap = -r


@dataclass
class RefRun:
    returncode: int
    stdout: str
    stderr: str
    solutions: str | None
    spots: str | None
    initial_solutions: int | None
    unique: int | None
    compare_seconds: float | None
    wall_seconds: float


def have_ref() -> bool:
    return os.path.exists(REF_BIN)


def run_reference(params_path, orient_path, hkl_path, image_path, ncpus=1,
                  timeout=3600) -> RefRun:
    """Run the reference LaueMatchingCPU on files; parse its report lines."""
    t0 = time.perf_counter()
    pr = subprocess.run([REF_BIN, params_path, orient_path, hkl_path, image_path,
                         str(ncpus)], capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    sol = spt = None
    if os.path.exists(image_path + ".solutions.txt"):
        with open(image_path + ".solutions.txt") as f:
            sol = f.read()
    if os.path.exists(image_path + ".spots.txt"):
        with open(image_path + ".spots.txt") as f:
            spt = f.read()
    m = re.search(r"Initial solutions: (\d+) Unique Orientations: (\d+)", pr.stdout)
    mc = re.search(r"Finished comparing, time elapsed after comparing with forward "
                   r"simulation: ([0-9.eE+-]+) seconds", pr.stdout)
    return RefRun(pr.returncode, pr.stdout, pr.stderr, sol, spt,
                  int(m.group(1)) if m else None, int(m.group(2)) if m else None,
                  float(mc.group(1)) if mc else None, wall)


@dataclass
class RefGpuRun:
    returncode: int
    stdout: str
    stderr: str
    n_matches: int | None
    chunks: list            # [(h2d_seconds, kernel_seconds)] per DB chunk
    read_seconds: float | None
    match_seconds: float | None
    compare_seconds: float | None
    wall_seconds: float


def have_ref_gpu() -> bool:
    return os.path.exists(REF_GPU_BIN)


def run_reference_gpu(params_path, orient_path, hkl_path, image_path, ncpus=1,
                      timeout=900, env=None) -> RefGpuRun:
    """Run the reference LaueMatchingGPU on files and parse its timing report:
    per-chunk H2D and kernel seconds (LaueMatchingGPU.cu:747), the match
    stage (:777), the forward-file read (:658) and NrMatches (:791)."""
    t0 = time.perf_counter()
    pr = subprocess.run([REF_GPU_BIN, params_path, orient_path, hkl_path, image_path,
                         str(ncpus)], capture_output=True, text=True, timeout=timeout,
                        env=env)
    wall = time.perf_counter() - t0
    num = r"([0-9.eE+-]+)"
    chunks = [(float(a), float(b)) for a, b in
              re.findall(r"chunk \d+/\d+: H2D=" + num + r"s\s+kernel=" + num + "s", pr.stdout)]

    def grab(pat, cast=float):
        m = re.search(pat, pr.stdout)
        return cast(m.group(1)) if m else None
    return RefGpuRun(pr.returncode, pr.stdout, pr.stderr, grab(r"NrMatches: (\d+)", int), chunks,
                     grab(r"Time elapsed to read the forward simulation: " + num),
                     grab(r"Time elapsed to match on the GPU: " + num),
                     grab(r"Finished comparing, time elapsed after comparing with forward "
                          r"simulation: " + num), wall)


def have_ref_stream() -> bool:
    return os.path.exists(REF_STREAM_BIN)


class RefStream:
    """The reference's LaueMatchingGPUStream daemon (sm_100a build) run through
    its own command line (LaueMatchingGPUStream.cu:536-540) in ``cwd``.  A
    reader thread time-stamps (time.monotonic) each image's last report line
    -- "[Image N] No matches, skipping fitting." or "[Image N] Total: ..."
    (finalize_stream, :452-533) -- so a client can measure per-image
    latency and throughput from outside.  stdout is line-buffered through
    stdbuf so a line appears when the daemon prints it."""

    READY = "LaueMatchingGPUStream ready"

    def __init__(self, params_path, orient_path, hkl_path, ncpus, cwd, env=None):
        import threading
        cmd = [REF_STREAM_BIN, params_path, orient_path, hkl_path, str(ncpus)]
        if shutil.which("stdbuf"):
            cmd = ["stdbuf", "-oL", "-eL"] + cmd
        self.proc = subprocess.Popen(cmd, cwd=cwd, stdout=subprocess.PIPE,
                                     stderr=subprocess.STDOUT, text=True, env=env)
        self.done = {}          # image number -> monotonic time of its last line
        self.lines = []
        self.ready = threading.Event()
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        pat = re.compile(r"^\[Image (\d+)\] (No matches|Total:)")
        for line in self.proc.stdout:
            t = time.monotonic()
            if len(self.lines) < 20000:
                self.lines.append(line)
            if self.READY in line:
                self.ready.set()
            m = pat.match(line)
            if m:
                self.done[int(m.group(1))] = t
        self.ready.set()

    def wait_ready(self, timeout=900.0) -> bool:
        self.ready.wait(timeout)
        return self.proc.poll() is None and any(self.READY in ln for ln in self.lines)

    def stop(self, timeout=120.0) -> int:
        """SIGINT: the daemon drains its streams and exits (:542-551, :1288)."""
        import signal
        if self.proc.poll() is None:
            self.proc.send_signal(signal.SIGINT)
        try:
            self.proc.wait(timeout)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self._t.join(5)
        return self.proc.returncode


def reference_case(workdir, params_text, orients, hkls, image, ncpus=1):
    """Write a case's files under ``workdir`` and run the reference."""
    from lauematching_b200 import formats
    os.makedirs(workdir, exist_ok=True)
    pp = os.path.join(workdir, "params.txt")
    op = os.path.join(workdir, "orients.bin")
    hp = os.path.join(workdir, "hkls.csv")
    ip = os.path.join(workdir, "image.bin")
    with open(pp, "w") as f:
        f.write(params_text)
    formats.write_orientations(op, orients)
    formats.write_hkls(hp, hkls)
    formats.write_image_bin(ip, image)
    return run_reference(pp, op, hp, ip, ncpus=ncpus)


def tempdir():
    return tempfile.mkdtemp(prefix="lmb_oracle_")
