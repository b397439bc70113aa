#!/usr/bin/env python
"""Benchmark: images/sec against a 100M-orientation DB on B200, batched vs plain.

Workload (synthetic, seeded; the reference's 100MilOrients.bin and detector
frames are not available): fcc a=3.52 A, the 1240 fcc-allowed HKLs with
|h|,|k|,|l|<=8, a 2048x2048 detector of 0.2 mm pixels 500 mm downstream
normal to the beam, 5-30 keV, MaxNrLaueSpots 30 -> 122-byte records.  The DB
(100,000,000 Shoemake-uniform orientations, seed 1) is forward-simulated on
the device by the DB-build kernel.  A step is one DB pass serving a batch of
64 uint8 frames, each with a grain count drawn from U{1..20} (grains picked
among DB orientations with >= MinNrSpots spots), Gaussian spots sigma 2 px,
amplitude U(50,255), Poisson(5) background removed by a fixed threshold.

  value   images/s of the batched pass with DB and images resident in HBM
          (CUDA events on the engine stream; the 12.2 GB DB is larger than L2)
  e2e     images/s through the public Python API from pinned host frames:
          upload + quantise 64 frames, the pass, survivor download
  plain   the same pass with one image (K=1)

`--impl reference` times the reference's own LaueMatchingCPU (compiled from
its sources into oracle/_ref/) on a bounded sample of the same workload.
`--impl reference-gpu` times the reference's plain single-image GPU executable
(LaueMatchingGPU.cu compiled for sm_100a into oracle/_ref/) on one 8-grain
frame against the full DB: one process and one DB stream per image.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "images/sec vs 100M-orient DB, batched vs plain on 1 B200; p50/p99 latency"
UNIT = "images/s"
REC_BYTES_PER_ORIENT = 122  # uint16[1 + 2*30]


def workload_params(min_intensity=200.0):
    from lauematching_b200 import params as P, synth
    txt = synth.params_text(max_nr_spots=30, min_nr_spots=5, min_intensity=min_intensity)
    return txt, P.parse_params_text(txt)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def scratch_dir(need_bytes):
    """/dev/shm when it has room (the reference memory-maps files there),
    else the default temporary directory."""
    try:
        st = os.statvfs("/dev/shm")
        if st.f_bavail * st.f_frsize > 1.5 * need_bytes:
            return "/dev/shm"
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled every ~2 ms through
    NVML while the timed region runs (nvidia-smi's 100+ ms period would miss a
    sub-second region; it is the fallback when NVML is unavailable).  Reads
    only; changes no setting."""
    REASONS = (("hw_slowdown", "HwSlowdown"), ("hw_thermal_slowdown", "HwThermalSlowdown"),
               ("sw_thermal_slowdown", "SwThermalSlowdown"), ("sw_power_cap", "SwPowerCap"))

    def __init__(self, device):
        self.device = device
        self.sm, self.reasons, self.mx, self.src = [], set(), None, None
        self._stop = threading.Event()
        self.t = None

    def _nvml_index(self):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        parts = [x.strip() for x in vis.split(",") if x.strip()]
        if parts and all(x.isdigit() for x in parts) and self.device < len(parts):
            return int(parts[self.device])
        return self.device

    def _run_nvml(self, nv, h):
        bits = {}
        for name, suffix in self.REASONS:
            v = getattr(nv, "nvmlClocksEventReason" + suffix, None)
            if v is None:
                v = getattr(nv, "nvmlClocksThrottleReason" + suffix, 0)
            bits[name] = v
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = get_reasons(h)
                for name, bit in bits.items():
                    if bit and (r & bit):
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.0001)  # the timed region can be a few ms long

    def _run_smi(self):
        proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self._nvml_index()), "--query-gpu=clocks.sm,clocks.max.sm,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "100"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self._proc = proc
        for line in proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 6:
                continue
            try:
                self.sm.append(float(f[0]))
                self.mx = float(f[1])
            except ValueError:
                continue
            for (name, _), v in zip(self.REASONS, f[2:6]):
                if v.lower().startswith("active"):
                    self.reasons.add(name)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self._nvml_index())
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.src = "nvml"
            self.t = threading.Thread(target=self._run_nvml, args=(nv, h), daemon=True)
        except Exception:
            self.src = "nvidia-smi"
            self.t = threading.Thread(target=self._run_smi, daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.sm and time.time() - t0 < 5:  # first sample before timing
            time.sleep(0.001)
        self.sm.clear()

    def stop(self):
        self._stop.set()
        if self.src == "nvidia-smi" and getattr(self, "_proc", None) is not None:
            self._proc.terminate()
        if self.t is not None:
            self.t.join(timeout=5)
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.mx,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": self.src}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def make_images(e, p, batch, seed, scan=2_000_000):
    from lauematching_b200 import synth
    rng = np.random.default_rng(seed)
    rec = e.download_db(0, min(scan, e.n_orient))
    imgs = []
    for _ in range(batch):
        g = synth.pick_grains(rec, int(rng.integers(1, 21)), p.min_nr_spots, rng)
        img = synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng)
        imgs.append(img.astype(np.uint8))
    return imgs, rec


def dbbuild_parity_sample(e, p, hkls, seed, n_orient, per_block=20000, blocks=5):
    """Records of the device-built DB against the oracle on sampled ID blocks."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    rng = np.random.default_rng(1234)
    starts = sorted(set(int(x) for x in rng.integers(0, max(1, n_orient - per_block), blocks)))
    mism = 0
    total = 0
    for s in starts:
        cnt = min(per_block, n_orient - s)
        om = e.synth_orientations(seed, s, cnt)
        ref = O.forward(p, om, hkls)
        got = e.download_db(s, cnt)
        mism += int(np.count_nonzero(np.any(ref != got, axis=1)))
        total += cnt
    return {"sampled_orientations": total, "records_differing": mism}


def _same_fields(sub, want):
    return (np.array_equal(sub["id"], want.ids.astype(np.uint64))
            and np.array_equal(sub["n_spots"], want.n_spots)
            and np.array_equal(sub["sum_u8"], want.sum_u8)
            and np.array_equal(sub["tot_int"].view(np.uint64), want.tot_int.view(np.uint64))
            and np.array_equal(sub["score"].view(np.uint64), want.score.view(np.uint64)))


def survivor_parity(e, p, img_u8, n_sample=None, chunk=4_000_000, sink=None):
    """This run's survivors of one bench image against the oracle over the
    DB's first n_sample records (all of them by default), chunk by chunk:
    ids, spot counts, uint8 sums and the FP64 intensity sums and scores bit
    for bit.  ``sink(first, records)`` also receives every chunk of records
    (to write the reference's input files from the same pass).  Returns
    (summary, our survivors over the whole DB, n_pass)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    e.load_image(0, img_u8, want_scale=False)
    e.match([0], p.min_nr_spots, p.min_intensity)
    ours, npass = e.results(0)
    n_sample = min(n_sample or e.n_orient, e.n_orient)
    img = img_u8.astype(np.float64)
    same, n_want, n_got, t_or = True, 0, 0, 0.0
    for first in range(0, n_sample, chunk):
        cnt = min(chunk, n_sample - first)
        rec = e.download_db(first, cnt)
        if sink is not None:
            sink(first, rec)
        t0 = time.perf_counter()
        want = O.compare(rec, p.max_nr_spots, img, p.nr_px_x, p.nr_px_y, p.min_nr_spots,
                         p.min_intensity, nthreads=os.cpu_count() or 1)
        t_or += time.perf_counter() - t0
        want.ids = want.ids.astype(np.uint64) + np.uint64(first)
        sub = ours[(ours["id"] >= first) & (ours["id"] < first + cnt)]
        same = same and _same_fields(sub, want)
        n_want += int(want.ids.shape[0])
        n_got += int(sub.shape[0])
    return {"records": n_sample, "survivors": n_got, "oracle_survivors": n_want,
            "identical": bool(same and n_got == n_want), "oracle_seconds": round(t_or, 2),
            "oracle_threads": os.cpu_count() or 1}, ours, npass


def full_db_parity_and_cpu_baseline(e, p, txt, hkls, img_u8, seed, cpu=True, parity=True):
    """One bench image over the whole device DB, three ways:

    * our survivors against the oracle on every record (survivor_parity);
    * the reference's own LaueMatchingCPU (DoFwd 0, all host cores) on the
      same DB written as its ForwardFile (the device build is byte-identical
      to the reference's cache) and the orientations as its orientation
      file: its compare stage, unscaled, is the CPU baseline;
    * its "Initial solutions" count and its solutions.txt / spots.txt
      against this library's post-stage on our survivors, byte for byte.

    Needs the DB files on the host (194 B per orientation, /dev/shm when it
    has room so the reference memory-maps them); a host too small for the
    whole DB gets the largest prefix that fits, and the records field says
    so."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lauematching_b200 import formats, post
    n = e.n_orient
    per = REC_BYTES_PER_ORIENT + 72
    base = scratch_dir(n * per)
    if base is None:
        import psutil
        n = int(min(n, psutil.virtual_memory().available * 0.4 // per))
    have_ref = cpu and O.have_ref() and n > 0
    wd = tempfile.mkdtemp(prefix="lmb_full_", dir=base)
    fwd, op = os.path.join(wd, "fwd.bin"), os.path.join(wd, "orients.bin")
    files = {}
    if have_ref:
        files = {"fwd": open(fwd, "wb"), "om": open(op, "wb")}

    def sink(first, rec):
        if files:
            rec.tofile(files["fwd"])
            e.synth_orientations(seed, first, rec.shape[0]).tofile(files["om"])
    out = {}
    try:
        t0 = time.perf_counter()
        par, ours, npass = survivor_parity(e, p, img_u8, n_sample=n, sink=sink)
        if parity:
            out["survivor_parity"] = par
        for f in files.values():
            f.close()
        t_write = time.perf_counter() - t0
        if not have_ref:
            return out
        hp, ip, pp = (os.path.join(wd, x) for x in ("hkls.csv", "image.bin", "params.txt"))
        formats.write_hkls(hp, hkls)
        img = img_u8.astype(np.float64)
        formats.write_image_bin(ip, img)
        with open(pp, "w") as f:
            f.write(txt + f"ForwardFile {fwd}\nDoFwd 0\n")
        cores = os.cpu_count() or 1
        r = O.run_reference(pp, op, hp, ip, ncpus=cores)
        if r.returncode != 0 or r.compare_seconds is None:
            raise RuntimeError("reference run failed: " + r.stdout[-500:] + r.stderr[-500:])
        sub = ours[ours["id"] < n]
        ids, sc = post.collected_matches(sub, sub.shape[0] if n < e.n_orient else npass)
        om = np.memmap(op, dtype=np.float64, mode="r").reshape(-1, 9)
        sol, spt, _ = post.post_process(p, e.geometry, om, ids, sc, img.astype(np.float32),
                                        hkls, num_threads=cores, merge_device=e.device)
        del om
        # the reference writes each grain's lines from an OpenMP loop inside a
        # critical section (LaueMatchingHeaders.h:1128-1150): with several
        # threads its line order follows the scheduling, so the lines are
        # compared as sorted sets, and the exact bytes are reported beside
        same_sol = sorted((r.solutions or "").splitlines()) == \
            sorted((post.SOLUTIONS_HEADER + sol).splitlines())
        same_spt = sorted((r.spots or "").splitlines()) == \
            sorted((post.SPOTS_HEADER + spt).splitlines())
        same_bytes = r.solutions == post.SOLUTIONS_HEADER + sol and \
            r.spots == post.SPOTS_HEADER + spt
        out["cpu_baseline"] = {
            "value": 1.0 / r.compare_seconds * (n / 1e8), "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": f"LaueMatchingCPU (reference source, gcc -O3 -fopenmp, NLopt stand-in) "
                      f"DoFwd 0, one bench image against {n:,} records (the device-built DB "
                      f"written as its ForwardFile{' in /dev/shm' if base else ''}): compare "
                      f"stage {r.compare_seconds:.3f} s"
                      + ("" if n == e.n_orient else f", scaled x{1e8 / n:g} to 1e8")
                      + f"; whole process {r.wall_seconds:.2f} s"}
        out["reference_full_db"] = {
            "records": n, "initial_solutions": {"reference": r.initial_solutions,
                                                "ours": int(sub.shape[0]),
                                                "identical": r.initial_solutions == sub.shape[0]},
            "unique_orientations": r.unique,
            "solutions_txt_lines_identical": bool(same_sol),
            "spots_txt_lines_identical": bool(same_spt),
            "files_byte_identical_in_order": bool(same_bytes),
            "reference_threads": cores, "files_written_s": round(t_write, 1)}
        # the reference's plain single-image GPU executable (LaueMatchingGPU.cu,
        # sm_100a build) on the same files: one process, the DB streamed to the
        # device in <= 4 GB chunks, its one-thread-per-orientation kernel
        if O.have_ref_gpu():
            env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
            rg = O.run_reference_gpu(pp, op, hp, ip, ncpus=cores, env=env)
            if rg.returncode == 0 and rg.chunks:
                k_s = sum(k for _, k in rg.chunks)
                out["reference_gpu"] = {
                    "binary": "oracle/_ref/LaueMatchingGPU (reference source, nvcc -O3 -w "
                              "-rdc=true sm_100a, NLopt stand-in)",
                    "records": n, "kernel_s_per_image": round(k_s, 5),
                    "kernel_images_per_s": round(1.0 / k_s, 2) if k_s > 0 else None,
                    "kernel_time_resolution_s": 0.001,
                    "match_stage_s_per_image": rg.match_seconds,
                    "match_stage_images_per_s": round(1.0 / rg.match_seconds, 3)
                    if rg.match_seconds else None,
                    "forward_read_s": rg.read_seconds, "chunks_h2d_kernel_s": rg.chunks,
                    "process_wall_s": round(rg.wall_seconds, 2),
                    "nr_matches": rg.n_matches, "n_pass_ours": int(npass)}
            else:
                out["reference_gpu"] = {"failed": (rg.stderr or rg.stdout)[-300:]}
        return out
    finally:
        for f in files.values():
            f.close()
        for fn in os.listdir(wd):
            os.remove(os.path.join(wd, fn))
        os.rmdir(wd)


# DRAM bytes (read + write) per orientation of one compare launch, from ncu
# captures of smaller DBs of this workload (the figures and commands are in
# profiles/compare_*.md); traffic grows with the DB, so roofline.traffic
# scales them to N.
TRAFFIC_BYTES_PER_ORIENT = {
    "reference": 271.1e6 / 2_000_000,  # compare_ws_kernel, 2M orientations, K=16
    "compact": 205.6e6 / 30_000_000,   # compare_clist_kernel, 30M orientations, K=64
}


def merge_timing(space_group, max_angle, device, n_base=800, per=12, seed=5):
    """The duplicate merge of ~1e4 candidates (near-duplicate families: base
    orientations and copies rotated by up to 4 degrees, shuffled): host loop
    (the reference's algorithm, all host threads) against the device merge."""
    from lauematching_b200 import post, synth
    rng = np.random.default_rng(seed)
    base = synth.shoemake_orientations(n_base, seed=seed).reshape(-1, 3, 3)
    om = []
    for b in base:
        om.append(b)
        for _ in range(per - 1):
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            ang = np.deg2rad(rng.uniform(0, 4.0))
            k = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            om.append((np.eye(3) + np.sin(ang) * k + (1 - np.cos(ang)) * (k @ k)) @ b)
    om = np.array(om).reshape(-1, 9)[rng.permutation(n_base * per)]
    rows = np.arange(om.shape[0], dtype=np.uint64)
    scores = rng.integers(1, 40, om.shape[0]).astype(np.float64) * 3.5
    post.merge_clusters(space_group, max_angle, om, rows[:2048], scores[:2048], device=device)
    t_devs = []
    for _ in range(3):
        t0 = time.perf_counter()
        dev = post.merge_clusters(space_group, max_angle, om, rows, scores, device=device)
        t_devs.append(time.perf_counter() - t0)
    t_dev = statistics.median(t_devs)
    t0 = time.perf_counter()
    host = post.merge_clusters(space_group, max_angle, om, rows, scores)
    t_host = time.perf_counter() - t0
    same = all(np.array_equal(a, b) for a, b in zip(host, dev))
    return {"candidates": int(om.shape[0]), "clusters": int(host[0].shape[0]),
            "host_ms": round(t_host * 1e3, 1), "host_threads": os.cpu_count(),
            "device_ms": round(t_dev * 1e3, 2), "device_ms_runs": [round(t * 1e3, 2) for t in t_devs],
            "identical": same}


# The tilted detector of APS 34-ID-E (P_Array, R_Array as the reference's
# example parameter files give them); spots per orientation ~20, so the
# refinement objective sees realistic valid-HKL lists.
TILTED_P = (0.028745, 0.002788, 0.513115)
TILTED_R = (-1.20131258, -1.21399082, -1.21881158)


def pass_stats(e, slots, p, n):
    """n passes back to back on the engine stream: mean compare-kernel time
    (per-pass events, synchronised) and the per-pass time of an unsynchronised
    stream of passes (CUDA events around the whole stream)."""
    import torch
    stream = torch.cuda.ExternalStream(e.stream)
    cmp = []
    for _ in range(max(3, n // 4)):
        e.match(slots, p.min_nr_spots, p.min_intensity)
        cmp.append(e.last_pass_ms()[0])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(n):
        e.match(slots, p.min_nr_spots, p.min_intensity)
    b.record(stream)
    b.synchronize()
    return statistics.mean(cmp), a.elapsed_time(b) / n


def survivor_lists(e, slots):
    return {k: e.results(k) for k in slots}


def same_survivors(x, y):
    for k in x:
        (a, na), (b, nb) = x[k], y[k]
        if na != nb or a.shape != b.shape:
            return False
        for f in ("id", "n_spots", "sum_u8"):
            if not np.array_equal(a[f], b[f]):
                return False
        for f in ("tot_int", "score"):
            if not np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)):
                return False
    return True


def gather_counts(rec, p, imgs, mask_shift):
    """Per DB record of a sample: spots, spots of the records that can pass
    (>= MinNrSpots on-detector spots), and the gathers left after the cell
    mask of the batch (cells of 2^shift consecutive pixels holding a positive
    pixel of any frame) -- the counts the compare kernels act on."""
    W, H = p.nr_px_x, p.nr_px_y
    S = p.max_nr_spots
    cnt = np.minimum(rec[:, 0].astype(np.int64), S)
    xs = rec[:, 1::2].astype(np.int64)
    ys = rec[:, 2::2].astype(np.int64)
    on = (np.arange(S)[None, :] < cnt[:, None]) & (xs < W) & (ys < H)
    pix = np.where(on, ys * W + xs, 0)
    c_on = on.sum(1)
    pos = np.zeros(W * H, bool)
    for im in imgs:
        pos |= np.asarray(im).ravel() > 0
    cells = np.zeros(((W * H) >> mask_shift) + 1, bool)
    cells[np.nonzero(pos)[0] >> mask_shift] = True
    hit = cells[pix >> mask_shift] & on
    ub = hit.sum(1)
    need = max(1, p.min_nr_spots)
    n = rec.shape[0]
    return {"spots_per_record": round(float(c_on.mean()), 3),
            "passable_records": round(float((c_on >= need).mean()), 4),
            "gathers_per_record_unfiltered": round(float(c_on[c_on >= need].sum()) / n, 3),
            "union_pixel_density": round(float(pos.mean()), 4),
            "cell_mask_shift": int(mask_shift),
            "cell_density": round(float(cells[:-1].mean()), 4),
            "records_past_cell_mask": round(float((ub >= need).mean()), 4),
            "gathers_per_record_cell_mask": round(float(hit[ub >= need].sum()) / n, 3),
            "sample_records": int(n)}


def tilted_leg(args, dev, K=64, n=None):
    """The batched pass at the reference's own detector geometry (APS 34-ID-E,
    simulation/params_sim.txt: tilted 2048^2 detector at ~0.51 m, fcc Ni-like
    a=3.52 A, 1240 HKLs, 5-30 keV, MaxNrLaueSpots 30, MinNrSpots 5): ~15
    on-detector spots per record instead of ~1.25, so nearly every record can
    pass and the image gathers, not the DB stream, decide the pass.  Every
    variant's survivors are compared; the automatic one is the headline."""
    from lauematching_b200 import params as P, synth
    from lauematching_b200.engine import Engine
    n = n or args.n_orient
    txt = synth.params_text(p=TILTED_P, r=TILTED_R, max_nr_spots=30, min_nr_spots=5,
                            min_intensity=args.min_intensity)
    p = P.parse_params_text(txt)
    hk = synth.hkls_cubic(8)
    e = Engine(p, device=dev)
    try:
        t0 = time.perf_counter()
        e.build_db_synthetic(seed=args.seed, n=n, hkls=hk)
        t_build = time.perf_counter() - t0
        imgs, rec = make_images(e, p, K, seed=2000)
        for k in range(K):
            e.load_image(k, imgs[k], want_scale=False)
        slots = list(range(K))
        nsteps = max(5, min(args.steps, 40))
        out = {"workload": f"{K} uint8 2048x2048 frames (U{{1..20}} fcc grains each) vs a "
                           f"{n:,}-orientation DB, tilted 34-ID-E detector",
               "n_orient": n, "batch": K, "min_nr_spots": p.min_nr_spots,
               "min_intensity": p.min_intensity, "dbbuild_s": round(t_build, 3)}
        runs = {}
        ref_surv = None
        for name, tun in (("auto", None), ("reference_layout", dict(variant=1)),
                          ("compact_no_mask", dict(variant=2, stages=2, consumers=3,
                                                   grid_mult=8)),
                          ("cell_mask_in_place", dict(variant=4)),
                          ("cell_mask_queued", dict(variant=4, cell_queue=1)),
                          ("cell_filter_then_count", dict(variant=5))):
            if tun is None:
                e._pinned_shape = False
                e._shape_bucket = None
            else:
                e.set_tuning(**tun)
            pass_stats(e, slots, p, 3)
            cmp_ms, step_ms = pass_stats(e, slots, p, nsteps)
            sv = survivor_lists(e, slots)
            if ref_surv is None:
                ref_surv = sv
            runs[name] = {"compare_ms": round(cmp_ms, 4), "step_ms": round(step_ms, 4),
                          "images_per_s": round(K / (step_ms * 1e-3), 1),
                          "variant": e.get_tuning()["last_variant"],
                          "identical_to_auto": same_survivors(sv, ref_surv)}
        lay = e.layout_info()
        surv = [int(ref_surv[k][0].shape[0]) for k in slots]
        out["runs"] = runs
        # the survivor volume downstream of the pass: ordering kernel,
        # download of the 64 lists, host post-stage (merge on the device from
        # 1024 candidates, evaluate-once refinement, text) per image
        e._pinned_shape = False
        e._shape_bucket = None
        e.match(slots, p.min_nr_spots, p.min_intensity)
        order_ms = e.last_pass_ms()[1]
        t0 = time.perf_counter()
        res = e.results_batch(slots)
        t_dl = time.perf_counter() - t0
        nb = sum(r.nbytes for r, _ in res.values())
        from lauematching_b200 import post
        # rows filled for the survivors only (the host generator: the same
        # rotations as the device's to the last bit or so; this part is timed,
        # not compared)
        om_sparse = np.zeros((n, 9))
        post_ms, uniq = [], []
        for k in slots[:8]:
            sv, npass = res[k]
            u = np.unique(sv["id"]).astype(np.int64)
            om_sparse[u] = synth.shoemake_orientations(0, args.seed, ids=u)
            ids, sc = post.collected_matches(sv, npass)
            t0 = time.perf_counter()
            _, _, nu = post.post_process(p, e.geometry, om_sparse, ids, sc,
                                         imgs[k].astype(np.float32), hk,
                                         num_threads=os.cpu_count() or 1, merge_device=dev)
            post_ms.append((time.perf_counter() - t0) * 1e3)
            uniq.append(nu)
        del om_sparse
        out["downstream"] = {"order_kernel_ms": round(order_ms, 4),
                             "results_download_ms": round(t_dl * 1e3, 3),
                             "results_bytes": int(nb),
                             "post_stage_ms_per_image_median": round(statistics.median(post_ms), 2),
                             "post_stage_images": len(post_ms),
                             "unique_grains_per_image": uniq,
                             "host_threads": os.cpu_count()}
        out["survivors_per_image"] = {"min": min(surv), "max": max(surv),
                                      "mean": statistics.mean(surv)}
        shift = 0
        while ((p.nr_px_x * p.nr_px_y) >> shift) > 8 * 131072:
            shift += 1
        out["gathers"] = gather_counts(rec, p, imgs, shift)
        out["compact_layout"] = lay
        # roofline of the automatic pass: on the reference records (the D6
        # headline bytes) and on the layout it streams
        peak, peak_src = hbm_peak()
        auto = runs["auto"]
        t = auto["compare_ms"] * 1e-3
        ref_bytes = n * REC_BYTES_PER_ORIENT + K * p.nr_px_x * p.nr_px_y
        streamed = (lay["bytes"] + p.nr_px_x * p.nr_px_y * 8) if auto["variant"] in (2, 4, 5) \
            else ref_bytes
        out["roofline"] = {"bound": "hbm", "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                           "reference_layout_bytes": ref_bytes,
                           "reference_layout_gbs": round(ref_bytes / t / 1e9, 1),
                           "reference_layout_frac": round(ref_bytes / t / 1e9 / peak, 4),
                           "streamed_bytes": streamed,
                           "achieved": round(streamed / t / 1e9, 1),
                           "frac": round(streamed / t / 1e9 / peak, 4)}
        if not args.no_parity:
            out["survivor_parity"] = survivor_parity(e, p, imgs[0])[0]
    finally:
        e.close()
    return out


def volume_leg(args, e, rec, dev, K=16, min_ints=(50.0, 30.0), post_images=4):
    """Survivor volume downstream of the pass (the MinIntensity that gives
    1e3-1e4 survivors per image).  Frames of the bench geometry with the
    Poisson background kept (no threshold: every pixel is positive, so every
    record with >= MinNrSpots on-detector spots reaches the intensity test),
    K of them in one pass over the resident 1e8 DB; per MinIntensity: the
    pass (compare and ordering kernels), the download of the K sorted lists,
    the host post-stage of a few images (merge on the device from 1024
    candidates, evaluate-once refinement, text), and one frame's survivors
    against the oracle over all records."""
    from lauematching_b200 import post, synth
    rng = np.random.default_rng(77)
    frames = []
    for _ in range(K):
        g = synth.pick_grains(rec, int(rng.integers(1, 21)), 5, rng)
        frames.append(synth.render_image(rec[g], e.params.nr_px_x, e.params.nr_px_y, rng,
                                         threshold=None).astype(np.uint8))
    hk = synth.hkls_cubic(8)
    slots = list(range(K))
    out = {"workload": f"{K} uint8 2048x2048 frames with the Poisson(5) background kept "
                       f"(U{{1..20}} fcc grains each) vs the {e.n_orient:,}-orientation DB, "
                       "MinNrSpots 5", "runs": []}
    for mi in min_ints:
        _, p = workload_params(mi)
        for k in slots:
            e.load_image(k, frames[k], want_scale=False)
        for _ in range(3):
            e.match(slots, p.min_nr_spots, p.min_intensity)
            e.results_batch(slots)
        cmp_ms, order_ms, step_ms, dl_ms = [], [], [], []
        for _ in range(max(3, min(args.steps, 10))):
            t0 = time.perf_counter()
            e.match(slots, p.min_nr_spots, p.min_intensity)
            res = e.results_batch(slots)
            step_ms.append((time.perf_counter() - t0) * 1e3)
            c, o = e.last_pass_ms()[:2]
            cmp_ms.append(c)
            order_ms.append(o)
        t0 = time.perf_counter()
        res = e.results_batch(slots)
        dl_ms.append((time.perf_counter() - t0) * 1e3)
        surv = [int(res[k][0].shape[0]) for k in slots]
        om_sparse = np.zeros((e.n_orient, 9))
        post_ms, uniq = [], []
        for k in slots[:post_images]:
            sv, npass = res[k]
            u = np.unique(sv["id"]).astype(np.int64)
            om_sparse[u] = synth.shoemake_orientations(0, args.seed, ids=u)
            ids, sc = post.collected_matches(sv, npass)
            t0 = time.perf_counter()
            _, _, nu = post.post_process(p, e.geometry, om_sparse, ids, sc,
                                         frames[k].astype(np.float32), hk,
                                         num_threads=os.cpu_count() or 1, merge_device=dev)
            post_ms.append((time.perf_counter() - t0) * 1e3)
            uniq.append(int(nu))
        del om_sparse
        run = {"min_intensity": mi,
               "survivors_per_image": {"min": min(surv), "max": max(surv),
                                       "mean": round(statistics.mean(surv), 1)},
               "compare_ms": round(statistics.median(cmp_ms), 4),
               "order_kernel_ms": round(statistics.median(order_ms), 4),
               "match_and_download_ms": round(statistics.median(step_ms), 3),
               "results_download_ms": round(dl_ms[0], 3),
               "results_bytes": int(sum(r.nbytes for r, _ in res.values())),
               "post_stage_ms_per_image": [round(x, 1) for x in post_ms],
               "unique_grains_per_image": uniq}
        if not args.no_parity:
            run["survivor_parity"] = survivor_parity(e, p, frames[0])[0]
        out["runs"].append(run)
    return out


def dbbuild_leg(args, dev):
    """The device DB build alone: n device-generated orientations (seed 1)
    forward-simulated with the 1240 fcc HKLs, on the bench's beam-normal
    detector and on the tilted 34-ID-E detector.  The first build of an
    engine includes the DB allocation (cudaMalloc of n x 122 B) and the
    kernels' first launch; the repeated builds run into the allocated DB.
    Times are synchronised wall time around the whole build call."""
    import torch
    from lauematching_b200 import params as P, synth
    from lauematching_b200.engine import Engine
    n = args.n_orient
    hk = synth.hkls_cubic(8)
    out = {"n_orient": n, "hkls": int(len(hk))}
    for name, geo in (("beam_normal", {}), ("tilted", dict(p=TILTED_P, r=TILTED_R))):
        p = P.parse_params_text(synth.params_text(max_nr_spots=30, **geo))
        with Engine(p, device=dev) as e:
            ts = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                e.build_db_synthetic(seed=args.seed, n=n, hkls=hk)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
        out[name] = {"first_build_s": round(ts[0], 3), "warm_build_s": round(min(ts[1:]), 3),
                     "warm_orientations_per_s": round(n / min(ts[1:]), 1),
                     "warm_hkl_evals_per_s": round(n * len(hk) / min(ts[1:]), 1)}
    return out


HEX_LATTICE = (0.295, 0.295, 0.468, 90.0, 90.0, 120.0)


def hex_leg(args, dev, K=32, grains=5, top=50, n=None):
    """Lower symmetry plus refinement: hexagonal a=2.95 A, c=4.68 A (SG 194),
    the 7790 HKLs with |h|,|k|,|l| <= 10, a DB of 1e8 rotations restricted to
    the hexagonal fundamental zone, built on the device (timed: the DB
    build's hardest HKL count); 32 frames of 5 grains each, every frame
    simulated with c/a scaled by 1+U(-1 %, +1 %); one batched pass; the top
    50 candidates of every frame by score go to the c/a refinement
    (tol_c_over_a 0.02, FitOrientation's box, LaueMatchingHeaders.h:664,714,
    738) with this library's Nelder-Mead, objective on the device and, for
    comparison, on host threads."""
    from lauematching_b200 import params as P, synth
    from lauematching_b200.engine import Engine
    from lauematching_b200.refine import Refiner
    n = n or args.n_orient
    seed = 3

    def text(lat, tol=0.0):
        return synth.params_text(lattice=lat, space_group=194, max_nr_spots=30, min_nr_spots=5,
                                 min_intensity=args.min_intensity, tol_c_over_a=tol)
    p = P.parse_params_text(text(HEX_LATTICE))
    pr = P.parse_params_text(text(HEX_LATTICE, 0.02))
    hk = synth.hkls_hexagonal(10)
    W, H = p.nr_px_x, p.nr_px_y
    e = Engine(p, device=dev)
    try:
        t0 = time.perf_counter()
        e.build_db_synthetic(seed=seed, n=n, hkls=hk, hex_fz=True)
        t_build = time.perf_counter() - t0
        scan = min(2_000_000, n)
        rec = e.download_db(0, scan)
        om_scan = e.synth_orientations(seed, 0, scan)
        rng = np.random.default_rng(3000)
        frames, ca_true, true_ids = [], [], []
        for _ in range(K):
            ca = 1.0 + rng.uniform(-0.01, 0.01)
            g = synth.pick_grains(rec, grains, p.min_nr_spots, rng)
            lat = (HEX_LATTICE[0], HEX_LATTICE[1], HEX_LATTICE[2] * ca) + HEX_LATTICE[3:]
            with Engine(P.parse_params_text(text(lat)), device=dev, survivor_capacity=1024) as eg:
                eg.build_db(om_scan[g], hk)
                grec = eg.download_db()
            frames.append(synth.render_image(grec, W, H, rng).astype(np.uint8))
            ca_true.append(ca)
            true_ids.append(g)
        del om_scan
        for k in range(K):
            e.load_image(k, frames[k], want_scale=False)
        slots = list(range(K))
        nsteps = max(5, min(args.steps, 40))
        pass_stats(e, slots, p, 3)
        cmp_ms, step_ms = pass_stats(e, slots, p, nsteps)
        res = {k: e.results(k) for k in slots}
        surv = [int(res[k][0].shape[0]) for k in slots]
        out = {"workload": f"{K} uint8 {W}x{H} frames of {grains} hexagonal grains (c/a x "
                           f"(1+U(-1%,+1%)) per frame) vs a {n:,}-orientation hexagonal "
                           f"fundamental-zone DB, SG 194, {len(hk)} HKLs",
               "n_orient": n, "batch": K, "hkls": int(len(hk)),
               "dbbuild": {"seconds": round(t_build, 3),
                           "orientations_per_s": round(n / t_build, 1),
                           "hkl_evals_per_s": round(n * len(hk) / t_build, 1)},
               "pass": {"compare_ms": round(cmp_ms, 4), "step_ms": round(step_ms, 4),
                        "images_per_s": round(K / (step_ms * 1e-3), 1),
                        "variant": e.get_tuning()["last_variant"]},
               "survivors_per_image": {"min": min(surv), "max": max(surv),
                                       "mean": statistics.mean(surv)}}
        # the top candidates of every frame into the c/a refinement
        cand, img_of, ca_of = [], [], []
        for k in slots:
            sv = res[k][0]
            order = np.argsort(-sv["score"], kind="stable")[:top]
            cand += [int(i) for i in sv["id"][order]]
            img_of += [k] * len(order)
            ca_of += [ca_true[k]] * len(order)
        om_c = np.concatenate([e.synth_orientations(seed, i, 1) for i in cand]) if cand \
            else np.zeros((0, 9))
        fl = [f.astype(np.float32).reshape(H, W) for f in frames]
        fits = {}
        for name, d in (("device", dev), ("host", None)):
            with Refiner(pr, e.geometry, hk, device=d) as r:
                r.set_images(fl)
                nv = r.set_grains(om_c, np.array(img_of, np.int32))
                x0, _, _ = r.start()
                r.fit("nelder-mead", 200)  # warm
                t0 = time.perf_counter()
                x, ov, ev = r.fit("nelder-mead", 200)
                dt = time.perf_counter() - t0
                st = r.last_stats()
                fits[name] = (x, ov, ev)
                out.setdefault("refine", {})[name] = {
                    "fit_ms": round(dt * 1e3, 2), "grains": int(len(cand)),
                    "evaluations": st["points"], "rounds": st["rounds"],
                    "objective_kernel_ms": round(st["kernel_ms"], 3)}
        x, ov, _ = fits["device"]
        ref = out["refine"]
        ref["identical_device_host"] = all(np.array_equal(a, b) for a, b in
                                           zip(fits["device"], fits["host"]))
        ref["valid_hkls_per_grain"] = round(float(nv.mean()), 1) if len(nv) else 0.0
        if len(cand):
            ca0 = P.parse_params_text(text(HEX_LATTICE)).lattice
            ca_orig = ca0[2] / ca0[0]
            truth = np.array(ca_of)
            # candidates that are one of their frame's true grains
            hit = np.array([c in set(true_ids[k].tolist()) for c, k in zip(cand, img_of)])
            err0 = np.abs(1.0 - truth)
            err1 = np.abs(x[:, 3] / ca_orig - truth)
            ref["c_over_a_rel_error_median"] = {
                "before": float(np.median(err0)), "after_all": float(np.median(err1)),
                "after_true_grains": float(np.median(err1[hit])) if hit.any() else None,
                "true_grain_candidates": int(hit.sum())}
        if not args.no_parity:
            out["survivor_parity"] = survivor_parity(e, p, frames[0])[0]
            out["dbbuild"]["parity"] = dbbuild_parity_sample(e, p, hk, seed, n, per_block=10000,
                                                             blocks=2)
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import ref_objective as RO
            if RO.available() and len(cand):
                ro = RO.RefObjective(pr, e.geometry, hk)
                m = min(64, len(cand))
                with Refiner(pr, e.geometry, hk, device=dev) as r:
                    r.set_images(fl)
                    r.set_grains(om_c[:m], np.array(img_of[:m], np.int32))
                    x0, _, _ = r.start()
                    pts = np.concatenate([x0, x[:m]])
                    gi = np.concatenate([np.arange(m), np.arange(m)])
                    val = r.evaluate(gi, pts)
                want = [ro.problem(pts[j], fl[img_of[gi[j]]], ro.prefilter(x0[gi[j]][:3]))
                        for j in range(len(gi))]
                out["refine"]["objective_vs_reference"] = {
                    "points": int(len(gi)),
                    "identical": bool(np.array_equal(val, np.array(want)))}
    finally:
        e.close()
    return out


def hbm_peak():
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        return float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def refine_scene(device, n_frames, per_frame, seed=17, min_spots=8):
    """Frames rendered from true grains and coarse matrices 0.05-0.3 degrees
    off them (a DB grid's neighbour), tilted detector, fcc Ni, 1240 HKLs.
    The true grains' spots come from the device DB build."""
    from lauematching_b200 import params as P, synth
    from lauematching_b200.engine import Engine
    txt = synth.params_text(p=TILTED_P, r=TILTED_R, max_nr_spots=30, min_nr_spots=5)
    p = P.parse_params_text(txt)
    hk = synth.hkls_cubic(8)
    rng = np.random.default_rng(seed)
    n_cand = 40 * n_frames * per_frame
    e = Engine(p, device=device)
    try:
        e.build_db_synthetic(seed, n_cand, hk)
        rec = e.download_db(0, n_cand)
        om_all = e.synth_orientations(seed, 0, n_cand)
    finally:
        e.close()
    ok = np.nonzero(rec[:, 0] >= min_spots)[0][:n_frames * per_frame]
    frames, image = [], []
    for f in range(n_frames):
        sel = ok[f * per_frame:(f + 1) * per_frame]
        img = synth.render_image(rec[sel], p.nr_px_x, p.nr_px_y, rng)
        frames.append(img.astype(np.float32).reshape(p.nr_px_y, p.nr_px_x))
        image += [f] * per_frame
    om_c = synth.perturb_orientations(om_all[ok], rng, 0.05, 0.3)
    return p, hk, frames, np.array(image, np.int32), om_c


def refine_timing(device, sizes=((32, 24), (32, 192)), max_eval=200, reps=3, cpu=True):
    """Refinement of the grains of a batch (FitOrientation of every grain,
    200 evaluations at most): this library's lockstep Nelder-Mead with the
    objective on the device (one launch per group round) against the same fit
    with the objective on all host threads (identical results), at a few
    grains per frame and at many (polycrystal frames), and the reference's
    own problem_function timed on one host thread."""
    from lauematching_b200.engine import geometry_from_params
    from lauematching_b200.refine import Refiner
    out = {"runs": []}
    for n_frames, per_frame in sizes:
        p, hk, frames, image, om_c = refine_scene(device, n_frames, per_frame)
        geo = geometry_from_params(p)
        run = {"workload": f"{len(om_c)} grains over {n_frames} 2048x2048 float frames "
                           f"(tilted detector, fcc, {len(hk)} HKLs), coarse matrices 0.05-0.3 deg "
                           f"off the true grains, Nelder-Mead <= {max_eval} evaluations per grain"}
        res = {}
        for name, dev in (("device", device), ("host", None)):
            with Refiner(p, geo, hk, device=dev) as r:
                t0 = time.perf_counter()
                r.set_images(frames)
                nv = r.set_grains(om_c, image)
                t_setup = time.perf_counter() - t0
                _, ov0, _ = r.fit("once")
                ts, kms = [], []
                for _ in range(reps if dev is not None else 1):
                    t0 = time.perf_counter()
                    x, ov, ev = r.fit("nelder-mead", max_eval)
                    ts.append(time.perf_counter() - t0)
                    kms.append(r.last_stats()["kernel_ms"])
                st = r.last_stats()
                res[name] = (x, ov, ev)
                fit_s = statistics.median(ts)
                run[name] = {"fit_ms": round(fit_s * 1e3, 2),
                             "grains_per_s": round(len(om_c) / fit_s, 1),
                             "evaluations_per_s": round(st["points"] / fit_s, 1),
                             "rounds": st["rounds"], "evaluations": st["points"],
                             "setup_ms": round(t_setup * 1e3, 1)}
                if dev is not None:
                    km = statistics.median(kms)
                    run[name]["objective_kernel_ms"] = round(km, 3)
                    run[name]["kernel_evaluations_per_s"] = round(st["points"] / (km * 1e-3), 1)
                    run["valid_hkls_per_grain"] = round(float(nv.mean()), 1)
                    run["overlap_start_mean"] = round(float(ov0.mean()), 1)
                    run["overlap_fit_mean"] = round(float(ov.mean()), 1)
                    run["improved_grains"] = int((ov > ov0).sum())
                else:
                    run[name]["threads"] = os.cpu_count()
        run["identical"] = all(np.array_equal(a, b) for a, b in zip(res["device"], res["host"]))
        run["device_over_host"] = round(run["host"]["fit_ms"] / run["device"]["fit_ms"], 2)
        out["runs"].append(run)
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref_objective as RO
        if RO.available():
            ref = RO.RefObjective(p, geo, hk)
            x0 = [ref.start(om_c[g])[0] for g in range(min(64, len(om_c)))]
            valid = [ref.prefilter(x[:3]) for x in x0]
            n_ev = 0
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 2.0:
                for g, x in enumerate(x0):
                    ref.problem(x, frames[int(image[g])], valid[g])
                    n_ev += 1
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {
                "kind": "reference", "cores": 1,
                "value": round(n_ev / dt, 1), "unit": "evaluations/s",
                "sample": f"the reference's problem_function (LaueMatchingHeaders.h, compiled "
                          f"from the reference tree) at the start points of {len(x0)} grains, "
                          f"{n_ev} evaluations in {dt:.2f} s on one thread; the reference runs "
                          f"one grain per OpenMP thread"}
    return out


def preprocess_timing(device, parity=True, cpu_port=True, frames=20):
    """Frame preprocessing (laue_index.preprocess_image's steps) of a 2048^2
    detector frame on the device: the image server's flow (background from
    the first frame's median, then per frame subtraction, adaptive threshold,
    components, centres, blur), timed through the public API, plus the CPU
    port of the same steps on one frame."""
    from lauematching_b200 import preprocess as PP, synth
    from lauematching_b200.engine import PinnedBuffer
    rng = np.random.default_rng(21)
    raw = synth.raw_frame(2048, 2048, rng, n_spots=600)
    cfg = dict(nr_px_x=2048, nr_px_y=2048, filter_radius=101, median_passes=1,
               threshold_method="adaptive", threshold_value=0.0, threshold_percentile=90.0,
               min_area=10, px_x=0.2, distance=0.513, orientation_spacing=0.4)
    h = PP.DevicePreprocessor(2048, 2048, device)
    med_ms, med_kernel = [], []
    for i in range(4):
        t0 = time.perf_counter()
        bg = h.median(raw, 101, 1)
        if i:
            med_ms.append(1e3 * (time.perf_counter() - t0))
            tm = h.timings()
            med_kernel.append(tm["median_ranks"] + tm["median"])
    h.close()

    def run(pre, frame):
        for _ in range(3):
            pre(frame)
        wall, devm = [], []
        for _ in range(frames):
            t0 = time.perf_counter()
            out = pre(frame)
            wall.append(1e3 * (time.perf_counter() - t0))
            tm = pre._h.timings()
            devm.append(tm["threshold"] + tm["components"] + tm["blur"])
        return float(np.median(wall)), float(np.median(devm)), pre._h.timings(), out

    fresh = PP.Preprocessor(cfg, bg)
    w_fresh, d_fresh, _, out = run(fresh, raw)
    pin = PinnedBuffer(raw.shape, np.uint16)
    pin.array[...] = raw.astype(np.uint16)
    fast = PP.Preprocessor(cfg, bg, blur_dtype=np.float32, reuse_outputs=True)
    w_fast, d_fast, stages, _ = run(fast, pin.array)
    res = {"workload": "2048x2048 detector frame (pedestal + Poisson + 600 spots), background "
                       "= median of radius 101 computed once, adaptive threshold, min_area 10",
           "centres": len(out[3]),
           "device_ms_per_frame": round(d_fast, 4),
           "device_frames_per_s": round(1e3 / d_fast, 1),
           "e2e_ms_per_frame": {"float64_frame_new_arrays": round(w_fresh, 3),
                                "pinned_uint16_frame_reused_outputs_float32_blur": round(w_fast, 3)},
           "e2e_frames_per_s": round(1e3 / w_fast, 1),
           "stages_ms": {k: v for k, v in stages.items() if not k.startswith("median")},
           "median_background_ms": {"radius": 101, "device": round(float(np.median(med_kernel)), 3),
                                    "e2e": round(float(np.median(med_ms)), 3)}}
    if parity or cpu_port:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import preprocess_oracle as PO
        t0 = time.perf_counter()
        want = PO.preprocess_image(raw, cfg, background=bg)
        t_port = time.perf_counter() - t0
        if parity:
            res["identical_to_oracle"] = bool(
                np.array_equal(out[0].view(np.uint8), want["blurred"].view(np.uint8))
                and np.array_equal(out[2], want["filt_labels"]))
        if cpu_port:
            res["cpu_port_s_per_frame"] = round(t_port, 3)
    fresh.close()
    fast.close()
    pin.free()
    return res


def raw_frame_pipeline(e, p, rec, K=64, reps=5, seed=33):
    """Raw detector frames to survivors on one GPU: K uint16 frames (pedestal,
    Poisson noise, spots of 1-20 DB grains) preprocessed straight into the
    engine's slots (background = median of the first frame, as the image
    server computes it), one batched pass, survivors downloaded; against the
    same with the blurred float32 frames taken to the host and loaded back
    (the image server -> daemon hop).  Survivors must be identical."""
    from lauematching_b200 import preprocess as PP, synth
    from lauematching_b200.engine import PinnedBuffer
    rng = np.random.default_rng(seed)
    n_distinct = 16
    frames = []
    for _ in range(n_distinct):
        g = synth.pick_grains(rec, int(rng.integers(1, 21)), p.min_nr_spots, rng)
        f = synth.raw_frame(p.nr_px_y, p.nr_px_x, rng, spot_records=rec[g], sigma=1.2,
                            amp_lo=300.0, amp_hi=4000.0)
        pb = PinnedBuffer(f.shape, np.uint16)
        pb.array[...] = np.clip(f, 0, 65535).astype(np.uint16)
        frames.append(pb)
    cfg = dict(nr_px_x=p.nr_px_x, nr_px_y=p.nr_px_y, filter_radius=101, median_passes=1,
               threshold_method="adaptive", threshold_value=0.0, threshold_percentile=90.0,
               min_area=10, px_x=p.px_x, distance=p.p_array[2], orientation_spacing=0.4)
    bg = PP.compute_background(frames[0].array, 101, 1)
    pre = PP.Preprocessor(cfg, bg, blur_dtype=np.float32, reuse_outputs=True)
    slots = list(range(K))

    pool = PP.PreprocessPool(cfg, bg, device=e.device)

    def fused():
        pool.to_slots(e, slots, [frames[k % n_distinct].array for k in slots])
        e.match(slots, p.min_nr_spots, p.min_intensity)
        return e.results_batch(slots)

    def fused_serial():
        for k in slots:
            pre.to_slot(e, k, frames[k % n_distinct].array)
        e.match(slots, p.min_nr_spots, p.min_intensity)
        return e.results_batch(slots)

    def two_hop():
        for k in slots:
            b = pre(frames[k % n_distinct].array)[0]
            e.load_image(k, b, want_scale=False)
        e.match(slots, p.min_nr_spots, p.min_intensity)
        return e.results_batch(slots)

    a = fused()
    b = two_hop()
    c = fused_serial()
    same = all(a[k][1] == b[k][1] and np.array_equal(a[k][0], b[k][0]) and
               c[k][1] == b[k][1] and np.array_equal(c[k][0], b[k][0]) for k in slots)
    t_f, t_h, t_s = [], [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        fused()
        t_f.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        fused_serial()
        t_s.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        two_hop()
        t_h.append(time.perf_counter() - t0)
    pool.close()
    pre.close()
    for pb in frames:
        pb.free()
    tf, th = float(np.median(t_f)), float(np.median(t_h))
    return {"workload": f"{K} raw 2048x2048 uint16 frames (pedestal + Poisson + spots of 1-20 DB "
                        "grains) -> preprocessing (3 frames in flight) -> one batched pass vs the "
                        "1e8-orientation DB -> survivors",
            "frames_per_s": round(K / tf, 1), "ms_per_batch": round(tf * 1e3, 2),
            "one_frame_at_a_time_frames_per_s": round(K / float(np.median(t_s)), 1),
            "two_hop_frames_per_s": round(K / th, 1),
            "survivors_per_frame_mean": round(float(np.mean([len(a[k][0]) for k in slots])), 1),
            "identical_to_two_hop": bool(same)}


def run_ours(args, rank, world):
    import torch
    from lauematching_b200 import synth
    from lauematching_b200.engine import Engine, PinnedBuffer

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    txt, p = workload_params(args.min_intensity)
    hkls = synth.hkls_cubic(8)
    N, K = args.n_orient, args.batch
    e = Engine(p, device=dev)
    if args.variant is not None:  # pin the compare variant (else: the autotuned table)
        e.set_tuning(variant=args.variant)
    t0 = time.perf_counter()
    e.build_db_synthetic(seed=args.seed, n=N, hkls=hkls)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    log(f"[rank {rank}] DB built on device: {N} orientations in {t_build:.2f} s")
    imgs, rec_head = make_images(e, p, K, seed=1000 + rank)
    mean_spots = float(rec_head[:, 0].mean())
    stream = torch.cuda.ExternalStream(e.stream)

    # ---- resident batched pass ---------------------------------------------
    for k in range(K):
        e.load_image(k, imgs[k], want_scale=False)
    slots = list(range(K))

    def timed(nsteps, slot_list):
        """Passes one at a time (synchronised): per-pass step and compare-kernel
        times, for the roofline."""
        step_ms, cmp_ms = [], []
        for _ in range(nsteps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e.match(slot_list, p.min_nr_spots, p.min_intensity)
            b.record(stream)
            b.synchronize()
            step_ms.append(a.elapsed_time(b))
            cmp_ms.append(e.last_pass_ms()[0])
        return step_ms, cmp_ms

    def timed_stream(nsteps, slot_list):
        """Passes back to back as a client queues them (no host wait between
        passes); CUDA events around each pass and around the whole run."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(nsteps)]
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for a, b in evs:
            a.record(stream)
            e.match(slot_list, p.min_nr_spots, p.min_intensity)
            b.record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs], t0.elapsed_time(t1)

    timed(args.warmup, slots)
    timed_stream(args.warmup, slots)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    step_ms, total_ms = timed_stream(args.steps, slots)
    clk = clocks.stop()
    _, cmp_ms = timed(min(args.steps, 200), slots)  # compare-kernel times, synchronised
    if dist:
        tt = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dist.barrier()
        total_ms = float(tt.item())
    value = world * K * args.steps / (total_ms / 1e3)
    surv = [int(e.results(k)[0].shape[0]) for k in range(K)]
    shape_main, lay_main = e.get_tuning(), e.layout_info()  # the timed pass's shape

    # ---- plain pass (one image) --------------------------------------------
    timed_stream(args.warmup, [0])
    pstep, ptotal = timed_stream(args.steps, [0])
    plain_ips = args.steps / (ptotal / 1e3)
    _, pcmp = timed(min(args.steps, 200), [0])

    # ---- end to end through the public API from pinned host frames ----------
    pins = []
    for k in range(K):
        pb = PinnedBuffer((p.nr_px_x * p.nr_px_y,), np.uint8)
        pb.array[:] = imgs[k]
        pins.append(pb)
    d2h = [0]

    frames_all = [pb.array for pb in pins]
    phase = {"seq_load": [], "seq_match": [], "seq_collect": [], "pipe_load": [],
             "pipe_match": [], "pipe_collect": []}

    def e2e_step():
        t0 = time.perf_counter()
        e.load_images(slots, frames_all)
        t1 = time.perf_counter()
        e.match(slots, p.min_nr_spots, p.min_intensity)
        t2 = time.perf_counter()
        nb = sum(r.nbytes for r, _ in e.results_batch(slots).values())
        t3 = time.perf_counter()
        phase["seq_load"].append(t1 - t0)
        phase["seq_match"].append(t2 - t1)
        phase["seq_collect"].append(t3 - t2)
        d2h[0] = nb + (2 * 64 + 1) * 4

    # sequential: upload 64 frames, one pass, download
    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    seq_lat = []
    te = time.perf_counter()
    for _ in range(args.steps):
        ts = time.perf_counter()
        e2e_step()
        seq_lat.append((time.perf_counter() - ts) * 1e3)
    seq_ips = world * K * args.steps / (time.perf_counter() - te)

    # pipelined: two halves of 32 slots; the frames of one half upload (load
    # stream) while the pass over the other half runs
    halves = [slots[: K // 2], slots[K // 2:]] if K >= 2 else [slots, slots]
    fidx = [0]

    def load_half(h):
        e.load_images(halves[h], [pins[(fidx[0] + i) % K].array for i in range(len(halves[h]))])
        fidx[0] += len(halves[h])

    def collect(h):
        return sum(r.nbytes for r, _ in e.results_batch(halves[h]).values())

    def pipelined(npasses, lat=None):
        load_half(0)
        e.match(halves[0], p.min_nr_spots, p.min_intensity)
        t_prev = time.perf_counter()
        nb = 0
        for i in range(npasses):
            h = i % 2
            t0 = time.perf_counter()
            if i + 1 < npasses:
                # next half: host scan while pass h runs, then its pass queued
                # behind pass h so the device never waits for the host
                load_half(1 - h)
            t1 = time.perf_counter()
            if i + 1 < npasses:
                e.match(halves[1 - h], p.min_nr_spots, p.min_intensity)
            t2 = time.perf_counter()
            nb += collect(h)
            if lat is not None:
                phase["pipe_load"].append(t1 - t0)
                phase["pipe_match"].append(t2 - t1)
                phase["pipe_collect"].append(time.perf_counter() - t2)
                t = time.perf_counter()
                lat.append((t - t_prev) * 1e3)
                t_prev = t
        return nb

    pipelined(2 * args.warmup)
    torch.cuda.synchronize()
    lat = []
    moved0 = e.bytes_moved()
    te = time.perf_counter()
    nb = pipelined(2 * args.steps, lat)
    e2e_s = time.perf_counter() - te
    moved1 = e.bytes_moved()
    e2e_ips = world * len(halves[0]) * 2 * args.steps / e2e_s
    # bytes that crossed the host link per step of 64 frames, as counted by
    # the engine (sparse frames travel as (index, value) pairs)
    h2d_step = (moved1[0] - moved0[0]) // args.steps
    d2h[0] = (moved1[1] - moved0[1]) // args.steps
    # plain e2e: one frame per step
    platency = []
    for i in range(args.warmup + args.steps):
        ts = time.perf_counter()
        e.load_image(0, pins[i % K].array, want_scale=False)
        e.match([0], p.min_nr_spots, p.min_intensity)
        e.results(0)
        if i >= args.warmup:
            platency.append((time.perf_counter() - ts) * 1e3)

    # ---- end to end from the reference's own input types ----------------------
    # float32 wire frames (LaueMatchingGPUStream.cu:1201-1205) and float64 .bin
    # frames (LaueMatchingGPU.cu:704-715), page-locked, quantised on the way in:
    # the same pipelined two-half loop as above, the host scan and the uint8
    # quantisation inside the timed region
    e2e_types = {}
    for name, dt in (("float32_wire_frames", np.float32), ("float64_bin_frames", np.float64)):
        tp = []
        for k in range(K // 2 * 2 or 1):
            pb = PinnedBuffer((p.nr_px_x * p.nr_px_y,), dt)
            pb.array[:] = imgs[k % K]
            tp.append(pb)
        hv = [slots[: K // 2], slots[K // 2:]] if K >= 2 else [slots, slots]
        nx = [0]

        def load_t(h):
            e.load_images(hv[h], [tp[(nx[0] + i) % len(tp)].array for i in range(len(hv[h]))])
            nx[0] += len(hv[h])

        def loop(npasses):
            load_t(0)
            e.match(hv[0], p.min_nr_spots, p.min_intensity)
            for i in range(npasses):
                h = i % 2
                if i + 1 < npasses:
                    load_t(1 - h)
                    e.match(hv[1 - h], p.min_nr_spots, p.min_intensity)
                e.results_batch(hv[h])
        loop(2 * args.warmup)
        m0 = e.bytes_moved()
        t0 = time.perf_counter()
        loop(2 * args.steps)
        dt_s = time.perf_counter() - t0
        m1 = e.bytes_moved()
        e2e_types[name] = {"value": round(world * len(hv[0]) * 2 * args.steps / dt_s, 2),
                           "unit": UNIT, "h2d_bytes_per_step": (m1[0] - m0[0]) // args.steps,
                           "d2h_bytes_per_step": (m1[1] - m0[1]) // args.steps,
                           "frame_bytes": int(p.nr_px_x * p.nr_px_y * np.dtype(dt).itemsize)}
        for pb in tp:
            pb.free()
    # survivors of the float frames equal those of the uint8 frames they hold
    for k in range(K):
        e.load_image(k, imgs[k], want_scale=False)
    e.match(slots, p.min_nr_spots, p.min_intensity)
    ref_lists = {k: e.results(k) for k in slots}
    f32 = [imgs[k].astype(np.float32) for k in range(K)]
    e.load_images(slots, f32)
    e.match(slots, p.min_nr_spots, p.min_intensity)
    e2e_types["float_frames_same_survivors"] = same_survivors(
        {k: e.results(k) for k in slots}, ref_lists)

    # ---- K sweep: images/s of the resident batched pass, K = 1 .. 64 ----------
    k_sweep = []
    for kk in (1, 2, 4, 8, 16, 32, 64):
        if kk > K:
            break
        for k in range(kk):
            e.load_image(k, imgs[k], want_scale=False)
        sl = list(range(kk))
        timed_stream(args.warmup, sl)
        nk = max(10, min(args.steps, 200))
        _, tk = timed_stream(nk, sl)
        k_sweep.append({"K": kk, "images_per_s": round(kk * nk / (tk * 1e-3), 1),
                        "ms_per_pass": round(tk / nk, 4)})
    for k in range(K):
        e.load_image(k, imgs[k], want_scale=False)

    # ---- the same batched pass gathering every spot ----------------------------
    # (records with fewer spots than MinNrSpots are otherwise not gathered:
    # they cannot pass; the survivors are identical either way)
    e.set_tuning(**dict(shape_main, full_gather=1))
    for k in range(K):
        e.load_image(k, imgs[k], want_scale=False)
    timed(args.warmup, slots)
    fg_n = max(10, min(args.steps, 300))
    _, fg_total = timed_stream(fg_n, slots)
    _, fg_cmp = timed(min(fg_n, 50), slots)
    fg_surv = [int(e.results(k)[0].shape[0]) for k in range(K)]
    full_gather = {"value": round(K * fg_n / (fg_total * 1e-3), 2), "unit": UNIT,
                   "compare_ms": round(statistics.mean(fg_cmp), 4),
                   "same_survivor_counts": fg_surv == surv}

    merge = merge_timing(p.space_group, p.max_angle, dev) if rank == 0 else None
    refine = refine_timing(dev, cpu=not args.no_cpu_baseline) if rank == 0 else None
    prep = preprocess_timing(dev, parity=not args.no_parity,
                             cpu_port=not args.no_cpu_baseline) if rank == 0 else None
    if prep is not None:
        prep["raw_frames_to_survivors"] = raw_frame_pipeline(e, p, rec_head)

    # ---- roofline of the compare kernel ----------------------------------------
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    # Algorithmic bytes of one pass: the reference records (122 B per
    # orientation) plus the K uint8 frames; with the compact layout, the bytes
    # that layout streams (1 B per orientation + 4 B per on-detector spot +
    # tile headers) plus the occupancy words the gathers read (8 B per pixel).
    lay, shape = lay_main, shape_main
    compact = shape.get("last_variant") == 2 and lay["compact"] == 1
    ref_bytes = N * REC_BYTES_PER_ORIENT + K * p.nr_px_x * p.nr_px_y
    alg_bytes = lay["bytes"] + p.nr_px_x * p.nr_px_y * 8 if compact else ref_bytes
    cmp_avg = statistics.mean(cmp_ms)
    achieved = alg_bytes / (cmp_avg * 1e-3) / 1e9
    tpo = TRAFFIC_BYTES_PER_ORIENT.get("compact" if compact else "reference")
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src,
            "kernel": "compare_clist_kernel" if compact else "compare_ws_kernel",
            "layout": "compact" if compact else "reference",
            "algorithmic_bytes_per_launch": alg_bytes,
            "avg_launch_ms": round(cmp_avg, 4),
            "traffic": round(tpo * N) if tpo else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per orientation "
                              "of a smaller capture, scaled to N (see profiles/)" if tpo else None,
            "reference_layout_bytes_per_launch": ref_bytes,
            "reference_layout_equivalent_gbs": round(ref_bytes / (cmp_avg * 1e-3) / 1e9, 1),
            "tuning": shape}
    if compact:
        roof["compact_layout"] = lay

    out = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"batched DB pass: {K} uint8 2048x2048 frames (U{{1..20}} fcc "
                               f"grains each) vs a {N:,}-orientation device-resident DB",
                   "n_orient": N, "batch": K, "detector": [p.nr_px_x, p.nr_px_y],
                   "max_nr_spots": p.max_nr_spots, "record_bytes": REC_BYTES_PER_ORIENT,
                   "hkls": int(len(hkls)), "mean_spots_per_orientation": round(mean_spots, 3),
                   "min_nr_spots": p.min_nr_spots, "min_intensity": p.min_intensity,
                   "l2": "inputs larger than L2 (12.2 GB DB streamed every pass)",
                   "parallelism": f"replicas x{world} (images split, DB replicated)"},
        "roofline": roof,
        "e2e": dict(e2e_types["float32_wire_frames"],
                    path="public Engine API from page-locked float32 frames (the daemon's wire "
                         "frames, LaueMatchingGPUStream.cu:1201-1205), host scan and uint8 "
                         "quantisation inside the timed region: per step 64 frames in two "
                         "passes of 32, the upload of one half overlapping the pass of the other "
                         "and its pass queued before the other's results are read (load_images "
                         "of 32 frames, match, results_batch of the previous 32, twice)"),
        "e2e_uint8_frames": {
            "value": round(e2e_ips, 2), "unit": UNIT,
            "h2d_bytes_per_step": h2d_step,
            "h2d_dense_frame_bytes_per_step": K * p.nr_px_x * p.nr_px_y,
            "d2h_bytes_per_step": d2h[0],
            "path": "the same loop from page-locked uint8 frames (already quantised)",
            "sequential": round(seq_ips, 2),
            # host wall time per call, median: load_images (host scan + copy
            # enqueue), match (enqueue), results_batch (wait for the pass + copy)
            "breakdown_ms_p50": {k: round(1e3 * float(np.median(v)), 3)
                                 for k, v in phase.items() if v}},
        # per timed pass: status reset, compare, ordering (one graph replay)
        "gpu_launches": 3 * args.steps,
        "clocks": clk,
        "latency_ms": {"batched_p50": round(float(np.percentile(seq_lat, 50)), 3),
                       "batched_p99": round(float(np.percentile(seq_lat, 99)), 3),
                       "pipelined_pass_p50": round(float(np.percentile(lat, 50)), 3),
                       "pipelined_pass_p99": round(float(np.percentile(lat, 99)), 3),
                       "plain_p50": round(float(np.percentile(platency, 50)), 3),
                       "plain_p99": round(float(np.percentile(platency, 99)), 3)},
        "plain": {"value": round(plain_ips, 2), "unit": UNIT,
                  "e2e": round(1e3 / statistics.mean(platency), 2),
                  "compare_ms": round(statistics.mean(pcmp), 4)},
        "batched_over_plain": round(value / world / plain_ips, 2),
        "e2e_input_types": e2e_types,
        "k_sweep": k_sweep,
        "full_gather": full_gather,
        "merge": merge,
        "refine": refine,
        "preprocess": prep,
        "survivors_per_image": {"min": min(surv), "max": max(surv), "mean": statistics.mean(surv)},
        "dbbuild": {"orientations_per_s": round(N / t_build, 1), "seconds": round(t_build, 3),
                    "hkl_evals_per_s": round(N * len(hkls) / t_build, 1)},
    }
    if rank == 0 and world == 1 and not args.no_parity:
        out["dbbuild"]["parity"] = dbbuild_parity_sample(e, p, hkls, args.seed, N)
    def guarded(name, fn):
        """A leg that fails is reported in the line instead of ending the run."""
        try:
            return fn()
        except Exception as exc:  # noqa: BLE001
            import traceback
            log(traceback.format_exc())
            return {"failed": f"{type(exc).__name__}: {exc}"[:500]}

    if rank == 0 and world == 1 and not (args.no_parity and args.no_cpu_baseline):
        r = guarded("full_db", lambda: full_db_parity_and_cpu_baseline(
            e, p, txt, hkls, imgs[0], args.seed, cpu=not args.no_cpu_baseline,
            parity=not args.no_parity))
        out.update(r if "failed" not in r else {"full_db_parity": r})
    # the other configurations' legs (one GPU, rank 0 only)
    legs = [x for x in args.legs.split(",") if x] if rank == 0 and world == 1 else []
    if "tilted" in legs:
        out["tilted"] = guarded("tilted", lambda: tilted_leg(args, dev, K=K))
    if "hex" in legs:
        out["hex"] = guarded("hex", lambda: hex_leg(args, dev))
    if "volume" in legs:
        out["survivor_volume"] = guarded("volume", lambda: volume_leg(args, e, rec_head, dev))
    if "serve" in legs:
        out["serving"] = guarded("serve", lambda: serve_leg(args, e))
    for pb in pins:
        pb.free()
    e.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU executable on the box's host cores
# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lauematching_b200 import formats, synth
    if not O.have_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/LaueMatchingCPU was not built (reference sources absent "
                          "when the repository was built)"}))
        return
    txt, p = workload_params(args.min_intensity)
    hkls = synth.hkls_cubic(8)
    n_s = args.ref_sample
    cores = os.cpu_count() or 1
    base = scratch_dir(n_s * REC_BYTES_PER_ORIENT)
    wd = tempfile.mkdtemp(prefix="lmb_ref_", dir=base)
    # the orientation file stays off /dev/shm: with DoFwd 1 the reference
    # free()s a memory-mapped orientation file at exit (LaueMatchingCPU.c:825-830)
    wd_o = tempfile.mkdtemp(prefix="lmb_ref_o_")
    fwd = os.path.join(wd, "fwd.bin")
    om = synth.shoemake_orientations(n_s, seed=args.seed)
    op = os.path.join(wd_o, "orients.bin")
    formats.write_orientations(op, om)
    hp = os.path.join(wd, "hkls.csv")
    formats.write_hkls(hp, hkls)
    # the reference builds the sample's forward cache itself (DoFwd 1)
    ip = os.path.join(wd, "image.bin")
    formats.write_image_bin(ip, np.zeros(p.nr_px_x * p.nr_px_y))
    pp = os.path.join(wd, "params.txt")
    with open(pp, "w") as f:
        f.write(txt + f"ForwardFile {fwd}\nDoFwd 1\n")
    rb = O.run_reference(pp, op, hp, ip, ncpus=cores)
    if rb.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": "reference DoFwd 1 run failed: "
                          + (rb.stderr or rb.stdout)[-200:].replace("\n", " ")}))
        return
    rec = np.fromfile(fwd, np.uint16).reshape(n_s, 61)
    rng = np.random.default_rng(1000)
    imgs = []
    for _ in range(max(1, min(args.batch, 8))):
        g = synth.pick_grains(rec, int(rng.integers(1, 21)), p.min_nr_spots, rng)
        imgs.append(synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng))
    # the full-size DB: the reference-built sample repeated up to 1e8 records
    # (cache and orientation file alike), in /dev/shm when it has room so the
    # reference memory-maps both; every timed run compares against all of it
    tiles = max(1, args.n_orient // n_s)
    per = REC_BYTES_PER_ORIENT + 72
    big = scratch_dir(tiles * n_s * per)
    if big is None:
        import psutil
        tiles = max(1, min(tiles, int(psutil.virtual_memory().available * 0.4 // (n_s * per))))
    n = tiles * n_s
    wd_f = tempfile.mkdtemp(prefix="lmb_ref_full_", dir=big)
    fwd_f, op_f = os.path.join(wd_f, "fwd.bin"), os.path.join(wd_f, "orients.bin")
    rec_bytes = rec.tobytes()
    om_bytes = open(op, "rb").read()
    with open(fwd_f, "wb") as ff, open(op_f, "wb") as fo:
        for _ in range(tiles):
            ff.write(rec_bytes)
            fo.write(om_bytes)
    del rec_bytes, om_bytes
    with open(pp, "w") as f:
        f.write(txt + f"ForwardFile {fwd_f}\nDoFwd 0\n")
    times, walls, inits = [], [], []
    for i in range(args.warmup + args.steps):
        formats.write_image_bin(ip, imgs[i % len(imgs)])
        r = O.run_reference(pp, op_f, hp, ip, ncpus=cores)
        if r.returncode != 0 or r.compare_seconds is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference run failed: "
                              + (r.stderr or r.stdout)[-200:].replace("\n", " ")}))
            return
        if i >= args.warmup:
            times.append(r.compare_seconds)
            walls.append(r.wall_seconds)
            inits.append(r.initial_solutions)
    for d in (wd, wd_o, wd_f):
        for fn in os.listdir(d):
            os.remove(os.path.join(d, fn))
        os.rmdir(d)
    scale = 1e8 / n
    per_img = statistics.mean(times) * scale
    value = 1.0 / per_img
    sample = (f"LaueMatchingCPU (reference source, gcc -O3 -fopenmp, NLopt stand-in) DoFwd 0, "
              f"one image per run against {n:,} records (a {n_s:,}-orientation DB built by the "
              f"reference itself, DoFwd 1 in {rb.compare_seconds:.2f} s, repeated x{tiles}"
              f"{' in /dev/shm' if big else ''}): compare stage mean of {args.steps} runs = "
              f"{statistics.mean(times):.4f} s"
              + ("" if n == 100_000_000 else f", scaled x{scale:g} to 1e8")
              + f"; whole process {statistics.mean(walls):.2f} s per run")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(per_img * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
           "config": {"workload": f"plain single-image compare vs a {n:,}-record DB "
                                  f"(reference-built {n_s:,}-orientation DB x{tiles})",
                      "n_orient": n, "max_nr_spots": 30, "hkls": int(len(hkls))},
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores,
                            "kind": "reference", "sample": sample},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "process_wall_s_per_step": round(statistics.mean(walls), 3),
           "initial_solutions_per_image": inits,
           "dbbuild_reference": {"orientations_per_s": round(n_s / rb.compare_seconds, 1),
                                 "sample": n_s}}
    print(json.dumps(out), flush=True)


def _ref_gpu_sample_size(n_want):
    """Largest DB (<= n_want) whose files fit the host: the forward cache
    (122 B) and orientations (72 B) per orientation, held twice (page cache and
    the reference's own read buffer), within half the available RAM and the
    temporary directory's free space."""
    import psutil
    per = 2 * (REC_BYTES_PER_ORIENT + 72)
    ram = psutil.virtual_memory().available // 2
    st = os.statvfs(tempfile.gettempdir())
    disk = int(st.f_bavail * st.f_frsize * 0.8) // (REC_BYTES_PER_ORIENT + 72)
    return max(0, min(n_want, ram // per, disk))


def run_reference_gpu(args, rank, world):
    """The reference's plain single-image GPU path (LaueMatchingGPU.cu built
    for sm_100a): one process per image, each streaming the forward cache to
    the device in <= 4 GB chunks (LaueMatchingGPU.cu:660-749) and running its
    one-thread-per-orientation kernel (:45-81) on each chunk.  The device DB
    build writes the input cache (byte-identical to the reference's own
    DoFwd 1 cache); nothing of ours runs inside the reference process."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lauematching_b200 import formats, synth
    from lauematching_b200.engine import Engine
    if not O.have_ref_gpu():
        print(json.dumps({"impl": "reference-gpu", "unavailable":
                          "oracle/_ref/LaueMatchingGPU was not built (reference sources or nvcc "
                          "absent when the repository was built)"}))
        return
    txt, p = workload_params(args.min_intensity)
    hkls = synth.hkls_cubic(8)
    n = _ref_gpu_sample_size(args.n_orient)
    if n < 1_000_000:
        print(json.dumps({"impl": "reference-gpu", "unavailable":
                          f"host RAM/disk too small for the reference's input files ({n})"}))
        return
    e = Engine(p)
    e.build_db_synthetic(seed=args.seed, n=n, hkls=hkls)
    wd = tempfile.mkdtemp(prefix="lmb_refgpu_")
    fwd, op = os.path.join(wd, "fwd.bin"), os.path.join(wd, "orients.bin")
    step = 4_000_000
    with open(fwd, "wb") as ff, open(op, "wb") as fo:
        for s in range(0, n, step):
            c = min(step, n - s)
            e.download_db(s, c).tofile(ff)
            e.synth_orientations(args.seed, s, c).tofile(fo)
    hp, ip, pp = (os.path.join(wd, x) for x in ("hkls.csv", "image.bin", "params.txt"))
    formats.write_hkls(hp, hkls)
    rng = np.random.default_rng(2000)
    rec = e.download_db(0, min(2_000_000, n))
    img = synth.render_image(rec[synth.pick_grains(rec, 8, p.min_nr_spots, rng)],
                             p.nr_px_x, p.nr_px_y, rng)
    formats.write_image_bin(ip, img)
    with open(pp, "w") as f:
        f.write(txt + f"ForwardFile {fwd}\nDoFwd 0\n")
    e.load_image(0, img)
    e.match([0], p.min_nr_spots, p.min_intensity)
    n_pass_ours = e.results(0)[1]
    e.close()
    cores = os.cpu_count() or 1
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    warm, runs = min(args.warmup, 1), max(1, min(args.steps, 3))
    kern, match, walls, reads, chunks, nm = [], [], [], [], None, None
    for i in range(warm + runs):
        r = O.run_reference_gpu(pp, op, hp, ip, ncpus=cores, env=env)
        if r.returncode != 0 or not r.chunks:
            print(json.dumps({"impl": "reference-gpu", "unavailable": "reference GPU run failed: "
                              + (r.stderr or r.stdout)[-200:].replace("\n", " ")}))
            return
        if i >= warm:
            kern.append(sum(k for _, k in r.chunks))
            match.append(r.match_seconds)
            walls.append(r.wall_seconds)
            reads.append(r.read_seconds)
            chunks, nm = r.chunks, r.n_matches
    for fn in os.listdir(wd):
        os.remove(os.path.join(wd, fn))
    os.rmdir(wd)
    scale = 1e8 / n
    k_img = statistics.median(kern) * scale
    m_img = statistics.median(match) * scale
    out = {"impl": "reference-gpu", "metric": METRIC, "value": round(1.0 / k_img, 3),
           "unit": UNIT, "n_gpus": 1, "steps": runs, "warmup": warm,
           "ms_per_step": round(k_img * 1e3, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "plain single-image compare (reference LaueMatchingGPU, sm_100a "
                                  "build) vs a 100,000,000-orientation DB"
                                  + ("" if n == 100_000_000 else f" (sampled: {n})"),
                      "n_orient": n, "max_nr_spots": 30, "hkls": int(len(hkls)), "grains": 8},
           "e2e": {"value": round(1.0 / m_img, 4), "unit": UNIT,
                   "h2d_bytes_per_step": int(n * REC_BYTES_PER_ORIENT + p.nr_px_x * p.nr_px_y * 4),
                   "d2h_bytes_per_step": int((nm or 0) * 12 + 4)},
           "reference_gpu": {
               "build": "nvcc -O3 -w -rdc=true -gencode arch=compute_100a,code=sm_100a "
                        "-Xcompiler=-fopenmp (reference CMake flags, sm_100a target)",
               "kernel_s_per_image": round(k_img, 5),
               "match_stage_s_per_image": round(m_img, 4),
               "chunks_h2d_kernel_s": chunks, "forward_read_s": statistics.median(reads),
               "process_wall_s": round(statistics.median(walls), 2),
               "module_loading": "EAGER", "cores": cores,
               "nr_matches": nm, "n_pass_ours": n_pass_ours}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# serving: Poisson arrivals of mixed 1024^2 / 2048^2 frames through the daemon
# ---------------------------------------------------------------------------
def _serve_client(port, wire, keys, n_total, rate, nsend, plain, sent):
    """Poisson arrivals of frames on nsend connections.  plain: the
    reference's message (2-byte host-endian image number + the float32 frame
    of the daemon's detector); else the extended header (b"LMB2", image
    number, width, height, dtype 1 = uint8).  sent[i] = time.monotonic() just
    before image i+1 is sent.

    Each distinct frame is written once to a file in shared memory and sent
    with sendfile (no copy through this process), so the load generator's
    own copies do not cap the rate the daemons are offered."""
    import socket
    import struct
    import threading as th

    tmp = tempfile.mkdtemp(prefix="lmb_client_",
                           dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    fds = {}
    for key, frs in wire.items():
        for q, fr in enumerate(frs):
            fn = os.path.join(tmp, f"{key[0]}x{key[1]}_{q}.bin")
            with open(fn, "wb") as fh:
                fh.write(fr)
            fds[(key, q)] = (os.open(fn, os.O_RDONLY), len(fr))

    def send_frame(s, key, q):
        fd, size = fds[(key, q)]
        off = 0
        while off < size:
            off += os.sendfile(s.fileno(), fd, off, size - off)

    def sender(j):
        r2 = np.random.default_rng(100 + j)
        s = socket.create_connection(("127.0.0.1", port))
        t = time.perf_counter()
        for i in range(j, n_total, nsend):
            t += r2.exponential(nsend / rate)
            dt = t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            key = keys[int(r2.integers(0, len(keys)))]
            q = int(r2.integers(0, len(wire[key])))
            num = (i % 65535) + 1
            sent[i] = time.monotonic()
            # header and frame as two sends (no 16 MiB concatenation per message)
            if plain:
                s.sendall(num.to_bytes(2, sys.byteorder))
            else:
                s.sendall(struct.pack("<4sHHHBB", b"LMB2", num, key[0], key[1], 1, 0))
            send_frame(s, key, q)
        s.close()
    try:
        ts = [th.Thread(target=sender, args=(j,)) for j in range(nsend)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    finally:
        for fd, _ in fds.values():
            os.close(fd)
        shutil.rmtree(tmp, ignore_errors=True)


def _serve_run(port, wire, keys, n_total, rate, plain, done_at, nsend=4, wait_s=120.0):
    """One Poisson run from a client process; latency per image = the moment
    its results were written (done_at: image number -> time.monotonic()) minus
    the moment its message started to go out."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    sent = ctx.Array("d", n_total, lock=False)
    client = ctx.Process(target=_serve_client,
                         args=(port, wire, keys, n_total, rate, nsend, plain, sent))
    client.start()
    client.join()
    deadline = time.monotonic() + wait_s
    while len(done_at) < n_total and time.monotonic() < deadline:
        time.sleep(0.02)
    done = dict(done_at)
    lat = [done[(i % 65535) + 1] - sent[i] for i in range(n_total) if (i % 65535) + 1 in done]
    first = min(sent[:n_total])
    last = max(done.values()) if done else first
    lat_ms = np.array(lat) * 1e3 if lat else np.zeros(1)
    return {"offered_rate": rate, "sent": n_total, "served": len(lat),
            "throughput": round(len(lat) / max(last - first, 1e-9), 1),
            "p50_ms": round(float(np.percentile(lat_ms, 50)), 2),
            "p99_ms": round(float(np.percentile(lat_ms, 99)), 2)}


def serve_leg(args, e2=None):
    """Serving under Poisson arrivals against device-resident 1e8 DBs.

    * mixed: half 1024^2, half 2048^2 uint8 frames (1-30 fcc grains) on the
      extended port of this library's daemon (one DB per detector size), in
      its batched form (continuous batching, up to 64 images per pass) and
      one image per pass;
    * vs_reference: 2048^2 float32 frames in the reference's own message
      (2-byte image number + float32 frame) to this library's daemon and to
      the reference's LaueMatchingGPUStream (built for sm_100a from its
      sources; its DB, the device-built one byte-identical to its cache, read
      from its ForwardFile): the plain one-pass-per-image serving baseline.
    Latency = results written minus message start, per image."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lauematching_b200 import formats, synth, params as P
    from lauematching_b200.engine import Engine
    from lauematching_b200.stream import PINNED_BYTES, FramePool, StreamServer
    txt2, _ = workload_params(args.min_intensity)
    p2 = P.parse_params_text(txt2 + "MinGoodSpots 5\n", binary="stream")
    txt1 = txt2.replace("NrPxX 2048", "NrPxX 1024").replace("NrPxY 2048", "NrPxY 1024")
    txt1 = txt1.replace("PxX 0.0002", "PxX 0.0004").replace("PxY 0.0002", "PxY 0.0004")
    p1 = P.parse_params_text(txt1 + "MinGoodSpots 5\n", binary="stream")
    hkls = synth.hkls_cubic(8)
    N = args.n_orient
    own2 = e2 is None
    if own2:
        e2 = Engine(p2)
        e2.build_db_synthetic(args.seed, N, hkls)
    om = np.empty((N, 9), np.float64)
    for s0 in range(0, N, 4_000_000):
        c = min(4_000_000, N - s0)
        om[s0:s0 + c] = e2.synth_orientations(args.seed, s0, c)
    e1 = Engine(p1)
    e1.build_db_synthetic(args.seed, N, hkls)
    rng = np.random.default_rng(11)
    pool, pool_f32 = {}, []
    for e, p in ((e2, p2), (e1, p1)):
        rec = e.download_db(0, min(2_000_000, N))
        frames = []
        for _ in range(16):
            g = synth.pick_grains(rec, int(rng.integers(1, 31)), p.min_nr_spots, rng)
            frames.append(synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng))
        pool[(p.nr_px_x, p.nr_px_y)] = [f.astype(np.uint8).tobytes() for f in frames]
        if e is e2:
            pool_f32 = [f.astype(np.float32).tobytes() for f in frames]
    key2 = (p2.nr_px_x, p2.nr_px_y)
    out = {"n_orient": N, "mixed": [], "vs_reference": {"ours": [], "reference": []}}
    secs = args.serve_seconds

    def free_ports():
        """Two ports the kernel just handed out as free (fixed numbers can
        collide with the ephemeral ports of earlier connections)."""
        import socket
        socks = [socket.socket() for _ in range(2)]
        for sk in socks:
            sk.bind(("127.0.0.1", 0))
        ports = [sk.getsockname()[1] for sk in socks]
        for sk in socks:
            sk.close()
        return ports

    def ours(mode_batch, rates, keys, wire, plain, nsend=4):
        res = []
        for rate in rates:
            port0, port1 = free_ports()
            srv = StreamServer([p2, p1], om, hkls, ncpus=os.cpu_count() or 1,
                               max_batch=mode_batch, result_dir=tempfile.mkdtemp(prefix="lmb_sv_"),
                               port=port0, ext_port=port1, host="127.0.0.1",
                               log=lambda *a: None, engines=[e2, e1], max_queue=256,
                               frame_pool=frames).start()
            time.sleep(0.3)
            n_total = int(min(args.serve_images, max(50, rate * secs)))
            r = _serve_run(port0 if plain else port1, wire, keys, n_total, rate, plain,
                           srv.done_at, nsend=nsend)
            st = srv.stop(close_engines=False)
            r.update({"passes": st["passes"], "mean_batch": round(st["mean_batch"], 2)})
            res.append(r)
            log(json.dumps(r))
        return res

    # receive buffers kept across the daemon runs (page-locked up to the
    # daemon's budget: those frames go to the device over the copy engine)
    frames = FramePool(PINNED_BYTES)
    out["receive_buffers"] = {"page_locked_bytes": PINNED_BYTES, "dense_share": 1.0}
    rates = [float(r) for r in args.serve_rates.split(",")]
    keys = list(pool)
    for mode, mb in (("batched", 64), ("one_image_per_pass", 1)):
        for r in ours(mb, rates, keys, pool, plain=False):
            r["mode"] = mode
            out["mixed"].append(r)
    # same float32 2048^2 frames in the reference's message, both daemons
    ref_rates = [float(r) for r in args.serve_ref_rates.split(",")]
    wire32 = {key2: pool_f32}
    # 16 MiB frames: eight sending connections, so the client is not the limit
    out["vs_reference"]["ours"] = ours(64, ref_rates, [key2], wire32, plain=True, nsend=8)
    if O.have_ref_stream():
        per = REC_BYTES_PER_ORIENT + 72
        base = scratch_dir(N * per)
        wd = tempfile.mkdtemp(prefix="lmb_refstream_", dir=base)
        fwd, op = os.path.join(wd, "fwd.bin"), os.path.join(wd, "orients.bin")
        try:
            with open(fwd, "wb") as ff:
                for s0 in range(0, N, 4_000_000):
                    e2.download_db(s0, min(4_000_000, N - s0)).tofile(ff)
            om.tofile(op)
            hp, pp = os.path.join(wd, "hkls.csv"), os.path.join(wd, "params.txt")
            formats.write_hkls(hp, hkls)
            with open(pp, "w") as f:
                f.write(txt2 + f"ForwardFile {fwd}\nDoFwd 0\nResultDir results_ref\n"
                              f"MinGoodSpots 5\n")
            cores = os.cpu_count() or 1
            t0 = time.perf_counter()
            rs = O.RefStream(pp, op, hp, cores, cwd=wd)
            if not rs.wait_ready():
                out["vs_reference"]["reference"] = {
                    "unavailable": "the reference daemon did not start: "
                                   + "".join(rs.lines[-5:])[-300:]}
                rs.stop()
            else:
                t_ready = time.perf_counter() - t0
                for rate in ref_rates:
                    rs.done.clear()
                    # its saturated rate is ~150 images/s: at most 1500 frames per rate
                    n_total = int(min(args.serve_images, 1500, max(50, rate * secs)))
                    r = _serve_run(60517, wire32, [key2], n_total, rate, True, rs.done, nsend=8)
                    out["vs_reference"]["reference"].append(r)
                    log(json.dumps(dict(r, daemon="reference")))
                rc = rs.stop()
                out["vs_reference"]["reference_daemon"] = {
                    "binary": "oracle/_ref/LaueMatchingGPUStream (reference source, nvcc -O3 "
                              "-rdc=true sm_100a, NLopt stand-in)",
                    "startup_s": round(t_ready, 1), "exit_code": rc, "cores": cores}
        finally:
            for fn in ("fwd.bin", "orients.bin", "hkls.csv", "params.txt"):
                if os.path.exists(os.path.join(wd, fn)):
                    os.remove(os.path.join(wd, fn))
            import shutil
            shutil.rmtree(wd, ignore_errors=True)
    else:
        out["vs_reference"]["reference"] = {"unavailable": "oracle/_ref/LaueMatchingGPUStream "
                                                           "was not built"}
    sat = lambda lst: max((r["throughput"] for r in lst), default=0.0) \
        if isinstance(lst, list) else 0.0  # noqa: E731
    out["vs_reference"]["saturation_images_per_s"] = {
        "ours": sat(out["vs_reference"]["ours"]), "reference": sat(out["vs_reference"]["reference"])}
    frames.close()
    e1.close()
    if own2:
        e2.close()
    return out


def run_serve(args):
    print(json.dumps({"metric": "serving: images/s and p50/p99 image latency under Poisson "
                                "arrivals, 1e8-orientation DB per detector size",
                      "serving": serve_leg(args)}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours",
                    help="reference: the reference's CPU path; reference-gpu: its plain "
                         "single-image GPU executable built for sm_100a")
    ap.add_argument("--n-orient", type=int, default=100_000_000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--variant", type=int, default=None, choices=[0, 1, 2],
                    help="pin the compare variant (default: the autotuned shape)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--min-intensity", type=float, default=200.0)
    ap.add_argument("--ref-sample", type=int, default=2_000_000,
                    help="orientations per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--preprocess", action="store_true",
                    help="only the frame-preprocessing leg (2048^2 frames; --steps frames)")
    ap.add_argument("--refine", action="store_true",
                    help="only the batched refinement leg (device against host threads)")
    ap.add_argument("--serve", action="store_true", help="serving benchmark (Poisson arrivals)")
    ap.add_argument("--legs", type=str, default="tilted,hex,volume,serve",
                    help="legs of the other configurations run after the headline one "
                         "(comma list of tilted, hex, volume, serve; empty for none)")
    ap.add_argument("--leg", choices=["tilted", "hex", "dbbuild"], default=None,
                    help="only one leg of the bench: tilted = the batched pass at the "
                         "reference's tilted 34-ID-E detector (~15 spots per record); "
                         "hex = hexagonal fundamental-zone DB, 32 frames with c/a "
                         "perturbed, top-50 candidates into the c/a refinement; "
                         "dbbuild = the device DB build alone (cold and warm)")
    ap.add_argument("--serve-rates", type=str, default="10,100,500,2000")
    ap.add_argument("--serve-ref-rates", type=str, default="50,200,1000,4000")
    ap.add_argument("--serve-seconds", type=float, default=2.5)
    ap.add_argument("--serve-images", type=int, default=4000)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.impl == "reference-gpu":
        run_reference_gpu(args, rank, world)
    elif args.serve:
        run_serve(args)
    elif args.leg == "tilted":
        print(json.dumps(tilted_leg(args, 0, K=args.batch)), flush=True)
    elif args.leg == "hex":
        print(json.dumps(hex_leg(args, 0)), flush=True)
    elif args.leg == "dbbuild":
        print(json.dumps(dbbuild_leg(args, 0)), flush=True)
    elif args.refine:
        print(json.dumps(refine_timing(0, cpu=not args.no_cpu_baseline)), flush=True)
    elif args.preprocess:
        print(json.dumps(preprocess_timing(0, parity=not args.no_parity,
                                           cpu_port=not args.no_cpu_baseline,
                                           frames=max(1, min(args.steps, 200)))), flush=True)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
