"""``LaueMatchingGPU`` command line, drop-in for the reference executable.

    LaueMatchingGPU <params.txt> <orientations.bin> <hkls.csv> <image.bin> <nCPUs>

Contract of LaueMatchingGPU.cu:107-111 / LaueMatchingCPU.c:48-52: a wrong
argument count prints the usage and exits 0; fatal input errors exit 1; the
results go to ``<image.bin>.solutions.txt`` and ``<image.bin>.spots.txt``.

* ``DoFwd 0`` with an existing ``ForwardFile``: the cache is uploaded to the
  device and compared against the uint8-quantised image (the reference CPU
  path, LaueMatchingCPU.c:668-690).
* ``DoFwd 1``, or a missing ``ForwardFile`` (LaueMatchingCPU.c:422-438): the
  DB is forward-simulated on the device, written to ``ForwardFile``, and
  compared against the float64 image, as the reference does in that mode
  (LaueMatchingCPU.c:649-653).

Survivors are handed to the post-stage in ascending ID, then merged, refined
and written (LaueMatchingCPU.c:735-811).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

USAGE = """LaueMatching on the GPU (B200)
Arguments:
* \tparameterFile (text)
* \tbinary files for candidate orientation list [double]
* \ttext of valid_hkls (preferably sorted on f2), space separated
* \tbinary file for image [double]
* \tnumber of CPU cores to use:

Parameter file with the following parameters:
\t\t* LatticeParameter (in nm and degrees),
\t\t* tol_latC (in %, 6 values),
\t\t* tol_c_over_a (in %, 1 value),
\t\t* SpaceGroup,
\t\t* P_Array, R_Array, PxX, PxY, NrPxX, NrPxY,
\t\t* Elo, Ehi, MaxNrLaueSpots, ForwardFile, DoFwd,
\t\t* MinNrSpots, MinIntensity, MaxAngle.
"""


def _device() -> int:
    return int(os.environ.get("LMB_DEVICE", "0"))


def main_gpu(argv=None) -> int:
    argv = sys.argv if argv is None else argv
    if len(argv) != 6:
        print(USAGE)
        return 0
    from . import formats, post
    from .engine import Engine
    from .params import ParamsError, read_params

    param_fn, orient_fn, hkl_fn, image_fn, ncpu_s = argv[1:6]
    t_start = time.perf_counter()
    print("Reading parameter file", flush=True)
    if not os.path.exists(param_fn):
        print(f"Could not open parameter file {param_fn}.")
        return 1
    try:
        p = read_params(param_fn, binary="gpu")
    except ParamsError as exc:
        print(str(exc), file=sys.stderr)
        return 1
    print("Parameters read", flush=True)
    try:
        ncpus = int(ncpu_s)
    except ValueError:
        ncpus = 0
    if ncpus < 1:
        print(f"FATAL: invalid thread count '{ncpu_s}' (need >= 1).", file=sys.stderr)
        return 1
    if not os.path.exists(orient_fn):
        print("Could not read orientation file, exiting.")
        return 1
    orients = formats.read_orientations(orient_fn)
    n = orients.shape[0]
    print(f"{n} Orientations read, took {time.perf_counter() - t_start:f} seconds, now reading hkls",
          flush=True)
    if not os.path.exists(hkl_fn):
        print(f"Could not read hkl file {hkl_fn}.")
        return 1
    hkls = formats.read_hkls(hkl_fn)
    print(f"{len(hkls)} hkls read. \nNow reading image file {image_fn}, number of pixels "
          f"{p.nr_px_x * p.nr_px_y}. \nminNrSpots: {p.min_nr_spots}, MinIntensity: "
          f"{int(p.min_intensity)}", flush=True)
    if not os.path.exists(image_fn):
        print(f"Could not read image file {image_fn}.")
        return 1
    try:
        image = formats.read_image_bin(image_fn, p.nr_px_x, p.nr_px_y)
    except ValueError as exc:
        print(str(exc))
        return 1
    print(f"Pixels with intensity: {int(np.count_nonzero(image > 0))}", flush=True)

    do_fwd = p.do_fwd
    fwd = p.forward_file
    if do_fwd == 0:
        print(f"Trying to see if the forward simulation exists. Looking for {fwd} file.")
        if not fwd or not os.path.exists(fwd):
            print("Could not read the forward simulation file. Running in simulation mode!")
            do_fwd = 1
        else:
            print(f"{fwd} file was found. Will not do forward simulation.")
    else:
        print(f"Forward simulation was requested, will be saved to {fwd}.")

    t0 = time.perf_counter()
    with Engine(p, device=_device()) as e:
        if do_fwd == 1:
            e.build_db(orients, hkls)
            if fwd:
                _write_cache(e, fwd, n)
            mode = 1
        else:
            rec = formats.read_forward_cache(fwd, n, p.max_nr_spots)
            e.upload_db(rec)
            mode = 0
        e.load_image(0, image, keep_f64=(mode == 1))
        e.match([0], p.min_nr_spots, p.min_intensity, value_mode=mode)
        surv, n_pass = e.results(0)
    t_cmp = time.perf_counter() - t0
    print(f"Finished comparing, time elapsed after comparing with forward simulation: "
          f"{t_cmp:f} seconds.\nSearching for unique solutions.", flush=True)

    ids, scores = post.collected_matches(surv, n_pass)
    sol, spt, n_unique = post.post_process(p, e.geometry, orients, ids, scores,
                                           image.astype(np.float32), hkls, num_threads=ncpus,
                                           merge_device=_device())
    try:
        with open(image_fn + ".solutions.txt", "w") as f:
            f.write(post.SOLUTIONS_HEADER + sol)
        with open(image_fn + ".spots.txt", "w") as f:
            f.write(post.SPOTS_HEADER + spt)
    except OSError:
        print("Could not open file for writing solutions. Exiting.")
        return 1
    t_all = time.perf_counter() - t0
    print(f"Finished, time elapsed in fitting: {t_all - t_cmp:f} seconds.\n"
          f"Initial solutions: {n_pass} Unique Orientations: {n_unique}\n"
          f"Total time: {time.perf_counter() - t_start:f} seconds.", flush=True)
    return 0


def _write_cache(e, path, n, chunk=4_000_000):
    """Write the device-built DB as the reference's ForwardFile (same bytes as
    LaueMatchingCPU.c:694-711 writes)."""
    from . import formats
    fd = os.open(path, os.O_CREAT | os.O_WRONLY, 0o600)
    os.close(fd)
    for off in range(0, n, chunk):
        cnt = min(chunk, n - off)
        formats.write_forward_cache(path, e.download_db(off, cnt), offset_records=off)
    fd = os.open(path, os.O_WRONLY)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)


if __name__ == "__main__":
    sys.exit(main_gpu())
