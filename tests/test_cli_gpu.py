"""The drop-in ``bin/LaueMatchingGPU`` executable, end to end on the GPU,
against the reference's own output files for the same inputs.

DoFwd 0: the golden forward cache is read, compared on the uint8 image.
DoFwd 1: the DB is simulated on the device and written as ForwardFile (must
equal the reference's cache), then compared on the float64 image.
Both runs must write solutions.txt / spots.txt identical to the reference's.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, golden_case
from lauematching_b200 import formats

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "bin", "LaueMatchingGPU")


def _case_files(c, tmp_path, do_fwd):
    fwd = str(tmp_path / "fwd.bin")
    txt = c.params_text
    lines = [ln for ln in txt.splitlines() if not ln.startswith(("ForwardFile", "DoFwd"))]
    lines += [f"ForwardFile {fwd}", f"DoFwd {do_fwd}"]
    pp = str(tmp_path / "params.txt")
    with open(pp, "w") as f:
        f.write("\n".join(lines) + "\n")
    op = str(tmp_path / "orients.bin")
    formats.write_orientations(op, c.orients)
    hp = str(tmp_path / "hkls.csv")
    formats.write_hkls(hp, c.hkls)
    ip = str(tmp_path / "image.bin")
    formats.write_image_bin(ip, c.image)
    if do_fwd == 0:
        c.records.tofile(fwd)
    return pp, op, hp, ip, fwd


@pytest.mark.parametrize("name", ["tilted_fcc", "tilted_dense", "tilted_scaled", "tilted_hex"])
@pytest.mark.parametrize("do_fwd", [0, 1])
def test_cli_writes_reference_files(name, do_fwd, tmp_path):
    c = golden_case(name)
    pp, op, hp, ip, fwd = _case_files(c, tmp_path, do_fwd)
    r = subprocess.run([sys.executable, EXE, pp, op, hp, ip, "4"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    key = "cmp" if do_fwd == 0 else "fwd"
    assert f"Initial solutions: {c.meta[key + '_initial']} " in r.stdout
    assert open(ip + ".solutions.txt").read() == (c.cmp_solutions if do_fwd == 0 else c.fwd_solutions)
    assert open(ip + ".spots.txt").read() == (c.cmp_spots if do_fwd == 0 else c.fwd_spots)
    if do_fwd == 1:
        assert np.array_equal(np.fromfile(fwd, np.uint16).reshape(c.records.shape), c.records)


def test_cli_usage_and_fatal_errors(tmp_path):
    r = subprocess.run([sys.executable, EXE, "a", "b"], capture_output=True, text=True)
    assert r.returncode == 0 and "Arguments" in r.stdout
    r = subprocess.run([sys.executable, EXE, str(tmp_path / "nope.txt"), "o", "h", "i", "1"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Could not open parameter file" in r.stdout


def test_cli_nelder_mead_writes_the_refined_solutions(tmp_path):
    """"Optimizer NelderMead" in the parameter file: the CLI's solutions.txt is
    the post-stage's Nelder-Mead text for the oracle's survivors (not the
    evaluate-once text of the reference built without NLopt)."""
    import oracle as O
    from lauematching_b200 import post
    from lauematching_b200.engine import geometry_from_params
    c = golden_case("tilted_dense")
    pp, op, hp, ip, fwd = _case_files(c, tmp_path, 0)
    with open(pp, "a") as f:
        f.write("Optimizer NelderMead\n")
    r = subprocess.run([sys.executable, EXE, pp, op, hp, ip, "4"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    p = c.params
    s = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity)
    surv = np.zeros(len(s.ids), [("id", "<u8"), ("score", "<f8")])
    surv["id"] = s.ids
    surv["score"] = s.score
    ids, sc = post.collected_matches(surv, s.n_pass)
    sol, _, _ = post.post_process(p, geometry_from_params(p), c.orients, ids, sc,
                                  c.image.astype(np.float32), c.hkls, optimizer="nelder-mead")
    got = open(ip + ".solutions.txt").read()
    assert got == post.SOLUTIONS_HEADER + sol
    assert got != c.cmp_solutions


def test_reference_indexer_invocation_writes_reference_files(tmp_path):
    """The invocation the reference's laue_index.indexer.run_indexer makes for
    compute_type="GPU" (recorded from the reference's module in
    tests/golden/indexer_invocation.json: the selected executable, argv,
    LD_LIBRARY_PATH, the caller's working directory, stdout/stderr into
    <output_path>.LaueMatching_std{out,err}.txt), replayed against this
    repository on a golden case: exit 0 (the reference's success), and
    solutions/spots byte-equal to the reference binary's files."""
    import json
    with open(os.path.join(ROOT, "tests", "golden", "indexer_invocation.json")) as f:
        fx = json.load(f)
    sel = {(r["compute_type"], r["do_forward"]): r["executable"] for r in fx["resolve"]}
    run = [r for r in fx["gpu_runs"] if r["exit_code"] == 0][0]
    c = golden_case("tilted_fcc")
    pp, op, hp, ip, _ = _case_files(c, tmp_path, 0)
    call = run["call"]
    actual = {call["config_file"]: pp, call["orient_db_file"]: op, call["hkl_file"]: hp,
              call["image_bin"]: ip, str(call["ncpus"]): "4"}
    exe = os.path.join(ROOT, sel[("GPU", False)])
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = ":".join(
        os.path.join(ROOT, p) if p and not p.startswith("/") else env.get("LD_LIBRARY_PATH", "")
        for p in run["ld_library_path"])
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([exe] + [actual[a] for a in run["argv"]], env=env, cwd=str(work),
                       capture_output=True, text=True)
    outp = str(tmp_path / "image.bin")
    with open(outp + run["result"]["stdout_log"], "w") as f:
        f.write(r.stdout)
    with open(outp + run["result"]["stderr_log"], "w") as f:
        f.write(r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr  # run_indexer's success
    assert f"Initial solutions: {c.meta['cmp_initial']} " in r.stdout
    assert open(ip + ".solutions.txt").read() == c.cmp_solutions
    assert open(ip + ".spots.txt").read() == c.cmp_spots
