"""The ``laue_index.indexer`` boundary (laue_index/indexer.py:33-97).

The reference's own ``run_indexer(repo_root=<this repository>,
compute_type="GPU")`` runs ``<repo_root>/bin/LaueMatchingGPU`` with the 5-arg
command line; this repository ships that executable, so the reference's
stage drives it unchanged.  How the reference's function selects and calls the
executable is pinned by ``tests/golden/indexer_invocation.json``, recorded by
``tests/golden/make_indexer_golden.py`` from the reference's module itself.
These CPU tests check this repository's side of that contract; the GPU replay
with byte comparison of the outputs is in test_cli_gpu.py.
"""
import json
import os
import subprocess
import sys

from conftest import ROOT

FIXTURE = os.path.join(ROOT, "tests", "golden", "indexer_invocation.json")


def _fixture():
    with open(FIXTURE) as f:
        return json.load(f)


def test_reference_selection_finds_this_repositorys_gpu_executable():
    fx = _fixture()
    sel = {(r["compute_type"], r["do_forward"]): r["executable"] for r in fx["resolve"]}
    assert sel[("GPU", False)] == os.path.join("bin", "LaueMatchingGPU")
    assert sel[("gpu", False)] == os.path.join("bin", "LaueMatchingGPU")
    exe = os.path.join(ROOT, sel[("GPU", False)])
    assert os.path.isfile(exe) and os.access(exe, os.X_OK)
    # DoFwd runs and other compute types go to the reference's CPU executable
    assert sel[("GPU", True)] == sel[("CPU", False)] == os.path.join("bin", "LaueMatchingCPU")
    assert sel[("B200", False)] == os.path.join("bin", "LaueMatchingCPU")


def test_recorded_command_line_is_the_five_argument_contract():
    fx = _fixture()
    for run in fx["gpu_runs"]:
        c = run["call"]
        assert run["argv"] == [c["config_file"], c["orient_db_file"], c["hkl_file"],
                               c["image_bin"], str(c["ncpus"])]
        assert run["cwd_is_callers"]
        assert run["result"]["stdout_log"] == ".LaueMatching_stdout.txt"
        assert run["result"]["stderr_log"] == ".LaueMatching_stderr.txt"
        assert run["result"]["success"] == (run["exit_code"] == 0)
        assert run["result"]["returncode"] == run["exit_code"]
        assert run["logs"]["stdout_log"].startswith("recorded stdout")
    assert fx["missing_executable"]["success"] is False


def test_gpu_executable_argument_errors_without_a_device(tmp_path):
    """LaueMatchingGPU.cu:107-111: a wrong argument count prints the usage and
    exits 0; an unreadable parameter file exits 1 before any device use."""
    exe = os.path.join(ROOT, "bin", "LaueMatchingGPU")
    r = subprocess.run([sys.executable, exe, "a", "b"], capture_output=True, text=True)
    assert r.returncode == 0 and "Arguments" in r.stdout
    run = _fixture()["gpu_runs"][0]
    argv = [str(tmp_path / a) if a != str(run["call"]["ncpus"]) else a for a in run["argv"]]
    r = subprocess.run([sys.executable, exe, *argv], capture_output=True, text=True,
                       cwd=str(tmp_path))
    assert r.returncode == 1 and "Could not open parameter file" in r.stdout
