"""Indexer drop-in: the reference's own checks (tests/test_indexer.py of
LaueMatching) plus the B200 selection and the fake-backend pattern of
tests/test_runimage_orchestration.py (a stand-in executable)."""
import os
import stat

from lauematching_b200.indexer import REPO_ROOT, resolve_executable, run_indexer


def test_resolve_executable_cpu_default():
    assert resolve_executable("/repo", "CPU", do_forward=False).endswith("bin/LaueMatchingCPU")


def test_resolve_executable_gpu():
    assert resolve_executable("/repo", "GPU", do_forward=False).endswith("bin/LaueMatchingGPU")


def test_resolve_executable_gpu_with_forward_falls_back_to_cpu():
    assert resolve_executable("/repo", "GPU", do_forward=True).endswith("bin/LaueMatchingCPU")


def test_resolve_executable_b200_builds_on_device():
    assert resolve_executable("/repo", "b200", do_forward=True).endswith("bin/LaueMatchingGPU")


def test_run_indexer_missing_binary():
    res = run_indexer(repo_root="/nonexistent_repo_xyz", config_file="c.txt",
                      orient_db_file="o.bin", hkl_file="h.csv", image_bin="i.bin",
                      ncpus=1, output_path="/tmp/_laue_test_out")
    assert res.success is False
    assert "not found" in (res.error or "")


def test_repository_ships_the_gpu_executable():
    exe = os.path.join(REPO_ROOT, "bin", "LaueMatchingGPU")
    assert os.path.exists(exe) and os.access(exe, os.X_OK)


def _fake_repo(tmp_path, rc):
    b = tmp_path / "bin"
    b.mkdir()
    exe = b / "LaueMatchingGPU"
    exe.write_text(f"#!/bin/sh\necho args:$#:$1:$5\necho oops 1>&2\nexit {rc}\n")
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_run_indexer_argv_logs_and_success(tmp_path):
    root = _fake_repo(tmp_path, 0)
    out = str(tmp_path / "img")
    res = run_indexer(repo_root=root, config_file="c.txt", orient_db_file="o.bin",
                      hkl_file="h.csv", image_bin="i.bin", ncpus=7, output_path=out,
                      compute_type="GPU")
    assert res.success and res.returncode == 0
    assert open(out + ".LaueMatching_stdout.txt").read().strip() == "args:5:c.txt:7"
    assert open(out + ".LaueMatching_stderr.txt").read().strip() == "oops"


def test_run_indexer_failure_code(tmp_path):
    root = _fake_repo(tmp_path, 3)
    res = run_indexer(repo_root=root, config_file="c.txt", orient_db_file="o.bin",
                      hkl_file="h.csv", image_bin="i.bin", ncpus=1,
                      output_path=str(tmp_path / "x"), compute_type="B200")
    assert not res.success and res.returncode == 3 and "code 3" in res.error
