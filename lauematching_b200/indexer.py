"""Indexer stage: drop-in for ``laue_index.indexer`` (laue_index/indexer.py:1-97).

Same names, keyword-only signature, argv contract, log files and result type
as the reference:

    <exe> <config.txt> <orientation_file> <hkls.csv> <blurred_image.bin> <ncpus>

with stdout/stderr saved to ``<output_path>.LaueMatching_std{out,err}.txt``
and success iff the exit code is 0.  Executable selection keeps the
reference's strings ("CPU", "GPU": ``bin/LaueMatchingGPU`` only without
DoFwd, laue_index/indexer.py:33-45) and adds ``"B200"``, which always picks
this repository's ``bin/LaueMatchingGPU`` because the B200 build simulates
the DB on the device (DoFwd 1 included).
"""
from __future__ import annotations

import logging
import os
import subprocess
from dataclasses import dataclass

logger = logging.getLogger("LaueMatching")

__all__ = ["IndexerResult", "resolve_executable", "run_indexer", "REPO_ROOT"]

REPO_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@dataclass
class IndexerResult:
    success: bool
    returncode: int | None = None
    stdout_log: str | None = None
    stderr_log: str | None = None
    error: str | None = None


def resolve_executable(repo_root: str, compute_type: str = "CPU",
                       do_forward: bool = False) -> str:
    """Pick the indexing executable path (<repo_root>/bin/<name>)."""
    compute_type = compute_type.upper()
    if compute_type == "B200" or (compute_type == "GPU" and not do_forward):
        name = "LaueMatchingGPU"
    else:
        name = "LaueMatchingCPU"
        if compute_type == "GPU" and do_forward:
            logger.warning("GPU requested but DoFwd is enabled. Using CPU implementation "
                           "(LaueMatchingCPU); use compute_type='B200' for the device DB build.")
        elif compute_type != "CPU":
            logger.warning(f"Processing type '{compute_type}' not recognized or incompatible. "
                           "Using CPU implementation.")
    return os.path.join(repo_root, "bin", name)


def _build_env(repo_root: str) -> dict:
    env = dict(os.environ)
    lib = os.path.join(repo_root, "LIBS", "NLOPT", "lib")
    lib64 = os.path.join(repo_root, "LIBS", "NLOPT", "lib64")
    env["LD_LIBRARY_PATH"] = f"{lib}:{lib64}:{env.get('LD_LIBRARY_PATH', '')}"
    return env


def run_indexer(*, repo_root: str, config_file: str, orient_db_file: str,
                hkl_file: str, image_bin: str, ncpus: int, output_path: str,
                compute_type: str = "CPU", do_forward: bool = False) -> IndexerResult:
    """Run the indexing executable on already-prepared inputs."""
    executable = resolve_executable(repo_root, compute_type, do_forward)
    if not os.path.exists(executable):
        logger.error(f"Indexing executable not found at: {executable}")
        return IndexerResult(success=False, error="Indexing executable not found")
    cmd = [executable, config_file, orient_db_file, hkl_file, image_bin, str(ncpus)]
    logger.info(f'Running indexing command: {" ".join(cmd)}')
    stdout_log = f"{output_path}.LaueMatching_stdout.txt"
    stderr_log = f"{output_path}.LaueMatching_stderr.txt"
    try:
        process = subprocess.run(cmd, env=_build_env(repo_root), capture_output=True,
                                 text=True, check=False)
        with open(stdout_log, "w") as f:
            f.write(process.stdout)
        with open(stderr_log, "w") as f:
            f.write(process.stderr)
        if process.returncode == 0:
            return IndexerResult(success=True, returncode=0, stdout_log=stdout_log,
                                 stderr_log=stderr_log)
        logger.error(f"Indexing command failed with exit code {process.returncode}.")
        return IndexerResult(success=False, returncode=process.returncode,
                             stdout_log=stdout_log, stderr_log=stderr_log,
                             error=f"Indexing command failed with code {process.returncode}")
    except FileNotFoundError:
        return IndexerResult(success=False, error="Indexing executable not found during execution")
    except Exception as e:  # noqa: BLE001 -- the reference's catch-all
        return IndexerResult(success=False, error=f"Unexpected error during indexing execution: {e}")
