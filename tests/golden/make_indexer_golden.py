"""Record how the reference's ``laue_index.indexer.run_indexer`` drives the
indexing executable, as a fixture for the drop-in tests.

The reference's Python stage (laue_index/indexer.py:33-97) is imported from the
reference tree named by ``--reference`` or ``LAUE_REFERENCE_ROOT`` and run
against a scratch ``repo_root`` whose ``bin/`` holds a recording stand-in:
the stand-in writes the argv, the LD_LIBRARY_PATH and the working directory
it was started with, prints one line on each stream and exits with a chosen
code.  Stored in ``indexer_invocation.json`` (paths relative to the scratch
repo root or the output path):

* which executable each (compute_type, do_forward) selects;
* the argv, the library path and the working directory of a run;
* the log files written, their contents, and the returned IndexerResult for
  exit codes 0 and 3, and for a repo root without the executable.

    python tests/golden/make_indexer_golden.py --reference <reference tree>

tests/test_indexer.py and tests/test_cli_gpu.py replay the GPU invocation
against this repository's ``bin/LaueMatchingGPU``.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import stat
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "indexer_invocation.json")

RECORDER = """#!/usr/bin/env python3
import json, os, sys
with open(os.environ["LMB_INDEXER_RECORD"], "w") as f:
    json.dump({"argv": sys.argv[1:], "ld_library_path": os.environ.get("LD_LIBRARY_PATH", ""),
               "cwd": os.getcwd()}, f)
print("recorded stdout line")
print("recorded stderr line", file=sys.stderr)
sys.exit(int(os.environ.get("LMB_INDEXER_EXIT", "0")))
"""


def _rel(path, root):
    return os.path.relpath(path, root) if path else path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LAUE_REFERENCE_ROOT"),
                    help="root of the reference tree (holds laue_index/)")
    args = ap.parse_args()
    if not args.reference or not os.path.isdir(os.path.join(args.reference, "laue_index")):
        sys.exit("give the reference tree with --reference or LAUE_REFERENCE_ROOT")
    sys.path.insert(0, args.reference)
    from laue_index import indexer as ref  # the reference's own module

    out = {"generator": "tests/golden/make_indexer_golden.py",
           "source": "laue_index/indexer.py (the reference's run_indexer and resolve_executable)"}
    with tempfile.TemporaryDirectory() as td:
        root = os.path.join(td, "repo")
        os.makedirs(os.path.join(root, "bin"))
        out["resolve"] = [
            {"compute_type": ct, "do_forward": fw,
             "executable": _rel(ref.resolve_executable(root, ct, fw), root)}
            for ct in ("CPU", "GPU", "gpu", "B200") for fw in (False, True)]
        # missing executable
        res = ref.run_indexer(repo_root=root, config_file="params.txt",
                              orient_db_file="orients.bin", hkl_file="hkls.csv",
                              image_bin="image.bin", ncpus=4,
                              output_path=os.path.join(td, "out", "image.bin"),
                              compute_type="GPU")
        out["missing_executable"] = dataclasses.asdict(res)
        exe = os.path.join(root, "bin", "LaueMatchingGPU")
        with open(exe, "w") as f:
            f.write(RECORDER)
        os.chmod(exe, os.stat(exe).st_mode | stat.S_IEXEC)
        work = os.path.join(td, "work")
        os.makedirs(os.path.join(td, "out"))
        os.makedirs(work)
        runs = []
        cwd0 = os.getcwd()
        os.chdir(work)
        try:
            for code in (0, 3):
                rec_path = os.path.join(td, f"record{code}.json")
                os.environ["LMB_INDEXER_RECORD"] = rec_path
                os.environ["LMB_INDEXER_EXIT"] = str(code)
                os.environ["LD_LIBRARY_PATH"] = "/caller/lib"
                outp = os.path.join(td, "out", "image.bin")
                res = ref.run_indexer(repo_root=root, config_file="params.txt",
                                      orient_db_file="orients.bin", hkl_file="hkls.csv",
                                      image_bin="image.bin", ncpus=4, output_path=outp,
                                      compute_type="GPU", do_forward=False)
                with open(rec_path) as f:
                    rec = json.load(f)
                d = dataclasses.asdict(res)
                logs = {}
                for key in ("stdout_log", "stderr_log"):
                    if d[key]:
                        with open(d[key]) as f:
                            logs[key] = f.read()
                        d[key] = d[key][len(outp):]  # suffix appended to output_path
                runs.append({
                    "exit_code": code,
                    "call": {"config_file": "params.txt", "orient_db_file": "orients.bin",
                             "hkl_file": "hkls.csv", "image_bin": "image.bin", "ncpus": 4},
                    "argv": rec["argv"],
                    "ld_library_path": [p if p == "/caller/lib" or not p else _rel(p, root)
                                        for p in rec["ld_library_path"].split(":")],
                    "cwd_is_callers": os.path.realpath(rec["cwd"]) == os.path.realpath(work),
                    "result": d, "logs": logs})
        finally:
            os.chdir(cwd0)
        out["gpu_runs"] = runs
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
