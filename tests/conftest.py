"""Shared test set-up.

* marker ``gpu``: needs a CUDA device and the built liblmb200.so;
* the oracle (oracle/, test infrastructure) is importable as ``oracle``;
* golden cases (tests/golden/*.npz, produced by the reference itself) are
  loaded through :func:`golden_case`.
"""
from __future__ import annotations

import glob
import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liblmb200.so")


class GoldenCase:
    def __init__(self, path):
        from lauematching_b200 import params as P, synth
        z = np.load(path, allow_pickle=False)
        self.name = os.path.splitext(os.path.basename(path))[0]
        self.params_text = str(z["params_text"])
        self.params = P.parse_params_text(self.params_text)
        self.seed = int(z["seed"])
        self.n = int(z["n"])
        self.orients = synth.shoemake_orientations(self.n, seed=self.seed)
        sha = hashlib.sha256(self.orients.tobytes()).hexdigest()
        assert sha == str(z["orients_sha256"]), (
            f"{self.name}: regenerated orientations differ from the golden ones")
        self.hkls = z["hkls"]
        self.img_u8 = z["img_u8"]
        self.img_scale = float(z["img_scale"])
        self.image = self.img_u8.astype(np.float64) * self.img_scale
        self.records = z["records"]
        self.meta = json.loads(str(z["meta"]))
        self.fwd_solutions = str(z["fwd_solutions"])
        self.fwd_spots = str(z["fwd_spots"])
        self.cmp_solutions = str(z["cmp_solutions"])
        self.cmp_spots = str(z["cmp_spots"])


_CACHE = {}


def golden_names():
    """Matching-path cases (the pp_*.npz files are preprocessing fixtures)."""
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("pp_"))


def golden_case(name) -> GoldenCase:
    if name not in _CACHE:
        _CACHE[name] = GoldenCase(os.path.join(GOLDEN, name + ".npz"))
    return _CACHE[name]


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch  # noqa: F401
        return torch.cuda.is_available()
    except Exception:
        return False
