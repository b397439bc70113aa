"""B200-native orientation matching for LaueMatching.

The hot path of LaueMatching (compare pass over the forward-simulated
orientation DB, the DB build, the batched pass and serving) as hand-written
sm_100a CUDA kernels behind a C ABI (include/lmb200.h, liblmb200.so), with
host code mirroring the reference's interfaces: the params/orientation/HKL/
forward-cache/image formats, the ``LaueMatchingGPU`` command line (which the
reference's own ``laue_index.indexer.run_indexer`` runs from ``bin/``) and
the ``LaueMatchingGPUStream`` daemon.
"""
from .params import LaueParams, read_params, parse_params_text  # noqa: F401

__version__ = "0.1.0"
