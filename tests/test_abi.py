"""The C ABI library loads and exports every entry point its header declares.

No compute call is made here (no GPU is needed).
"""
import ctypes as C
import os
import re

from conftest import ROOT
from lauematching_b200 import _lib

HEADER = os.path.join(ROOT, "include", "lmb200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"#define[^\n]*", "", txt)
    return sorted(set(re.findall(r"\b(lmb_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_the_binding_list():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_binding_loads_and_reports_version():
    L = _lib.lib()
    assert L.lmb_version().decode().startswith("lmb200")


def test_struct_layouts_match_header():
    assert C.sizeof(_lib.LmbSurvivor) == 32
    # 9+9+3 doubles, 4 doubles, 4 int32
    assert C.sizeof(_lib.LmbGeometry) == (21 + 4) * 8 + 4 * 4
    assert C.sizeof(_lib.LmbPreParams) == 2 * 4 + 3 * 8
    assert C.sizeof(_lib.LmbPreCounts) == 2 * 8 + 2 * 4


def test_geometry_is_bitwise_the_oracle_geometry():
    """lmb_geometry_init is host code: no GPU needed.  It must reproduce the
    reference's detector rotation and reciprocal basis bit for bit."""
    import numpy as np
    import oracle as O
    from lauematching_b200.engine import geometry_from_params
    from lauematching_b200 import synth, params as P
    for kw in [dict(), dict(r=(-1.20131258, -1.21399082, -1.21881158)),
               dict(lattice=(0.295, 0.295, 0.468, 90, 90, 120), space_group=194),
               dict(lattice=(0.45, 0.45, 0.45, 58, 58, 58), space_group=166)]:
        p = P.parse_params_text(synth.params_text(**kw))
        g = geometry_from_params(p)
        rt, rc = O.geometry(p)
        assert np.array_equal(np.array(g.rot_t[:]), rt)
        assert np.array_equal(np.array(g.recip[:]), rc)
