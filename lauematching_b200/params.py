"""Parameter-file reader with the reference executables' exact semantics.

The reference parses its params text with a chain of ``strncmp`` prefix tests
(LaueMatchingCPU.c:75-204, LaueMatchingGPU.cu:132-259,
LaueMatchingGPUStream.cu:576-715):

* a line is tested against the keys in a fixed order and the FIRST key that
  is a prefix of the line wins; the rest of the chain is skipped;
* values are read with ``sscanf("%s %lf ...")``: the first token is
  discarded, then each conversion takes the longest valid numeric prefix and
  scanning stops at the first conversion that fails (values not read keep
  their previous value);
* unknown keys are ignored, so ``#`` comments after values are harmless;
* lines are read with ``fgets`` into a 1000-byte buffer, so a physical line
  longer than 999 bytes is seen as several lines.

Defaults differ per executable and are reproduced by :func:`read_params`
(``binary`` = ``"cpu"``, ``"gpu"`` or ``"stream"``).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

__all__ = ["LaueParams", "read_params", "parse_params_text", "ParamsError"]


class ParamsError(ValueError):
    """Raised for the fatal checks the reference performs after parsing
    (LaueMatchingCPU.c:210-220)."""


@dataclass
class LaueParams:
    lattice: list = field(default_factory=lambda: [0.0] * 6)  # nm, degrees
    p_array: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    r_array: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    tol_c_over_a: float = 0.0
    px_x: float = 0.0
    px_y: float = 0.0
    elo: float = 5.0
    ehi: float = 30.0
    do_fwd: int = 1
    nr_px_x: int = 0
    nr_px_y: int = 0
    max_nr_spots: int = 500
    batch_size: int = 1000000
    min_nr_spots: int = 5
    space_group: int = 225
    min_intensity: float = 1000.0
    max_angle: float = 2.0
    forward_file: str = ""
    tol_latc: list = field(default_factory=lambda: [0.0] * 6)
    optimizer: str = "BOBYQA"
    result_dir: str = "results_stream"
    min_good_spots: int = 5
    extra: dict = field(default_factory=dict)  # keys this reader does not use

    @property
    def c_over_a(self) -> float:
        return self.lattice[2] / self.lattice[0] if self.lattice[0] else math.nan


# C-like numeric prefix scanners (sscanf %d / %lf after whitespace skip).
_INT_RE = re.compile(rb"[ \t\n\v\f\r]*([+-]?[0-9]+)")
_FLT_RE = re.compile(
    rb"[ \t\n\v\f\r]*([+-]?(?:(?:inf(?:inity)?|nan(?:\([0-9A-Za-z_]*\))?)|"
    rb"(?:0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)(?:[pP][+-]?[0-9]+)?)|"
    rb"(?:(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?)))",
    re.IGNORECASE)
_TOK_RE = re.compile(rb"[ \t\n\v\f\r]*([^ \t\n\v\f\r]+)")


def _c_int(v: int) -> int:
    """sscanf %d stores into an int: wrap like a 32-bit store."""
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= (1 << 31) else v


def _scan(line: bytes, fmt: str):
    """Emulate sscanf(line, "%s" + fmt...) returning the list of converted
    values after the dummy %s (stops at the first failing conversion)."""
    m = _TOK_RE.match(line)
    if not m:
        return []
    pos = m.end()
    out = []
    for c in fmt:
        if c == "s":
            m = _TOK_RE.match(line, pos)
            if not m:
                break
            out.append(m.group(1).decode("latin-1"))
        elif c == "d":
            m = _INT_RE.match(line, pos)
            if not m:
                break
            out.append(_c_int(int(m.group(1))))
        elif c == "z":  # %zu
            m = _INT_RE.match(line, pos)
            if not m:
                break
            out.append(int(m.group(1)) & 0xFFFFFFFFFFFFFFFF)
        elif c == "f":
            m = _FLT_RE.match(line, pos)
            if not m:
                break
            txt = m.group(1).decode("ascii").lower()
            if txt.lstrip("+-").startswith("nan"):
                val = math.nan
            elif "x" in txt:
                val = float.fromhex(txt)
            else:
                val = float(txt)
            out.append(val)
        pos = m.end()
    return out


# (key, conversions, setter) in the reference's code order.
def _set_list(attr, n):
    def f(p, vals):
        lst = getattr(p, attr)
        for i, v in enumerate(vals[:n]):
            lst[i] = v
    return f


def _set_one(attr):
    def f(p, vals):
        if vals:
            setattr(p, attr, vals[0])
    return f


def _set_batch(p, vals):
    if vals:
        p.batch_size = vals[0] if vals[0] != 0 else 1000000  # :155


def _set_opt(p, vals):
    if vals:
        p.optimizer = "NelderMead" if vals[0][:10] == "NelderMead" else p.optimizer


_COMMON_HEAD = [
    ("LatticeParameter", "ffffff", _set_list("lattice", 6)),
    ("P_Array", "fff", _set_list("p_array", 3)),
    ("R_Array", "fff", _set_list("r_array", 3)),
    ("tol_c_over_a", "f", _set_one("tol_c_over_a")),
    ("PxX", "f", _set_one("px_x")),
    ("PxY", "f", _set_one("px_y")),
    ("Elo", "f", _set_one("elo")),
    ("Ehi", "f", _set_one("ehi")),
    ("DoFwd", "d", _set_one("do_fwd")),
    ("NrPxX", "d", _set_one("nr_px_x")),
    ("NrPxY", "d", _set_one("nr_px_y")),
    ("MaxNrLaueSpots", "d", _set_one("max_nr_spots")),
]
_COMMON_TAIL = [
    ("MinNrSpots", "d", _set_one("min_nr_spots")),
    ("SpaceGroup", "d", _set_one("space_group")),
    ("MinIntensity", "f", _set_one("min_intensity")),
    ("MaxAngle", "f", _set_one("max_angle")),
    ("ForwardFile", "s", _set_one("forward_file")),
    ("tol_LatC", "ffffff", _set_list("tol_latc", 6)),
    ("Optimizer", "s", _set_opt),
]
_KEYS = {
    # LaueMatchingCPU.c:75-204 (BatchSize sits between MaxNrLaueSpots and MinNrSpots)
    "cpu": _COMMON_HEAD + [("BatchSize", "z", _set_batch)] + _COMMON_TAIL,
    # LaueMatchingGPU.cu:132-259
    "gpu": _COMMON_HEAD + _COMMON_TAIL,
    # LaueMatchingGPUStream.cu:576-715
    "stream": _COMMON_HEAD + _COMMON_TAIL + [
        ("ResultDir", "s", _set_one("result_dir")),
        ("MinGoodSpots", "d", _set_one("min_good_spots")),
    ],
}


def _fgets_lines(data: bytes):
    """Split like repeated fgets(buf, 1000, f)."""
    pos, n = 0, len(data)
    while pos < n:
        nl = data.find(b"\n", pos, pos + 999)
        end = (nl + 1) if nl >= 0 else min(pos + 999, n)
        yield data[pos:end]
        pos = end


def parse_params_text(data: bytes | str, binary: str = "cpu",
                      validate: bool = True) -> LaueParams:
    if isinstance(data, str):
        data = data.encode("latin-1")
    keys = _KEYS[binary]
    p = LaueParams()
    for line in _fgets_lines(data):
        for key, fmt, setter in keys:
            if line.startswith(key.encode()):
                setter(p, _scan(line, fmt))
                break
        else:
            m = _TOK_RE.match(line)
            if m:
                p.extra[m.group(1).decode("latin-1")] = line.decode("latin-1").strip()
    if p.tol_c_over_a != 0:  # LaueMatchingCPU.c:205-208
        p.tol_latc = [0.0] * 6
    if validate:
        if p.nr_px_x <= 0 or p.nr_px_y <= 0:  # :211-215
            raise ParamsError(
                f"FATAL: NrPxX/NrPxY missing or non-positive ({p.nr_px_x} x {p.nr_px_y}). "
                "Check the parameter file.")
        if p.lattice[0] == 0.0:  # :216-220
            raise ParamsError("FATAL: LatticeParameter[a] is zero/unset. Check the parameter file.")
    return p


def read_params(path: str, binary: str = "cpu", validate: bool = True) -> LaueParams:
    with open(path, "rb") as f:
        return parse_params_text(f.read(), binary=binary, validate=validate)
