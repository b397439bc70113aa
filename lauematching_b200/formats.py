"""Binary and text file formats shared with the reference executables.

* Orientation file: row-major 3x3 float64 per orientation, 72 B, no header;
  the count is ``floor(filesize / 72)`` (LaueMatchingCPU.c:251-254,
  scripts/GenerateOrientations.py:11-14).
* HKL file: text, one reflection per line, the first three integers of each
  line via ``sscanf("%d %d %d")``; every line counts, even one that does not
  parse (its missing values stay 0); at most 200000 lines
  (LaueMatchingCPU.c:290-312, LaueMatchingHeaders.h:35).  File order is the
  simulation order.
* Forward cache ("ForwardFile"): per orientation ``uint16[1 + 2*S]`` =
  ``[count, x0, y0, x1, y1, ...]`` zero padded, record ``i`` at byte
  ``i * (1 + 2*S) * 2``, no header (LaueMatchingCPU.c:488-495, 645-648, 667).
* Image: raw float64 ``NrPxX * NrPxY``, row-major ``[y][x]``, pixel ``(x, y)``
  at index ``y * NrPxX + x`` (LaueMatchingCPU.c:324-332, 676).
"""
from __future__ import annotations

import os

import numpy as np

from .params import _fgets_lines, _INT_RE, _TOK_RE, _c_int

__all__ = [
    "MAX_NHKLS", "read_orientations", "write_orientations", "read_hkls",
    "write_hkls", "record_u16", "read_forward_cache", "write_forward_cache",
    "read_image_bin", "write_image_bin",
]

MAX_NHKLS = 200000  # LaueMatchingHeaders.h:35


def read_orientations(path: str, mmap: bool = True) -> np.ndarray:
    """Return an (N, 9) float64 array (memory-mapped when ``mmap``)."""
    size = os.path.getsize(path)
    n = size // 72
    if n == 0:
        return np.zeros((0, 9), np.float64)
    if mmap:
        return np.memmap(path, dtype=np.float64, mode="r", shape=(n, 9))
    return np.fromfile(path, dtype=np.float64, count=n * 9).reshape(n, 9)


def write_orientations(path: str, om: np.ndarray) -> None:
    np.ascontiguousarray(om, dtype=np.float64).reshape(-1, 9).tofile(path)


def read_hkls(path: str) -> np.ndarray:
    """Return an (n, 3) int32 array with the reference's line semantics."""
    with open(path, "rb") as f:
        data = f.read()
    rows = []
    for line in _fgets_lines(data):
        if len(rows) >= MAX_NHKLS:
            break
        vals = [0, 0, 0]
        pos = 0
        for i in range(3):
            m = _INT_RE.match(line, pos)
            if not m:
                break
            vals[i] = _c_int(int(m.group(1)))
            pos = m.end()
        rows.append(vals)
    return np.asarray(rows, dtype=np.int32).reshape(-1, 3)


def write_hkls(path: str, hkls: np.ndarray) -> None:
    """Write ``h k l h^2+k^2+l^2`` lines, the layout GenerateHKLs.py saves."""
    h = np.asarray(hkls, dtype=np.int64).reshape(-1, 3)
    with open(path, "w") as f:
        for a, b, c in h:
            f.write(f"{a} {b} {c} {a * a + b * b + c * c}\n")


def record_u16(max_nr_spots: int) -> int:
    """uint16 words per forward-cache record."""
    return 1 + 2 * int(max_nr_spots)


def read_forward_cache(path: str, n_orient: int, max_nr_spots: int,
                       mmap: bool = True) -> np.ndarray:
    R = record_u16(max_nr_spots)
    need = n_orient * R * 2
    size = os.path.getsize(path)
    if size < need:
        raise ValueError(f"forward cache {path} holds {size} bytes, "
                         f"{need} needed for {n_orient} records of {R} uint16")
    if mmap:
        return np.memmap(path, dtype=np.uint16, mode="r", shape=(n_orient, R))
    return np.fromfile(path, dtype=np.uint16, count=n_orient * R).reshape(n_orient, R)


def write_forward_cache(path: str, records: np.ndarray, offset_records: int = 0) -> None:
    """Write records at their ID offset (``pwrite`` semantics, file not truncated)."""
    rec = np.ascontiguousarray(records, dtype=np.uint16)
    flags = os.O_CREAT | os.O_WRONLY
    fd = os.open(path, flags, 0o600)
    try:
        off = offset_records * rec.shape[1] * 2
        mv = memoryview(rec).cast("B")
        done = 0
        while done < len(mv):
            done += os.pwrite(fd, mv[done:], off + done)
    finally:
        os.close(fd)


def read_image_bin(path: str, nr_px_x: int, nr_px_y: int) -> np.ndarray:
    n = nr_px_x * nr_px_y
    img = np.fromfile(path, dtype=np.float64, count=n)
    if img.size != n:
        raise ValueError(f"Error: Unexpected end of file while reading image {path}")
    return img


def write_image_bin(path: str, img: np.ndarray) -> None:
    np.ascontiguousarray(img, dtype=np.float64).tofile(path)
