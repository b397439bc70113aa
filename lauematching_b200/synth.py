"""Seeded synthetic workloads in the reference's file formats.

The reference benchmarks on a downloaded 100M-orientation DB and real detector
frames, none of which exist on these machines.  These generators make inputs
with the same shapes, sizes and value distributions:

* orientations: uniform random rotations by Shoemake's method (K. Shoemake,
  "Uniform random rotations", Graphics Gems III, 1992) driven by a
  counter-based generator (SplitMix64 finaliser of ``(seed, counter)``), so
  orientation ``i`` of seed ``s`` is the same whichever subset is generated,
  and the device generator in the CUDA library draws the same uniforms;
* HKL lists: all reflections allowed by the centring rule with
  ``|h|,|k|,|l| <= m``, excluding 000, sorted by ``h^2+k^2+l^2`` with ties
  kept in ascending (h, k, l) order (a stable sort of the meshgrid order of
  scripts/GenerateHKLs.py:159-210);
* images: Gaussian spots (sigma 2 px, amplitude U(50, 255)) at the
  forward-simulated pixels of each grain, a Poisson(5) background, a fixed
  background threshold, rounded to integers in [0, 255] with the maximum
  forced to 255 (so the uint8 quantisation scale is exactly 1).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "uniform_u01", "shoemake_orientations", "hkls_cubic", "hkls_hexagonal",
    "params_text", "render_image", "pick_grains",
]

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)
SEEDMUL = np.uint64(0xD1B54A32D192ED03)


def _splitmix_finalize(z: np.ndarray) -> np.ndarray:
    z = z ^ (z >> np.uint64(30))
    z = z * np.uint64(0xBF58476D1CE4E5B9)
    z = z ^ (z >> np.uint64(27))
    z = z * np.uint64(0x94D049BB133111EB)
    z = z ^ (z >> np.uint64(31))
    return z


def uniform_u01(seed: int, counters: np.ndarray) -> np.ndarray:
    """U[0,1) doubles for 64-bit ``counters`` (53 random bits each)."""
    with np.errstate(over="ignore"):
        c = np.asarray(counters, dtype=np.uint64)
        z = c * GOLDEN + np.uint64(seed & 0xFFFFFFFFFFFFFFFF) * SEEDMUL
        z = _splitmix_finalize(z)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def shoemake_orientations(n: int, seed: int, start: int = 0, ids=None) -> np.ndarray:
    """(n, 9) float64 row-major rotation matrices for IDs start..start+n-1 (or
    for the given ``ids``).  The device generator draws the same uniforms; its
    sines and cosines may differ from numpy's in the last bit."""
    ids = np.arange(start, start + n, dtype=np.uint64) if ids is None else \
        np.asarray(ids, dtype=np.uint64)
    n = ids.shape[0]
    u1 = uniform_u01(seed, ids * np.uint64(3) + np.uint64(0))
    u2 = uniform_u01(seed, ids * np.uint64(3) + np.uint64(1))
    u3 = uniform_u01(seed, ids * np.uint64(3) + np.uint64(2))
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    t2 = 2.0 * np.pi * u2
    t3 = 2.0 * np.pi * u3
    x, y = a * np.sin(t2), a * np.cos(t2)
    z, w = b * np.sin(t3), b * np.cos(t3)
    om = np.empty((n, 9), np.float64)
    om[:, 0] = 1.0 - 2.0 * (y * y + z * z)
    om[:, 1] = 2.0 * (x * y - z * w)
    om[:, 2] = 2.0 * (x * z + y * w)
    om[:, 3] = 2.0 * (x * y + z * w)
    om[:, 4] = 1.0 - 2.0 * (x * x + z * z)
    om[:, 5] = 2.0 * (y * z - x * w)
    om[:, 6] = 2.0 * (x * z - y * w)
    om[:, 7] = 2.0 * (y * z + x * w)
    om[:, 8] = 1.0 - 2.0 * (x * x + y * y)
    return om


_HEX_SYM = np.array([[1, 0, 0, 0], [0.86603, 0, 0, 0.5], [0.5, 0, 0, 0.86603], [0, 0, 0, 1],
                     [0.5, 0, 0, -0.86603], [0.86603, 0, 0, -0.5], [0, 1, 0, 0],
                     [0, 0.86603, 0.5, 0], [0, 0.5, 0.86603, 0], [0, 0, 1, 0],
                     [0, -0.5, 0.86603, 0], [0, -0.86603, 0.5, 0]])


def _om_to_quat(om: np.ndarray) -> np.ndarray:
    """Unit quaternions (w >= 0) of row-major rotation matrices (n, 9)."""
    m = om.reshape(-1, 3, 3)
    w = 0.5 * np.sqrt(np.maximum(0.0, 1.0 + m[:, 0, 0] + m[:, 1, 1] + m[:, 2, 2]))
    x = 0.5 * np.sqrt(np.maximum(0.0, 1.0 + m[:, 0, 0] - m[:, 1, 1] - m[:, 2, 2]))
    y = 0.5 * np.sqrt(np.maximum(0.0, 1.0 - m[:, 0, 0] + m[:, 1, 1] - m[:, 2, 2]))
    z = 0.5 * np.sqrt(np.maximum(0.0, 1.0 - m[:, 0, 0] - m[:, 1, 1] + m[:, 2, 2]))
    x = np.copysign(x, m[:, 2, 1] - m[:, 1, 2])
    y = np.copysign(y, m[:, 0, 2] - m[:, 2, 0])
    z = np.copysign(z, m[:, 1, 0] - m[:, 0, 1])
    q = np.stack([w, x, y, z], 1)
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _quat_to_om(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q.T
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                     2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                     2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1)


def hexagonal_fundamental_zone(om: np.ndarray) -> np.ndarray:
    """Reduce rotations to the hexagonal (622) fundamental zone: of the 12
    symmetry-equivalent quaternions q*s (the operator order and product of
    LaueMatchingHeaders.h:111-122,166-178) keep the one with the largest
    scalar part.  Uniform rotations map to uniform rotations in the zone."""
    q = _om_to_quat(np.asarray(om, np.float64))
    s = _HEX_SYM / np.linalg.norm(_HEX_SYM, axis=1, keepdims=True)
    # product Q = q (x) r with the reference's component formula
    w = s[None, :, 0] * q[:, None, 0] - s[None, :, 1] * q[:, None, 1] \
        - s[None, :, 2] * q[:, None, 2] - s[None, :, 3] * q[:, None, 3]
    best = np.argmax(np.abs(w), axis=1)
    r = s[best]
    Q = np.stack([
        r[:, 0] * q[:, 0] - r[:, 1] * q[:, 1] - r[:, 2] * q[:, 2] - r[:, 3] * q[:, 3],
        r[:, 1] * q[:, 0] + r[:, 0] * q[:, 1] + r[:, 3] * q[:, 2] - r[:, 2] * q[:, 3],
        r[:, 2] * q[:, 0] + r[:, 0] * q[:, 2] + r[:, 1] * q[:, 3] - r[:, 3] * q[:, 1],
        r[:, 3] * q[:, 0] + r[:, 0] * q[:, 3] + r[:, 2] * q[:, 1] - r[:, 1] * q[:, 2]], 1)
    Q *= np.where(Q[:, :1] < 0, -1.0, 1.0)
    Q /= np.linalg.norm(Q, axis=1, keepdims=True)
    return _quat_to_om(Q)


def _sorted_hkls(mask_fn, m: int) -> np.ndarray:
    r = np.arange(-m, m + 1)
    h, k, l = np.meshgrid(r, r, r, indexing="ij")
    h, k, l = h.ravel(), k.ravel(), l.ravel()
    keep = ~((h == 0) & (k == 0) & (l == 0)) & mask_fn(h, k, l)
    hkl = np.stack([h[keep], k[keep], l[keep]], 1).astype(np.int32)
    f2 = (hkl.astype(np.int64) ** 2).sum(1)
    return hkl[np.argsort(f2, kind="stable")]


def hkls_cubic(m: int = 8, centring: str = "F") -> np.ndarray:
    """Centring rules of scripts/GenerateHKLs.py:175-186."""
    rules = {
        "F": lambda h, k, l: ((h + k) % 2 == 0) & ((k + l) % 2 == 0),
        "I": lambda h, k, l: (h + k + l) % 2 == 0,
        "P": lambda h, k, l: np.ones_like(h, bool),
    }
    return _sorted_hkls(rules[centring], m)


def hkls_hexagonal(m: int = 10) -> np.ndarray:
    """Hexagonal rule of scripts/GenerateHKLs.py:194-195."""
    return _sorted_hkls(lambda h, k, l: ((h + 2 * k) % 3 != 0) | (l % 2 == 0), m)


def params_text(*, lattice=(0.352, 0.352, 0.352, 90, 90, 90), space_group=225,
                p=(0.0, 0.0, 0.5), r=(0.0, 0.0, 1e-12), px=0.0002,
                nr_px=(2048, 2048), elo=5.0, ehi=30.0, max_nr_spots=30,
                min_nr_spots=5, min_intensity=200.0, max_angle=2.0,
                forward_file="", do_fwd=0, min_good_spots=5,
                result_dir="results_stream", tol_c_over_a=0.0,
                extra: str = "") -> str:
    """Params text for the synthetic geometry: detector normal to the beam at
    ``p[2]`` metres (R_Array is a tiny non-zero vector because the reference
    divides by ``|R|``, LaueMatchingCPU.c:225-226)."""
    lines = [
        f"LatticeParameter {' '.join(repr(float(v)) for v in lattice)}",
        f"SpaceGroup {space_group}",
        f"P_Array {p[0]!r} {p[1]!r} {p[2]!r}",
        f"R_Array {r[0]!r} {r[1]!r} {r[2]!r}",
        f"PxX {px!r}",
        f"PxY {px!r}",
        f"NrPxX {nr_px[0]}",
        f"NrPxY {nr_px[1]}",
        f"Elo {elo!r}",
        f"Ehi {ehi!r}",
        f"MaxNrLaueSpots {max_nr_spots}",
        f"MinNrSpots {min_nr_spots}",
        f"MinIntensity {min_intensity!r}",
        f"MaxAngle {max_angle!r}",
        f"MinGoodSpots {min_good_spots}",
        f"ResultDir {result_dir}",
        f"DoFwd {do_fwd}",
    ]
    if tol_c_over_a:
        lines.append(f"tol_c_over_a {tol_c_over_a!r}")
    if forward_file:
        lines.append(f"ForwardFile {forward_file}")
    if extra:
        lines.append(extra)
    return "\n".join(lines) + "\n"


def pick_grains(records: np.ndarray, n_grains: int, min_spots: int,
                rng: np.random.Generator, id_offset: int = 0) -> np.ndarray:
    """Seeded choice of grain orientation IDs among DB records with at least
    ``min_spots`` spots (an image made of them is indexable)."""
    counts = records[:, 0].astype(np.int64)
    ok = np.nonzero(counts >= min_spots)[0]
    if ok.size == 0:
        return np.zeros(0, np.int64)
    pick = rng.choice(ok, size=min(n_grains, ok.size), replace=False)
    return np.sort(pick) + id_offset


def perturb_orientations(om: np.ndarray, rng: np.random.Generator, lo_deg: float,
                         hi_deg: float) -> np.ndarray:
    """Each orientation matrix (n, 9) turned by an angle uniform in
    [lo_deg, hi_deg] about a random axis (left-multiplied rotation): coarse
    starting points of a refinement, as a DB grid's nearest neighbour is."""
    om = np.asarray(om, np.float64).reshape(-1, 3, 3)
    ax = rng.normal(size=(om.shape[0], 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = np.deg2rad(rng.uniform(lo_deg, hi_deg, size=om.shape[0]))
    K = np.zeros((om.shape[0], 3, 3))
    K[:, 0, 1], K[:, 0, 2], K[:, 1, 2] = -ax[:, 2], ax[:, 1], -ax[:, 0]
    K[:, 1, 0], K[:, 2, 0], K[:, 2, 1] = ax[:, 2], -ax[:, 1], ax[:, 0]
    s, c = np.sin(ang)[:, None, None], np.cos(ang)[:, None, None]
    R = np.eye(3)[None] + s * K + (1 - c) * (K @ K)
    return (R @ om).reshape(-1, 9)


def render_image(grain_records: np.ndarray, nr_px_x: int, nr_px_y: int,
                 rng: np.random.Generator, sigma: float = 2.0,
                 amp_lo: float = 50.0, amp_hi: float = 255.0,
                 background: float = 5.0, threshold: float | None = 20.0,
                 force_max: float | None = 255.0) -> np.ndarray:
    """Float64 image (row-major [y][x]) with one Gaussian per listed spot.

    ``grain_records`` are forward-cache records (uint16[1+2S]) of the grains.
    Pixels below ``threshold`` after adding the Poisson background are set to
    0 (background removal); ``threshold=None`` keeps the background.
    """
    img = np.zeros((nr_px_y, nr_px_x), np.float64)
    rad = int(np.ceil(4 * sigma))
    off = np.arange(-rad, rad + 1)
    for rec in np.atleast_2d(grain_records):
        c = int(rec[0])
        for s in range(c):
            x, y = int(rec[1 + 2 * s]), int(rec[2 + 2 * s])
            a = rng.uniform(amp_lo, amp_hi)
            xs, ys = x + off, y + off
            mx = (xs >= 0) & (xs < nr_px_x)
            my = (ys >= 0) & (ys < nr_px_y)
            gx = np.exp(-0.5 * (off[mx] / sigma) ** 2)
            gy = np.exp(-0.5 * (off[my] / sigma) ** 2)
            img[np.ix_(ys[my], xs[mx])] += a * np.outer(gy, gx)
    if background:
        img += rng.poisson(background, size=img.shape)
    if threshold is not None:
        img[img < threshold] = 0.0
    img = np.clip(np.rint(img), 0, 255)
    if force_max is not None:
        mx = img.max()
        if mx > 0:
            img *= force_max / mx
            img = np.rint(img)
    return img.ravel()


def raw_frame(nr_px_y: int, nr_px_x: int, rng: np.random.Generator, n_spots: int = 200,
              spot_records: np.ndarray | None = None, sigma: float = 1.6,
              amp_lo: float = 40.0, amp_hi: float = 4000.0, pedestal: float = 100.0,
              gradient: float = 60.0, noise: float = 5.0, integer: bool = True) -> np.ndarray:
    """Unprocessed detector frame (float64 [y][x]) as the image server reads
    it: a smooth pedestal with a gradient, Poisson counting noise and one
    Gaussian per spot, before any background removal.  Spots come from the
    given forward-cache records, else at ``n_spots`` seeded positions.
    ``integer`` rounds to counts (a detector's values); otherwise adds a
    uniform fraction to every pixel, so nearly all values differ."""
    yy = np.linspace(0.0, 1.0, nr_px_y)[:, None]
    xx = np.linspace(0.0, 1.0, nr_px_x)[None, :]
    img = pedestal + gradient * (0.6 * yy + 0.4 * xx)
    img = rng.poisson(np.broadcast_to(img, (nr_px_y, nr_px_x)) + noise).astype(np.float64)
    if spot_records is not None:
        pts = []
        for rec in np.atleast_2d(spot_records):
            c = int(rec[0])
            pts += [(int(rec[2 + 2 * s]), int(rec[1 + 2 * s])) for s in range(c)]
        pts = np.array(pts, np.int64).reshape(-1, 2)
    else:
        pts = np.stack([rng.integers(0, nr_px_y, n_spots), rng.integers(0, nr_px_x, n_spots)], 1)
    rad = int(np.ceil(4 * sigma))
    off = np.arange(-rad, rad + 1)
    for y, x in pts:
        a = rng.uniform(amp_lo, amp_hi)
        s = sigma * rng.uniform(0.6, 1.6)
        xs, ys = x + off, y + off
        mx = (xs >= 0) & (xs < nr_px_x)
        my = (ys >= 0) & (ys < nr_px_y)
        gx = np.exp(-0.5 * (off[mx] / s) ** 2)
        gy = np.exp(-0.5 * (off[my] / s) ** 2)
        img[np.ix_(ys[my], xs[mx])] += a * np.outer(gy, gx)
    if integer:
        return np.rint(img)
    return img + rng.random(img.shape)
