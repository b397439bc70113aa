"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs the reference's own LaueMatchingCPU (built from its sources by
oracle/Makefile into oracle/_ref/) on seeded synthetic cases and stores, per
case, the inputs and the reference's outputs:

  <case>.npz   params text, the orientation seed/count (matrices regenerated
               by synth.shoemake_orientations, pinned by their SHA-256), HKLs,
               the image (uint8 values times a scale),
               the forward cache written by the reference (DoFwd 1),
               the reference's "Initial solutions" / "Unique Orientations"
               counts for DoFwd 1 and DoFwd 0, and its solutions.txt /
               spots.txt (one thread, so the line order is deterministic).

Usage (in a checkout where the reference tree and oracle/_ref exist):
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from lauematching_b200 import params as P, synth  # noqa: E402

TILTED = dict(p=(0.028745, 0.002788, 0.513115), r=(-1.20131258, -1.21399082, -1.21881158))

CASES = {
    # survey geometry: detector normal to the beam at 0.5 m, fcc a=3.52 A
    "beamnormal_fcc": dict(n=20000, seed=0, hkl=("cubic", 8), geom={}, S=30, grains=3,
                           min_spots=5, min_int=200.0, grain_min=5),
    # the reference's own 34-ID-E geometry (params_sim.txt), fcc
    "tilted_fcc": dict(n=20000, seed=2, hkl=("cubic", 8), geom=TILTED, S=30, grains=3,
                       min_spots=5, min_int=200.0, grain_min=8),
    # imScale != 1: image maximum 643.7, FP64 sums of raw*imScale
    "tilted_scaled": dict(n=12000, seed=3, hkl=("cubic", 8), geom=TILTED, S=30, grains=4,
                          min_spots=6, min_int=700.0, grain_min=8, scale=643.7 / 255.0),
    # background kept (no threshold): many survivors
    "tilted_dense": dict(n=6000, seed=4, hkl=("cubic", 6), geom=TILTED, S=30, grains=3,
                         min_spots=5, min_int=60.0, grain_min=8, threshold=None,
                         nr_px=(512, 512), px=0.0008),
    # small S: the cap at MaxNrLaueSpots decides which HKLs fill the record
    "tilted_cap5": dict(n=8000, seed=5, hkl=("cubic", 8), geom=TILTED, S=5, grains=3,
                        min_spots=3, min_int=100.0, grain_min=4),
    # hexagonal (SG 194, a=2.95 A, c=4.68 A), |h|,|k|,|l|<=10
    "tilted_hex": dict(n=3000, seed=6, hkl=("hex", 10), geom=TILTED, S=30, grains=2,
                       min_spots=5, min_int=200.0, grain_min=8,
                       lattice=(0.295, 0.295, 0.468, 90, 90, 120), sg=194),
    # rhombohedral setting (SG 166) exercises the other calcRecipArray branch
    "tilted_rhomb": dict(n=3000, seed=7, hkl=("cubic", 6, "P"), geom=TILTED, S=30, grains=2,
                         min_spots=5, min_int=200.0, grain_min=6,
                         lattice=(0.45, 0.45, 0.45, 58, 58, 58), sg=166),
    # hexagonal with c/a refinement (tol_c_over_a): the lattice of the refined
    # grains comes from the c/a path of FitOrientation (cbrt of the cell volume)
    "tilted_hex_ca": dict(n=3000, seed=8, hkl=("hex", 8), geom=TILTED, S=30, grains=3,
                          min_spots=5, min_int=200.0, grain_min=8,
                          lattice=(0.295, 0.295, 0.468, 90, 90, 120), sg=194,
                          tol_c_over_a=0.01, max_angle=5.0),
}


def make_case(name, c, workdir):
    lattice = c.get("lattice", (0.352, 0.352, 0.352, 90, 90, 90))
    sg = c.get("sg", 225)
    fwd = os.path.join(workdir, name + ".fwd.bin")
    txt = synth.params_text(lattice=lattice, space_group=sg, max_nr_spots=c["S"],
                            min_nr_spots=c["min_spots"], min_intensity=c["min_int"],
                            forward_file=fwd, do_fwd=1, nr_px=c.get("nr_px", (2048, 2048)),
                            px=c.get("px", 0.0002), tol_c_over_a=c.get("tol_c_over_a", 0.0),
                            max_angle=c.get("max_angle", 2.0), **c["geom"])
    p = P.parse_params_text(txt)
    om = synth.shoemake_orientations(c["n"], seed=c["seed"])
    kind = c["hkl"][0]
    if kind == "cubic":
        hk = synth.hkls_cubic(c["hkl"][1], *(c["hkl"][2:] or ("F",)))
    else:
        hk = synth.hkls_hexagonal(c["hkl"][1])
    rec_oracle = O.forward(p, om, hk)
    rng = np.random.default_rng(c["seed"] + 100)
    g = synth.pick_grains(rec_oracle, c["grains"], c["grain_min"], rng)
    img = synth.render_image(rec_oracle[g], p.nr_px_x, p.nr_px_y, rng,
                             threshold=c.get("threshold", 20.0))
    img_u8 = img.astype(np.uint8)
    assert np.array_equal(img_u8, img)
    scale = c.get("scale", 1.0)
    img = img_u8 * scale
    r1 = O.reference_case(os.path.join(workdir, name + "_fwd"), txt, om, hk, img, ncpus=1)
    assert r1.returncode == 0, r1.stdout + r1.stderr
    rec_ref = np.fromfile(fwd, np.uint16).reshape(c["n"], 1 + 2 * c["S"])
    txt0 = txt.replace("DoFwd 1", "DoFwd 0")
    r0 = O.reference_case(os.path.join(workdir, name + "_cmp"), txt0, om, hk, img, ncpus=1)
    assert r0.returncode == 0, r0.stdout + r0.stderr
    meta = dict(grains=[int(x) for x in g], fwd_initial=r1.initial_solutions,
                fwd_unique=r1.unique, cmp_initial=r0.initial_solutions, cmp_unique=r0.unique)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        params_text=np.array(txt0), seed=np.array(c["seed"]), n=np.array(c["n"]),
        orients_sha256=np.array(hashlib.sha256(om.tobytes()).hexdigest()), hkls=hk,
        img_u8=img_u8, img_scale=np.array(scale), records=rec_ref,
        meta=np.array(json.dumps(meta)),
        fwd_solutions=np.array(r1.solutions or ""), fwd_spots=np.array(r1.spots or ""),
        cmp_solutions=np.array(r0.solutions or ""), cmp_spots=np.array(r0.spots or ""))
    same = np.array_equal(rec_ref, rec_oracle)
    print(f"{name}: n={c['n']} nhkl={len(hk)} mean_spots={rec_ref[:, 0].mean():.2f} "
          f"fwd_initial={r1.initial_solutions} cmp_initial={r0.initial_solutions} "
          f"unique={r0.unique} oracle_records_identical={same}")


def main():
    if not O.have_ref():
        sys.exit("oracle/_ref/LaueMatchingCPU missing: run `make -C oracle` where the "
                 "reference tree is present")
    wd = O.tempdir()
    names = sys.argv[1:] or list(CASES)
    for name in names:
        make_case(name, CASES[name], wd)


if __name__ == "__main__":
    main()
