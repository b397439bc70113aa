"""Autotuner of the compare pass launch shape.

Sweeps kernel variant (block-barrier ring / warp-specialised / compact
layout), tile size, ring depth, consumer warps and grid size on the device for
a DB of the given record size and batch width, checks that every shape
returns the same survivors, and writes the fastest shape per (record words,
batch bucket) to ``tuning.json`` next to this file.  With ``--dense`` it
sweeps the cell-mask pass (variant 4) on a DB of many spots per record and
writes the ``_dense`` entries, the shape the automatic variant uses when it
picks that pass.  Engines load the table at creation.

    python -m lauematching_b200.autotune --n-orient 100000000 --batches 1,64 --write
    python -m lauematching_b200.autotune --dense --n-orient 100000000 --batches 64 --write
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")
BATCH_BUCKETS = (1, 4, 16, 64)


def batch_bucket(k: int) -> int:
    for b in BATCH_BUCKETS:
        if k <= b:
            return b
    return BATCH_BUCKETS[-1]


def load_table() -> dict:
    if os.path.exists(TABLE):
        with open(TABLE) as f:
            return json.load(f)
    return {}


def lookup(R: int, k: int, dense: bool = False) -> dict | None:
    """Best shape for records of R uint16 words and a pass of k images; with
    ``dense``, the cell-mask pass's shape (variant 4), which the automatic
    variant runs when the records that can pass hold many spots."""
    t = load_table().get("entries", {})
    suffix = f"_K{batch_bucket(k)}" + ("_dense" if dense else "")
    key = f"R{R}{suffix}"
    if key in t:
        return t[key]["shape"]
    # nearest record size with the same batch bucket
    cands = [(abs(int(kk.split("_")[0][1:]) - R), v) for kk, v in t.items()
             if kk.endswith(suffix)]
    return min(cands, key=lambda x: x[0])[1]["shape"] if cands else None


def candidate_shapes_dense():
    # the two-kernel cell-mask pass (what the automatic variant runs on dense
    # DBs): ring stages (tiles in flight per SM) and consumer warps, a
    # multiple of the stages (warps per stage split its tiles' chunks), 24 at
    # most; then a few shapes of the one-kernel pass for comparison
    for st, cpt in itertools.product((4, 6, 8, 10, 12, 16), (1, 2, 3, 4)):
        if st * cpt <= 24:
            yield dict(variant=5, stages=st, consumers=st * cpt)
    for q, cons in itertools.product((0, 1), (8, 12)):
        yield dict(variant=4, consumers=cons, cell_queue=q)


def candidate_shapes():
    # compact layout: the tile comes with the layout; ring depth 0 = as deep as fits
    # several small blocks per SM (each its own producer and ring) beat one big one
    for cons, st, gm in itertools.product((2, 3, 4, 6, 8), (2, 3, 4), (2, 3, 4, 5, 6, 8)):
        yield dict(variant=2, stages=st, consumers=cons, grid_mult=gm)
    for cons, st in itertools.product((8, 16), (0, 8)):
        yield dict(variant=2, stages=st, consumers=cons, grid_mult=1)
    for ts, st, cons in itertools.product((4, 8), (4, 6, 8, 12), (8, 12, 16)):
        yield dict(variant=1, tile_sub=ts, stages=st, consumers=cons)
    for ts, st, bps in itertools.product((4, 8), (2, 3, 4), (1, 2, 3)):
        yield dict(variant=0, tile_sub=ts, stages=st, blocks_per_sm=bps)


def time_shape(e, slots, p, reps=5, warm=2):
    for _ in range(warm):
        e.match(slots, p.min_nr_spots, p.min_intensity)
        e.last_pass_ms()
    ms = []
    for _ in range(reps):
        e.match(slots, p.min_nr_spots, p.min_intensity)
        ms.append(e.last_pass_ms()[0])
    return statistics.median(ms)


def main():
    sys.path.insert(0, os.path.dirname(HERE))
    from lauematching_b200 import synth, params as P
    from lauematching_b200.engine import Engine
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-orient", type=int, default=100_000_000)
    ap.add_argument("--batches", type=str, default="1,64")
    ap.add_argument("--max-nr-spots", type=int, default=30)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--write", action="store_true", help="update tuning.json")
    ap.add_argument("--dense", action="store_true",
                    help="tune the cell-mask pass (variant 4) on a DB of many spots per "
                         "record (the reference's tilted 34-ID-E detector); stored as the "
                         "table's _dense entries")
    args = ap.parse_args()
    geo = dict(p=(0.028745, 0.002788, 0.513115),
               r=(-1.20131258, -1.21399082, -1.21881158)) if args.dense else {}
    txt = synth.params_text(max_nr_spots=args.max_nr_spots, min_nr_spots=5, min_intensity=200.0,
                            **geo)
    p = P.parse_params_text(txt)
    hk = synth.hkls_cubic(8)
    e = Engine(p)
    t0 = time.time()
    e.build_db_synthetic(args.seed, args.n_orient, hk)
    print(f"DB of {args.n_orient} built in {time.time() - t0:.1f} s", file=sys.stderr)
    rec = e.download_db(0, min(2_000_000, args.n_orient))
    rng = np.random.default_rng(7)
    kmax = max(int(b) for b in args.batches.split(","))
    for k in range(kmax):
        g = synth.pick_grains(rec, int(rng.integers(1, 21)), p.min_nr_spots, rng)
        e.load_image(k, synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng).astype(np.uint8),
                     want_scale=False)
    table = load_table()
    entries = table.setdefault("entries", {})
    R = 1 + 2 * args.max_nr_spots
    for kb in (int(b) for b in args.batches.split(",")):
        slots = list(range(kb))
        ref = None
        results = []
        for shape in (candidate_shapes_dense() if args.dense else candidate_shapes()):
            e.set_tuning(**shape)
            try:
                ms = time_shape(e, slots, p)
            except Exception as exc:  # a shape that does not fit is skipped
                print(f"skip {shape}: {exc}", file=sys.stderr)
                continue
            got = [e.results(k)[0] for k in slots]
            if ref is None:
                ref = got
            same = all(np.array_equal(a, b) for a, b in zip(ref, got))
            used = dict(e.get_tuning(), cell_queue=shape.get("cell_queue", 0))
            results.append((ms, used, same))
            print(f"K={kb} {used} {ms:.4f} ms identical={same}", file=sys.stderr)
        ok = [r for r in results if r[2]]
        # the dense entry shapes the pass the automatic variant runs there (5)
        best = min([r for r in ok if not args.dense or r[1]["variant"] == 5] or ok,
                   key=lambda r: r[0])
        bytes_pass = args.n_orient * R * 2 + kb * p.nr_px_x * p.nr_px_y
        shape = dict(best[1])
        shape.pop("last_variant", None)
        if shape["variant"] == 2:  # engines pick the layout per pass (automatic variant 3)
            shape["variant"] = 3
        entries[f"R{R}_K{batch_bucket(kb)}" + ("_dense" if args.dense else "")] = {
            "shape": shape, "compare_ms": round(best[0], 4),
            "gbs": round(bytes_pass / (best[0] * 1e-3) / 1e9, 1), "n_orient": args.n_orient,
            "swept": len(results),
            "all": [{"shape": r[1], "ms": round(r[0], 4)} for r in sorted(results, key=lambda r: r[0])],
        }
        print(json.dumps({"K": kb, "best": best[1], "ms": best[0]}))
    table["device"] = "NVIDIA B200"
    if args.write:
        with open(TABLE, "w") as f:
            json.dump(table, f, indent=1)
    e.close()


if __name__ == "__main__":
    main()
