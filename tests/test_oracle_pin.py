"""The oracle is pinned against the reference's own outputs.

Golden cases were produced by running the reference LaueMatchingCPU (built
from its sources) on seeded inputs; the oracle's FP64 restatement must give
the same forward cache byte for byte and the same survivor count ("Initial
solutions") for both the float64-image path (DoFwd 1) and the uint8 path
(DoFwd 0).  When the reference binary is present, a fresh small case is also
run through it directly.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden_case, golden_names
from lauematching_b200 import synth, params as P


@pytest.mark.parametrize("name", golden_names())
def test_oracle_forward_matches_reference_cache(name):
    c = golden_case(name)
    rec = O.forward(c.params, c.orients, c.hkls)
    assert rec.shape == c.records.shape
    assert np.array_equal(rec, c.records)


@pytest.mark.parametrize("name", golden_names())
def test_oracle_compare_counts_match_reference(name):
    c = golden_case(name)
    p = c.params
    s0 = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                   p.min_nr_spots, p.min_intensity, mode=0)
    assert s0.n_pass == c.meta["cmp_initial"]
    s1 = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                   p.min_nr_spots, p.min_intensity, mode=1)
    assert s1.n_pass == c.meta["fwd_initial"]
    # survivors are in ascending ID and include every grain the image was made of
    assert np.all(np.diff(s0.ids) > 0)
    assert set(c.meta["grains"]) <= set(s0.ids.tolist())


@pytest.mark.parametrize("name", golden_names())
def test_oracle_survivor_rows_appear_in_reference_solutions(name):
    """Every orientationRowNr the reference wrote is one of the oracle's survivors."""
    c = golden_case(name)
    p = c.params
    s0 = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                   p.min_nr_spots, p.min_intensity, mode=0)
    ids = set(s0.ids.tolist())
    score = dict(zip(s0.ids.tolist(), s0.score.tolist()))
    for line in c.cmp_solutions.splitlines()[1:]:
        cols = line.split("\t")
        cols = [x for x in cols if x.strip() != ""]
        row = int(cols[-1])
        coarse = float(cols[-3])
        assert row in ids
        assert abs(score[row] - coarse) <= 5e-5 * max(1.0, abs(coarse))


def test_quantize_known_answers():
    img = np.array([0.0, -3.0, 0.2, 1.0, 254.9, 255.0, 510.0, np.nan, 1e-300])
    u8, scale = O.quantize(img)
    # max 510 -> inv 0.5: 0.2*0.5 < 1 -> 1; 1*0.5 -> 1; 254.9*0.5=127.45 -> 127
    assert scale == 510.0 / 255.0
    assert u8.tolist() == [0, 0, 1, 1, 127, 127, 255, 0, 1]


@pytest.mark.skipif(not O.have_ref(), reason="reference binary not built here")
def test_fresh_case_against_reference_binary(tmp_path):
    """A case that is not in the golden set, run through the reference now."""
    txt = synth.params_text(p=(0.02, -0.01, 0.45), r=(-1.2, -1.21, -1.22), max_nr_spots=12,
                            min_nr_spots=4, min_intensity=150.0,
                            forward_file=str(tmp_path / "fwd.bin"), do_fwd=1)
    p = P.parse_params_text(txt)
    om = synth.shoemake_orientations(4000, seed=11)
    hk = synth.hkls_cubic(7, "I")
    rec = O.forward(p, om, hk)
    rng = np.random.default_rng(5)
    g = synth.pick_grains(rec, 2, 6, rng)
    img = synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng) * 1.3
    r = O.reference_case(str(tmp_path / "case"), txt, om, hk, img, ncpus=2)
    assert r.returncode == 0
    ref = np.fromfile(str(tmp_path / "fwd.bin"), np.uint16).reshape(rec.shape)
    assert np.array_equal(ref, rec)
    s1 = O.compare(rec, 12, img, p.nr_px_x, p.nr_px_y, 4, 150.0, mode=1)
    assert s1.n_pass == r.initial_solutions
