"""Batched refinement on host threads (lmb_refine_*, device < 0) against the
reference's own refinement objective.

_ref/libref_objective.so exports prefilterHKLs, problem_function and
OrientMat2Euler compiled from the reference's LaueMatchingHeaders.h; the
golden cases give the scenes (frames, HKLs, geometry) and the oracle's
compare survivors the grains.  Host code only: runs without a GPU.
"""
import copy

import numpy as np
import pytest

import oracle as O
import ref_objective as RO
from conftest import golden_case
from lauematching_b200.engine import geometry_from_params
from lauematching_b200.refine import Refiner

pytestmark = pytest.mark.skipif(not RO.available(), reason="oracle/_ref/libref_objective.so not built")

CASES = ["tilted_fcc", "tilted_hex_ca", "tilted_dense", "beamnormal_fcc", "tilted_rhomb",
         "tilted_hex"]


def scene(name, crystal="params", n_grains=24):
    c = golden_case(name)
    p = copy.deepcopy(c.params)
    if crystal == "lattice":  # three lattice entries refined with the angles
        p.tol_latc = [0.01, 0.02, 0.0, 0.0, 0.005, 0.0]
        p.tol_c_over_a = 0.0
    elif crystal == "c_over_a":
        p.tol_c_over_a = 0.01
    s = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity)
    order = np.argsort(-np.asarray(s.score), kind="stable")[:n_grains]
    ids = np.asarray(s.ids)[order]
    if len(ids) < 4:  # few survivors: add orientations with many on-detector spots
        cnt = c.records[:, 0].astype(np.int64)
        ids = np.concatenate([ids, np.argsort(-cnt, kind="stable")[:n_grains - len(ids)]])
    img = c.image.astype(np.float32).reshape(p.nr_px_y, p.nr_px_x)
    return c, p, geometry_from_params(p), c.orients[ids], img


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("crystal", ["params", "lattice", "c_over_a"])
def test_host_objective_equals_reference(name, crystal):
    c, p, geo, om, img = scene(name, crystal)
    ref = RO.RefObjective(p, geo, c.hkls)
    with Refiner(p, geo, c.hkls, device=None, num_threads=4) as r:
        assert r.dims == ref.n
        r.set_images([img])
        nv = r.set_grains(om, 0)
        x0, lo, hi = r.start()
        rng = np.random.default_rng(5)
        pts, grains, want = [], [], []
        for g in range(om.shape[0]):
            rx, rlo, rhi = ref.start(om[g])
            assert np.array_equal(x0[g], rx) and np.array_equal(lo[g], rlo)
            assert np.array_equal(hi[g], rhi)
            valid = ref.prefilter(rx[:3])
            assert nv[g] == len(valid)
            for k in range(6):
                x = x0[g] if k == 0 else lo[g] + rng.random(r.dims) * (hi[g] - lo[g])
                pts.append(x)
                grains.append(g)
                want.append(ref.problem(x, img, valid))
        got = r.evaluate(np.array(grains), np.array(pts))
        assert np.array_equal(got, np.array(want))  # bit-identical FP64
        assert (np.array(want) < 0).any()


@pytest.mark.parametrize("name", ["tilted_fcc", "tilted_hex_ca"])
def test_host_fit_once_and_nelder_mead(name):
    c, p, geo, om, img = scene(name, "lattice" if name == "tilted_fcc" else "params")
    ref = RO.RefObjective(p, geo, c.hkls)
    with Refiner(p, geo, c.hkls, device=None, num_threads=4) as r:
        r.set_images([img])
        r.set_grains(om, 0)
        x0, lo, hi = r.start()
        xo, ovo, evo = r.fit("once")
        assert np.array_equal(xo, x0) and (evo == 1).all()
        for g in range(om.shape[0]):
            assert ovo[g] == -ref.problem(x0[g], img, ref.prefilter(x0[g][:3]))
        xn, ovn, evn = r.fit("nelder-mead", max_eval=200)
        assert (ovn >= ovo).all()  # never worse than the start point
        assert (xn >= lo).all() and (xn <= hi).all()
        assert (evn <= 200).all() and (evn >= r.dims + 1).all()
        st = r.last_stats()
        assert st["points"] == int(evn.sum()) and st["rounds"] >= 2
        # the fitted point's value is the reference objective there
        for g in range(om.shape[0]):
            assert ovn[g] == -ref.problem(xn[g], img, ref.prefilter(x0[g][:3]))
        # deterministic
        xn2, ovn2, evn2 = r.fit("nelder-mead", max_eval=200)
        assert np.array_equal(xn, xn2) and np.array_equal(ovn, ovn2) and np.array_equal(evn, evn2)


def test_host_refine_rejects_bad_arguments():
    c, p, geo, om, img = scene("tilted_fcc", n_grains=4)
    with Refiner(p, geo, c.hkls, device=None) as r:
        with pytest.raises(Exception):
            r.set_grains(om, 0)  # no images yet
        r.set_images([img])
        with pytest.raises(Exception):
            r.set_grains(om, 1)  # image index out of range
        r.set_grains(om, 0)
        with pytest.raises(Exception):
            r.evaluate([7], np.zeros((1, r.dims)))  # grain out of range
        with pytest.raises(Exception):
            r.fit("nelder-mead", max_eval=0)
        with pytest.raises(ValueError):
            r.set_images([img[:10]])


def synthetic_scene(n_frames=3, per_frame=24, seed=3, case="tilted_fcc", min_spots=8):
    """Frames rendered from true grain orientations (spots of the oracle's
    forward simulation) and coarse starting matrices turned 0.05-0.3 degrees
    away from them, as a DB grid's neighbour is."""
    from lauematching_b200 import synth
    c = golden_case(case)
    p = copy.deepcopy(c.params)
    rng = np.random.default_rng(seed)
    om_all = synth.shoemake_orientations(400 * per_frame * n_frames // 8 + 2000, seed=seed + 10)
    rec = O.forward(p, om_all, c.hkls)
    ok = np.nonzero(rec[:, 0] >= min_spots)[0][:n_frames * per_frame]
    assert len(ok) == n_frames * per_frame
    frames, image = [], []
    for f in range(n_frames):
        sel = ok[f * per_frame:(f + 1) * per_frame]
        img = synth.render_image(rec[sel], p.nr_px_x, p.nr_px_y, rng)
        frames.append(img.astype(np.float32).reshape(p.nr_px_y, p.nr_px_x))
        image += [f] * per_frame
    om_true = om_all[ok]
    om_coarse = synth.perturb_orientations(om_true, rng, 0.05, 0.3)
    return c, p, geometry_from_params(p), frames, np.array(image, np.int32), om_true, om_coarse


def test_host_fit_on_a_synthetic_scene_moves_toward_the_true_grains():
    c, p, geo, frames, image, om_true, om_c = synthetic_scene(n_frames=2, per_frame=16)
    with Refiner(p, geo, c.hkls, device=None, num_threads=4) as r:
        r.set_images(frames)
        r.set_grains(om_true, image)
        _, ov_true, _ = r.fit("once")
        r.set_grains(om_c, image)
        _, ov0, _ = r.fit("once")
        x, ov, ev = r.fit("nelder-mead", 200)
        assert (ov >= ov0).all() and ov.sum() > ov0.sum()
        assert ov_true.min() > 0  # every true grain sits on its spots


def test_host_objective_at_the_spot_cap_equals_reference():
    """MaxNrLaueSpots lowered to 12: valid lists of the hexagonal scene (7790
    HKLs) are longer than the 36 kept spots calcOverlapFiltered allows."""
    c, p, geo, om, img = scene("tilted_hex", "params", n_grains=40)
    p.max_nr_spots = 12
    geo = geometry_from_params(p)
    ref = RO.RefObjective(p, geo, c.hkls)
    with Refiner(p, geo, c.hkls, device=None, num_threads=4) as r:
        r.set_images([img])
        nv = r.set_grains(om, 0)
        assert nv.max() > 36
        x0, lo, hi = r.start()
        want = [ref.problem(x0[g], img, ref.prefilter(x0[g][:3])) for g in range(om.shape[0])]
        assert np.array_equal(r.evaluate(np.arange(om.shape[0]), x0), np.array(want))
