"""Batched refinement on the device (lmb_refine_*, refine.cu) against the
reference's own refinement objective and against host evaluation.

Objective values are compared bit for bit: with the reference's
problem_function (prefilterHKLs + calcOverlapFiltered from the reference's
LaueMatchingHeaders.h, _ref/libref_objective.so) on the golden scenes, and
with host evaluation of the same points.  Because the values are identical,
the lockstep Nelder-Mead takes the same steps on device and host: fitted
points, overlaps and evaluation counts must agree exactly.
"""
import numpy as np
import pytest

import ref_objective as RO
from lauematching_b200.engine import geometry_from_params
from lauematching_b200.refine import Refiner
from test_refine_host import CASES, scene, synthetic_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("crystal", ["params", "lattice", "c_over_a"])
def test_device_objective_equals_reference_and_host(name, crystal):
    if not RO.available():
        pytest.skip("oracle/_ref/libref_objective.so not built")
    c, p, geo, om, img = scene(name, crystal, n_grains=32)
    ref = RO.RefObjective(p, geo, c.hkls)
    with Refiner(p, geo, c.hkls, device=0) as d, Refiner(p, geo, c.hkls, device=None,
                                                        num_threads=8) as h:
        for r in (d, h):
            r.set_images([img])
        nvd = d.set_grains(om, 0)
        nvh = h.set_grains(om, 0)
        assert np.array_equal(nvd, nvh)
        x0, lo, hi = d.start()
        rng = np.random.default_rng(9)
        pts, grains, want = [], [], []
        for g in range(om.shape[0]):
            valid = ref.prefilter(x0[g][:3])
            assert nvd[g] == len(valid)
            for k in range(8):
                x = x0[g] if k == 0 else lo[g] + rng.random(d.dims) * (hi[g] - lo[g])
                pts.append(x)
                grains.append(g)
                want.append(ref.problem(x, img, valid))
        pts, grains = np.array(pts), np.array(grains)
        got = d.evaluate(grains, pts)
        assert np.array_equal(got, np.array(want))
        assert np.array_equal(got, h.evaluate(grains, pts))


def test_device_fit_equals_host_fit_on_a_synthetic_scene():
    c, p, geo, frames, image, om_true, om_c = synthetic_scene(n_frames=4, per_frame=32)
    with Refiner(p, geo, c.hkls, device=0) as d, Refiner(p, geo, c.hkls, device=None,
                                                        num_threads=8) as h:
        out = []
        for r in (d, h):
            r.set_images(frames)
            r.set_grains(om_c, image)
            once = r.fit("once")
            nm = r.fit("nelder-mead", 200)
            out.append((once, nm, r.last_stats()))
        (od, nd, sd), (oh, nh, sh) = out
        for a, b in zip(od + nd, oh + nh):
            assert np.array_equal(a, b)
        assert sd["points"] == sh["points"] and sd["rounds"] == sh["rounds"]
        assert sd["kernel_ms"] > 0
        assert (nd[1] >= od[1]).all() and nd[1].sum() > od[1].sum()


def test_device_objective_many_points_and_spot_cap():
    """Points of many grains in one launch (several blocks, every warp slot of
    the last block), on the scene with the largest valid lists (hexagonal,
    7790 HKLs), with MaxNrLaueSpots lowered to 12 so that the 3 x
    MaxNrLaueSpots cap on kept spots is reached."""
    c, p, geo, om, img = scene("tilted_hex", "params", n_grains=40)
    p.max_nr_spots = 12
    geo = geometry_from_params(p)
    with Refiner(p, geo, c.hkls, device=0) as d, Refiner(p, geo, c.hkls, device=None,
                                                        num_threads=8) as h:
        for r in (d, h):
            r.set_images([img])
        nv = d.set_grains(om, 0)
        h.set_grains(om, 0)
        assert nv.max() > 3 * p.max_nr_spots  # lists longer than the cap
        x0, lo, hi = d.start()
        rng = np.random.default_rng(2)
        m = 1021
        grains = rng.integers(0, om.shape[0], m)
        pts = lo[grains] + rng.random((m, d.dims)) * (hi[grains] - lo[grains])
        assert np.array_equal(d.evaluate(grains, pts), h.evaluate(grains, pts))
        assert d.evaluate([], np.zeros((0, d.dims))).shape == (0,)


def test_device_fit_reproduces_the_post_stage_nelder_mead_text():
    """The post-stage with "Optimizer NelderMead" fits on host threads; the same
    grains fitted on the device give the same overlaps, printed as the
    post-stage prints them (NMatches*sqrt(Intensity), %-13.4lf)."""
    import copy

    import oracle as O
    from conftest import golden_case
    from lauematching_b200 import post

    c = golden_case("tilted_dense")
    p = copy.deepcopy(c.params)
    s = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity)
    surv = np.zeros(len(s.ids), [("id", "<u8"), ("score", "<f8")])
    surv["id"] = s.ids
    surv["score"] = s.score
    ids, sc = post.collected_matches(surv, s.n_pass)
    geo = geometry_from_params(p)
    img = c.image.astype(np.float32)
    sol, _, _ = post.post_process(p, geo, c.orients, ids, sc, img, c.hkls, num_threads=8,
                                  optimizer="nelder-mead")
    rows, _, _ = post.merge_clusters(p.space_group, p.max_angle, c.orients, ids, sc)
    with Refiner(p, geo, c.hkls, device=0) as r:
        r.set_images([img.reshape(p.nr_px_y, p.nr_px_x)])
        r.set_grains(c.orients[rows.astype(np.int64)], 0)
        _, ov, _ = r.fit("nelder-mead", 200)
    printed = {int(f[0]): f[4] for f in (ln.split() for ln in sol.splitlines() if ln.strip())}
    assert len(printed) > 100
    for g, txt in printed.items():
        assert txt == "%.4f" % ov[g - 1]


def test_post_stage_refines_many_grains_on_the_device_with_the_host_text():
    """2200 grains on one frame, "Optimizer NelderMead", merge device given:
    the post-stage refines on the device (2048 or more grains) and writes the
    same solutions and spots text as on host threads."""
    from lauematching_b200 import post
    c, p, geo, frames, image, om_true, om_c = synthetic_scene(n_frames=1, per_frame=2200)
    ids = np.arange(om_c.shape[0], dtype=np.uint64)
    sc = np.linspace(100.0, 500.0, om_c.shape[0])
    img = frames[0].ravel()
    host = post.post_process(p, geo, om_c, ids, sc, img, c.hkls, num_threads=8,
                             optimizer="nelder-mead")
    st_host = post.last_refine_stats()
    dev = post.post_process(p, geo, om_c, ids, sc, img, c.hkls, num_threads=8,
                            optimizer="nelder-mead", merge_device=0)
    st_dev = post.last_refine_stats()
    assert host[2] >= 2048
    assert dev == host
    # the device path ran on the merge device, the host one on host threads
    assert st_host["device"] == -1 and st_host["kernel_ms"] == 0.0
    assert st_dev["device"] == 0 and st_dev["rounds"] > 0 and st_dev["kernel_ms"] > 0.0
    assert st_dev["points"] == st_host["points"] > 0
    # a second image reuses the post-stage's refinement handle: same text
    dev2 = post.post_process(p, geo, om_c, ids, sc, img, c.hkls, num_threads=8,
                             optimizer="nelder-mead", merge_device=0)
    assert dev2 == host and post.last_refine_stats()["device"] == 0
