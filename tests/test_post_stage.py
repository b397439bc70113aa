"""Host post-stage (merge + evaluate-once refinement + output text) against the
reference's own solutions.txt / spots.txt.

The golden text was written by the reference LaueMatchingCPU (one thread,
NLopt replaced by an evaluate-once stand-in).  Feeding the oracle's
survivors of the same case to lmb_post_process must give the same bytes.
Host code only: runs without a GPU.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden_case, golden_names
from lauematching_b200 import post
from lauematching_b200.engine import geometry_from_params


def _strip_header(txt):
    return "".join(txt.splitlines(keepends=True)[1:])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode", [0, 1])
def test_post_stage_text_matches_reference(name, mode):
    c = golden_case(name)
    p = c.params
    s = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity, mode=mode)
    surv = np.zeros(len(s.ids), [("id", "<u8"), ("score", "<f8")])
    surv["id"] = s.ids
    surv["score"] = s.score
    ids, sc = post.collected_matches(surv, s.n_pass)
    sol, spt, nu = post.post_process(p, geometry_from_params(p), c.orients, ids, sc,
                                     c.image.astype(np.float32), c.hkls, num_threads=4)
    ref_sol = c.cmp_solutions if mode == 0 else c.fwd_solutions
    ref_spt = c.cmp_spots if mode == 0 else c.fwd_spots
    assert ref_sol.splitlines(keepends=True)[0] == post.SOLUTIONS_HEADER
    assert ref_spt.splitlines(keepends=True)[0] == post.SPOTS_HEADER
    assert sol == _strip_header(ref_sol)
    assert spt == _strip_header(ref_spt)
    assert nu == c.meta["cmp_unique" if mode == 0 else "fwd_unique"]


def test_post_stage_tolerates_no_survivors():
    c = golden_case("tilted_fcc")
    p = c.params
    sol, spt, nu = post.post_process(p, geometry_from_params(p), c.orients,
                                     np.zeros(0, np.uint64), np.zeros(0),
                                     c.image.astype(np.float32), c.hkls)
    assert (sol, spt, nu) == ("", "", 0)


@pytest.mark.parametrize("name", golden_names())
def test_merge_alone_gives_the_reference_unique_count(name):
    """lmb_merge_clusters (host path) on the oracle's collected matches gives
    the reference's "Unique Orientations" count, and counts that add up."""
    c = golden_case(name)
    p = c.params
    s = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity)
    surv = np.zeros(len(s.ids), [("id", "<u8"), ("score", "<f8")])
    surv["id"] = s.ids
    surv["score"] = s.score
    ids, sc = post.collected_matches(surv, s.n_pass)
    rows, scores, counts = post.merge_clusters(p.space_group, p.max_angle, c.orients, ids, sc)
    assert rows.shape[0] == c.meta["cmp_unique"]
    assert int(counts.sum()) == len(ids)


def test_post_stage_nelder_mead_refines_the_grains():
    """optimizer 1 (the parameter file's "Optimizer NelderMead"): this library's
    Nelder-Mead moves the grains off their coarse orientations and never
    lowers NMatches*sqrt(Intensity); the same clusters; deterministic."""
    import copy
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
    sol0, _, nu0 = post.post_process(p, geo, c.orients, ids, sc, img, c.hkls, num_threads=4)
    sol1, spt1, nu1 = post.post_process(p, geo, c.orients, ids, sc, img, c.hkls, num_threads=4,
                                        optimizer="nelder-mead")
    p.optimizer = "NelderMead"
    sol2, spt2, nu2 = post.post_process(p, geo, c.orients, ids, sc, img, c.hkls, num_threads=2)
    assert (sol2, spt2, nu2) == (sol1, spt1, nu1)
    assert nu0 == nu1

    def rows(txt):
        return {int(f[0]): [float(v) for v in f[2:]]
                for f in (ln.split() for ln in txt.splitlines() if ln.strip())}
    r0, r1 = rows(sol0), rows(sol1)
    common = sorted(set(r0) & set(r1))
    assert len(common) >= 0.8 * len(r0)
    # columns after GrainNr, NumberOfSolutions: Intensity, NMatches*Intensity,
    # NMatches*sqrt(Intensity), ...; misorientation is the second to last
    moved = improved = 0
    for g in common:
        assert r1[g][2] >= r0[g][2] - 1e-9 * abs(r0[g][2])
        improved += r1[g][2] > r0[g][2]
        moved += r1[g][-2] > 0
    assert improved > 0 and moved >= improved


def test_post_stage_rejects_unknown_optimizer():
    import ctypes as C
    from lauematching_b200 import _lib
    c = golden_case("tilted_fcc")
    p = c.params
    pp = post.make_post_params(p)
    pp.optimizer = 2
    geo = geometry_from_params(p)
    img = c.image.astype(np.float32)
    hk = np.ascontiguousarray(c.hkls, np.int32)
    om = np.ascontiguousarray(c.orients, np.float64)
    out = _lib.LmbPostOutput()
    rc = _lib.lib().lmb_post_process(C.byref(geo), C.byref(pp), om.ctypes.data, om.shape[0],
                                     None, None, 0, img.ctypes.data, hk.ctypes.data,
                                     hk.shape[0], C.byref(out))
    assert rc == _lib.LMB_ERR_INVALID
