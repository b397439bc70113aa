"""The duplicate merge on the device (mergeDuplicateOrientations,
LaueMatchingHeaders.h:969-1065): the same clusters, kept rows, scores and
counts as the host loop, which restates the reference; and the same
solutions/spots text through the post-stage.

Candidate sets are seeded near-duplicate families: base orientations with
copies rotated by up to ~4 degrees, so that many pairs fall on either side of
MaxAngle = 2 degrees, with tied scores.
"""
import numpy as np
import pytest

from conftest import golden_case
from lauematching_b200 import post, synth

pytestmark = pytest.mark.gpu


def _rot(axis, ang):
    a = axis / np.linalg.norm(axis)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(ang) * k + (1 - np.cos(ang)) * (k @ k)


def _families(n_base, per, seed, max_deg=4.0):
    rng = np.random.default_rng(seed)
    base = synth.shoemake_orientations(n_base, seed=seed).reshape(-1, 3, 3)
    om = []
    for b in base:
        om.append(b)
        for _ in range(per - 1):
            om.append(_rot(rng.normal(size=3), np.deg2rad(rng.uniform(0, max_deg))) @ b)
    om = np.array(om).reshape(-1, 9)
    order = rng.permutation(om.shape[0])  # families interleaved in input order
    rows = np.sort(rng.choice(np.arange(om.shape[0] * 2), om.shape[0], replace=False))
    full = np.zeros((om.shape[0] * 2, 9))
    full[rows] = om[order]
    scores = rng.integers(1, 40, om.shape[0]).astype(np.float64) * 3.5  # many ties
    return full, rows.astype(np.uint64), scores


@pytest.mark.parametrize("sg,n_base,per", [(225, 120, 12), (194, 100, 15), (166, 300, 5)])
def test_device_merge_equals_host_merge(sg, n_base, per):
    orients, rows, scores = _families(n_base, per, seed=sg)
    assert rows.shape[0] >= 1024
    host = post.merge_clusters(sg, 2.0, orients, rows, scores)
    dev = post.merge_clusters(sg, 2.0, orients, rows, scores, device=0)
    # a wide band: many pairs decided by the host function inside the device run
    band = post.merge_clusters(sg, 2.0, orients, rows, scores, device=0, host_band=0.05)
    for got in (dev, band):
        for a, b in zip(host, got):
            assert np.array_equal(a, b)
    assert host[0].shape[0] < rows.shape[0]  # families did merge


def test_device_merge_in_the_post_stage_writes_the_same_text():
    c = golden_case("tilted_fcc")
    p = c.params
    orients, rows, scores = _families(90, 14, seed=7)
    args = (p, _geometry(p), orients, rows, scores, c.image.astype(np.float32), c.hkls)
    host = post.post_process(*args, num_threads=8)
    dev = post.post_process(*args, num_threads=8, merge_device=0)
    assert host == dev
    assert host[2] > 1


def _geometry(p):
    from lauematching_b200.engine import geometry_from_params
    return geometry_from_params(p)
