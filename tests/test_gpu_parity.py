"""GPU parity: the sm_100a kernels, called through the C ABI, against the
oracle and the reference's golden outputs.

Bar: bit-exact.  Records byte for byte; survivors' IDs, spot counts and uint8
sums equal; the FP64 intensity sums and scores equal to the last bit (the
kernels reproduce the reference's operation order and rounding).
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden_case, golden_names
from lauematching_b200 import synth, params as P
from lauematching_b200._lib import OverflowError_, LmbError

pytestmark = pytest.mark.gpu


def engine_for(p, cap=0):
    from lauematching_b200.engine import Engine
    return Engine(p, device=0, survivor_capacity=cap)


def assert_same_survivors(got, ref):
    assert got.shape[0] == ref.ids.shape[0]
    assert np.array_equal(got["id"], ref.ids.astype(np.uint64))
    assert np.array_equal(got["n_spots"], ref.n_spots)
    assert np.array_equal(got["sum_u8"], ref.sum_u8)
    assert np.array_equal(got["tot_int"].view(np.uint64), ref.tot_int.view(np.uint64))
    assert np.array_equal(got["score"].view(np.uint64), ref.score.view(np.uint64))


@pytest.mark.parametrize("name", golden_names())
def test_db_build_matches_reference_cache(name):
    c = golden_case(name)
    with engine_for(c.params) as e:
        e.build_db(c.orients, c.hkls)
        assert np.array_equal(e.download_db(), c.records)


@pytest.mark.parametrize("name", ["tilted_fcc", "tilted_hex", "beamnormal_fcc", "tilted_rhomb", "tilted_cap5"])
def test_db_build_fp32_screen_equals_all_fp64(name):
    c = golden_case(name)
    om = synth.shoemake_orientations(200000, seed=123)
    with engine_for(c.params) as e:
        e.build_db(om, c.hkls, exact_fp64=True)
        full = e.download_db()
        e.build_db(om, c.hkls)
        assert np.array_equal(e.download_db(), full)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode", [0, 1])
def test_compare_matches_oracle(name, mode):
    c = golden_case(name)
    p = c.params
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity, mode=mode)
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(5, c.image, keep_f64=(mode == 1))
        e.match([5], p.min_nr_spots, p.min_intensity, value_mode=mode)
        got, npass = e.results(5)
    assert npass == ref.n_pass
    assert npass == c.meta["cmp_initial" if mode == 0 else "fwd_initial"]
    assert_same_survivors(got, ref)


def _batch_case(n=300000, k=12, seed=9, S=30, min_spots=5, min_int=150.0):
    txt = synth.params_text(p=(0.028745, 0.002788, 0.513115),
                            r=(-1.20131258, -1.21399082, -1.21881158), max_nr_spots=S,
                            min_nr_spots=min_spots, min_intensity=min_int)
    p = P.parse_params_text(txt)
    hk = synth.hkls_cubic(8)
    return p, hk


def test_batched_pass_equals_single_passes_and_oracle():
    """K images of uneven grain counts in one DB pass == K separate passes
    == the oracle, each image alone."""
    p, hk = _batch_case()
    rng = np.random.default_rng(3)
    with engine_for(p) as e:
        om = e.build_db_synthetic(seed=77, n=300000, hkls=hk, return_orients=True)
        rec = e.download_db()
        imgs = []
        for k in range(12):
            g = synth.pick_grains(rec, int(rng.integers(1, 21)), 8, rng)
            img = synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng,
                                     threshold=None if k == 3 else 20.0)
            if k == 7:
                img = img * 2.71
            imgs.append(img)
            e.load_image(k, img)
        e.match(range(12), p.min_nr_spots, p.min_intensity)
        batched = [e.results(k) for k in range(12)]
        for k in range(12):
            e.match([k], p.min_nr_spots, p.min_intensity)
            single = e.results(k)
            assert single[1] == batched[k][1]
            assert np.array_equal(single[0], batched[k][0])
    assert np.array_equal(O.forward(p, om[:20000], hk), rec[:20000])
    for k in (0, 3, 7, 11):
        ref = O.compare(rec, p.max_nr_spots, imgs[k], p.nr_px_x, p.nr_px_y,
                        p.min_nr_spots, p.min_intensity)
        assert batched[k][1] == ref.n_pass
        assert_same_survivors(batched[k][0], ref)


def test_results_batch_equals_per_slot_results():
    c = golden_case("tilted_dense")
    p = c.params
    with engine_for(p) as e:
        e.upload_db(c.records)
        for k, s in enumerate((0.5, 1.0, 2.0)):
            e.load_image(k * 7, c.image * s)
        e.match([0, 7, 14], p.min_nr_spots, p.min_intensity)
        per = {k: e.results(k) for k in (14, 0, 7)}
        e.match([0, 7, 14], p.min_nr_spots, p.min_intensity)
        bat = e.results_batch([14, 0, 7])
    for k in (0, 7, 14):
        assert bat[k][1] == per[k][1] and np.array_equal(bat[k][0], per[k][0])


def test_input_dtypes_f32_u8_match_f64():
    c = golden_case("tilted_fcc")
    p = c.params
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(0, c.image)
        e.load_image(1, c.image.astype(np.float32))
        e.load_image(2, c.img_u8)
        e.match([0, 1, 2], p.min_nr_spots, p.min_intensity)
        r = [e.results(k) for k in range(3)]
    for k in (1, 2):
        assert np.array_equal(r[0][0], r[k][0]) and r[0][1] == r[k][1]


@pytest.mark.parametrize("variant,full_gather,queue", [(1, 0, 0), (1, 1, 0), (2, 0, 0), (2, 1, 0),
                                                      (4, 0, 0), (4, 1, 0), (4, 0, 1), (4, 1, 1),
                                                      (5, 0, 0), (5, 1, 0)])
def test_edge_records_partial_tiles_and_thresholds(variant, full_gather, queue):
    """Counts above S (clamped), pixels off the detector (skipped), DB sizes
    that are not a multiple of the tile, MinNrSpots <= 0 and > S; in the
    reference layout (variant 1), the compact one (variant 2) and the compact
    one filtered by the cell mask (variant 4), with and without skipping
    records that have fewer spots than MinNrSpots."""
    rng = np.random.default_rng(1)
    txt = synth.params_text(nr_px=(300, 200), max_nr_spots=7, min_nr_spots=2,
                            min_intensity=3.0)
    p = P.parse_params_text(txt)
    for n in (0, 1, 7, 255, 256, 257, 1000, 4099, 70000):
        rec = np.zeros((n, 15), np.uint16)
        if n:
            rec[:, 0] = rng.integers(0, 12, n)       # some counts exceed S=7
            rec[:, 1::2] = rng.integers(0, 330, (n, 7))  # some x >= 300
            rec[:, 2::2] = rng.integers(0, 220, (n, 7))  # some y >= 200
        img = np.where(rng.random(300 * 200) < 0.3, rng.integers(1, 256, 300 * 200), 0)
        img = img.astype(np.float64) * 0.77
        with engine_for(p) as e:
            e.set_tuning(variant=variant, full_gather=full_gather, cell_queue=queue)
            e.upload_db(rec)
            e.load_image(0, img)
            for ms, mi in ((2, 3.0), (0, 0.0), (-3, -1.0), (8, 0.0), (1, 1e9)):
                e.match([0], ms, mi)
                got, npass = e.results(0)
                ref = O.compare(rec, 7, img, 300, 200, ms, mi)
                assert npass == ref.n_pass, (n, ms, mi)
                assert_same_survivors(got, ref)
            if variant in (2, 4, 5) and n:
                assert e.layout_info()["compact"] == 1
                assert e.get_tuning()["last_variant"] == variant


@pytest.mark.parametrize("name", golden_names())
def test_automatic_variant_follows_the_spots_that_can_pass(name):
    """The default (automatic) variant runs the compact layout while the
    records that can pass hold at most 3 spots per DB record, the compact
    layout filtered by the frames' cell mask otherwise; both give the
    oracle's survivors."""
    c = golden_case(name)
    p = c.params
    cnt = np.minimum(c.records[:, 0], p.max_nr_spots).astype(np.int64)  # all on the detector
    gathered = cnt[cnt >= max(p.min_nr_spots, 0)].sum() / cnt.shape[0]
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity)
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(1, c.image)
        e.match([1], p.min_nr_spots, p.min_intensity)
        got, npass = e.results(1)
        used = e.get_tuning()
    assert used["variant"] == 3
    assert used["last_variant"] == (2 if gathered <= 3.0 else 5), gathered
    assert npass == ref.n_pass
    assert_same_survivors(got, ref)


@pytest.mark.parametrize("variant", [2, 3, 4, 5])
def test_many_spots_per_record_keep_the_reference_layout(variant):
    """MaxNrLaueSpots above 255 (uint8 counts cannot hold it): a pass asked for
    the compact layout (alone, automatic or with the cell mask) runs over the
    reference records and matches the oracle."""
    rng = np.random.default_rng(3)
    S = 300
    txt = synth.params_text(nr_px=(256, 256), max_nr_spots=S, min_nr_spots=20,
                            min_intensity=10.0)
    p = P.parse_params_text(txt)
    n = 3000
    rec = np.zeros((n, 1 + 2 * S), np.uint16)
    rec[:, 0] = rng.integers(0, S + 5, n)
    rec[:, 1::2] = rng.integers(0, 260, (n, S))
    rec[:, 2::2] = rng.integers(0, 260, (n, S))
    img = np.where(rng.random(256 * 256) < 0.2, rng.integers(1, 256, 256 * 256), 0).astype(np.float64)
    ref = O.compare(rec, S, img, 256, 256, p.min_nr_spots, p.min_intensity)
    with engine_for(p) as e:
        e.set_tuning(variant=variant)
        e.upload_db(rec)
        e.load_image(0, img)
        e.match([0], p.min_nr_spots, p.min_intensity)
        got, npass = e.results(0)
        assert e.layout_info()["compact"] == -1
        assert e.get_tuning()["last_variant"] == 1
    assert npass == ref.n_pass
    assert_same_survivors(got, ref)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode", [0, 1])
def test_compact_layout_matches_oracle(name, mode):
    """Variant 2 (compact device layout) on the reference's golden cases."""
    c = golden_case(name)
    p = c.params
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity, mode=mode)
    with engine_for(p) as e:
        e.set_tuning(variant=2)
        e.upload_db(c.records)
        e.load_image(5, c.image, keep_f64=(mode == 1))
        e.load_image(6, c.image * 0.5, keep_f64=(mode == 1))
        e.match([5, 6], p.min_nr_spots, p.min_intensity, value_mode=mode)
        got, npass = e.results(5)
        info = e.layout_info()
    assert info["compact"] == 1 and 0 < info["bytes"]
    assert npass == ref.n_pass
    assert_same_survivors(got, ref)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("variant,queue", [(4, 0), (4, 1), (5, 0)])
def test_cell_mask_pass_matches_oracle(name, mode, variant, queue):
    """Variant 4 (compact layout filtered by the cell mask of the pass's
    frames) on the reference's golden cases.  A frame in a slot outside the
    pass, positive everywhere, must not widen or change anything: the mask is
    built from the pass's slots."""
    c = golden_case(name)
    p = c.params
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity, mode=mode)
    ref2 = O.compare(c.records, p.max_nr_spots, c.image * 0.5, p.nr_px_x, p.nr_px_y,
                     p.min_nr_spots, p.min_intensity, mode=mode)
    with engine_for(p) as e:
        e.set_tuning(variant=variant, cell_queue=queue)
        e.upload_db(c.records)
        e.load_image(5, c.image, keep_f64=(mode == 1))
        e.load_image(6, c.image * 0.5, keep_f64=(mode == 1))
        e.load_image(9, np.full(p.nr_px_x * p.nr_px_y, 7.0), keep_f64=(mode == 1))
        for _ in range(2):  # eager pass, then the graph replay
            e.match([5, 6], p.min_nr_spots, p.min_intensity, value_mode=mode)
            got, npass = e.results(5)
            got2, npass2 = e.results(6)
            assert e.get_tuning()["last_variant"] == variant
            assert npass == ref.n_pass and npass2 == ref2.n_pass
            assert_same_survivors(got, ref)
            assert_same_survivors(got2, ref2)


@pytest.mark.parametrize("nr_px", [(1100, 1001), (2048, 2048), (1024, 1024)])
def test_cell_mask_cells_and_detector_sizes(nr_px):
    """Cell masks of 2^shift-pixel cells (shift 0 for 1024^2, 1 with a
    partial last cell for 1100x1001, 2 for 2048^2) on dense random records
    and frames of a few percent positive pixels: the oracle's survivors, for
    MinNrSpots from 1 to above the records' spot counts."""
    rng = np.random.default_rng(11)
    W, H = nr_px
    S = 30
    txt = synth.params_text(nr_px=(W, H), max_nr_spots=S, min_nr_spots=3, min_intensity=5.0)
    p = P.parse_params_text(txt)
    n = 40000
    rec = np.zeros((n, 1 + 2 * S), np.uint16)
    rec[:, 0] = rng.integers(8, 25, n)
    rec[:, 1::2] = rng.integers(0, W, (n, S))
    rec[:, 2::2] = rng.integers(0, H, (n, S))
    # frames: positive pixels around the spots of a few records (so records
    # match) plus scattered singles, the last pixel of the detector included
    imgs = []
    for k in range(3):
        img = np.zeros(W * H)
        img[rng.integers(0, W * H, W * H // 40)] = rng.integers(1, 256, W * H // 40)
        for r in rng.integers(0, n, 30):
            c = int(rec[r, 0])
            img[rec[r, 2:2 + 2 * c:2].astype(np.int64) * W + rec[r, 1:1 + 2 * c:2]] = 200.0
        img[-1] = 99.0
        imgs.append(img)
    with engine_for(p) as e:
        e.upload_db(rec)
        for k in range(3):
            e.load_image(k, imgs[k])
        for variant, queue in ((4, 0), (4, 1), (5, 0)):
            e.set_tuning(variant=variant, cell_queue=queue)
            for ms in (1, 3, 6, 24, 30):
                e.match([0, 1, 2], ms, 5.0)
                assert e.get_tuning()["last_variant"] == variant
                for k in range(3):
                    got, npass = e.results(k)
                    ref = O.compare(rec, S, imgs[k], W, H, ms, 5.0)
                    assert npass == ref.n_pass, (ms, k, queue)
                    assert_same_survivors(got, ref)


@pytest.mark.parametrize("nb", [7, 8])
def test_compact_layout_sized_for_more_blocks_matches_oracle(nb):
    """The compact layout built for 7 or 8 blocks per SM (smaller tiles) and
    passes at that block count: the oracle's survivors on two golden cases."""
    for name in ("tilted_fcc", "beamnormal_fcc"):
        c = golden_case(name)
        p = c.params
        ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                        p.min_nr_spots, p.min_intensity)
        with engine_for(p) as e:
            e.set_tuning(variant=2, consumers=3, stages=2, grid_mult=nb)
            e.upload_db(c.records)
            e.load_image(0, c.image)
            e.match([0], p.min_nr_spots, p.min_intensity)
            got, npass = e.results(0)
            info = e.layout_info()
        assert info["compact"] == 1 and info["tile_bytes"] % 128 == 0
        assert npass == ref.n_pass
        assert_same_survivors(got, ref)


def test_compact_layout_batched_equals_reference_layout():
    """Twelve uneven frames in one pass: variant 2 == variant 1, slot by slot,
    on a 300k-orientation device-built DB, for several tile shapes."""
    p, hk = _batch_case()
    rng = np.random.default_rng(5)
    with engine_for(p) as e:
        e.build_db_synthetic(seed=78, n=300000, hkls=hk)
        rec = e.download_db(0, 100000)
        for k in range(12):
            g = synth.pick_grains(rec, int(rng.integers(1, 21)), 8, rng)
            e.load_image(k, synth.render_image(rec[g], p.nr_px_x, p.nr_px_y, rng,
                                               threshold=None if k == 3 else 20.0))
        e.set_tuning(variant=1)
        e.match(range(12), p.min_nr_spots, p.min_intensity)
        ref = e.results_batch(range(12))
        for shape in ({}, {"consumers": 4}, {"consumers": 17, "stages": 2}, {"grid_mult": 3},
                      {"full_gather": 1}, {"consumers": 3, "stages": 2, "grid_mult": 6},
                      {"consumers": 3, "stages": 2, "grid_mult": 6, "full_gather": 1},
                      {"consumers": 3, "stages": 2, "grid_mult": 7},
                      {"consumers": 3, "stages": 2, "grid_mult": 8},
                      {"consumers": 3, "stages": 2, "grid_mult": 8, "full_gather": 1}):
            e.set_tuning(variant=2, **shape)
            e.match(range(12), p.min_nr_spots, p.min_intensity)
            got = e.results_batch(range(12))
            for k in range(12):
                assert got[k][1] == ref[k][1] and np.array_equal(got[k][0], ref[k][0])
        # the cell-mask pass (variant 4) under several shapes
        for shape in ({}, {"consumers": 4}, {"consumers": 12, "stages": 2}, {"stages": 3},
                      {"full_gather": 1}, {"consumers": 1}, {"cell_queue": 1},
                      {"cell_queue": 1, "consumers": 11}, {"cell_queue": 1, "full_gather": 1}):
            e.set_tuning(variant=4, **shape)
            e.match(range(12), p.min_nr_spots, p.min_intensity)
            got = e.results_batch(range(12))
            assert e.get_tuning()["last_variant"] == 4
            for k in range(12):
                assert got[k][1] == ref[k][1] and np.array_equal(got[k][0], ref[k][0])
        # the two-kernel cell-mask pass (variant 5): filter then count
        for shape in ({}, {"stages": 6, "consumers": 24}, {"stages": 8, "consumers": 8},
                      {"stages": 3, "consumers": 6}, {"stages": 1, "consumers": 1},
                      {"full_gather": 1}):
            for _ in range(2):  # eager, then graph replay (candidate buffer reused)
                e.set_tuning(variant=5, **shape)
                e.match(range(12), p.min_nr_spots, p.min_intensity)
                got = e.results_batch(range(12))
                assert e.get_tuning()["last_variant"] == 5
                for k in range(12):
                    assert got[k][1] == ref[k][1] and np.array_equal(got[k][0], ref[k][0])
        assert e.layout_info()["compact"] == 1


@pytest.mark.parametrize("n_rec", [30000, 150000])
def test_long_survivor_lists_are_ordered_like_the_oracle(n_rec):
    """Lists far longer than the ordering kernel's shared-memory tile (8192
    keys): ~21k and ~100k survivors in one slot, so the tile-wise network
    runs two and four size levels beyond the tile; ids ascending as the
    reference collects them (LaueMatchingCPU.c:781-788)."""
    txt = synth.params_text(nr_px=(256, 256), max_nr_spots=7, min_nr_spots=1,
                            min_intensity=1.0)
    p = P.parse_params_text(txt)
    rng = np.random.default_rng(n_rec)
    rec = np.zeros((n_rec, 15), np.uint16)
    rec[:, 0] = rng.integers(0, 8, n_rec)
    rec[:, 1::2] = rng.integers(0, 256, (n_rec, 7))
    rec[:, 2::2] = rng.integers(0, 256, (n_rec, 7))
    img = np.where(rng.random(256 * 256) < 0.4, rng.integers(1, 256, 256 * 256), 0)
    img = img.astype(np.float64)
    ref = O.compare(rec, p.max_nr_spots, img, p.nr_px_x, p.nr_px_y, p.min_nr_spots,
                    p.min_intensity)
    assert ref.ids.shape[0] > 2 * 8192
    with engine_for(p) as e:
        e.upload_db(rec)
        for slot in (0, 37):
            e.load_image(slot, img)
        e.match([0, 37], p.min_nr_spots, p.min_intensity)
        for slot in (0, 37):
            got, npass = e.results(slot)
            assert npass == ref.n_pass
            assert_same_survivors(got, ref)


def test_survivor_overflow_is_reported():
    c = golden_case("tilted_dense")
    p = c.params
    with engine_for(p, cap=64) as e:
        e.upload_db(c.records)
        e.load_image(0, c.image)
        e.match([0], p.min_nr_spots, p.min_intensity)
        with pytest.raises(OverflowError_):
            e.results(0)


def test_sparse_and_dense_uploads_agree_and_slots_reuse_cleanly():
    """Frames sent as (index, value) pairs give the same survivors as dense
    frames, for every dtype, and a slot reloaded many times (sparse after
    dense after sparse) holds only its latest frame."""
    c = golden_case("tilted_fcc")
    p = c.params
    rng = np.random.default_rng(4)
    frames = [c.image, c.image * 0.37, c.image.astype(np.float32), c.img_u8]
    other = synth.render_image(c.records[rng.choice(np.nonzero(c.records[:, 0] >= 8)[0], 3)],
                               p.nr_px_x, p.nr_px_y, rng)
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.set_sparse_uploads(False)
        refs = []
        for f in frames:
            e.load_image(0, f)
            e.match([0], p.min_nr_spots, p.min_intensity)
            refs.append(e.results(0))
        e.set_sparse_uploads(True)
        for k, f in enumerate(frames):
            e.load_image(3, other)  # previous content of the slot
            e.load_image(3, f)
            e.match([3], p.min_nr_spots, p.min_intensity)
            got = e.results(3)
            assert got[1] == refs[k][1] and np.array_equal(got[0], refs[k][0])
        # dense frame into a slot last used by a sparse one, and back
        dense = c.image + 3.0  # every pixel positive: sent dense
        e.load_image(3, dense)
        e.set_sparse_uploads(False)
        e.load_image(4, dense)
        e.set_sparse_uploads(True)
        e.match([3, 4], p.min_nr_spots, p.min_intensity)
        a, b = e.results(3), e.results(4)
        assert a[1] == b[1] and np.array_equal(a[0], b[0])
        e.load_image(3, c.image)
        e.match([3], p.min_nr_spots, p.min_intensity)
        got = e.results(3)
        assert got[1] == refs[0][1] and np.array_equal(got[0], refs[0][0])


@pytest.mark.parametrize("dtype", [np.uint8, np.float32, np.float64])
def test_batched_frame_loads_equal_single_loads(dtype):
    """load_images (one host scan per frame, one copy, two kernels per batch)
    leaves every slot as load_image does: same survivors, same imScale, for
    sparse frames, a dense frame in the same batch, batches of 1..3 frames
    (several scan segments per frame) and slots that held other frames."""
    c = golden_case("tilted_fcc")
    p = c.params
    rng = np.random.default_rng(8)
    base = [c.image, c.image * 0.37, c.image * 3.0 + 0.0]
    other = synth.render_image(c.records[rng.choice(np.nonzero(c.records[:, 0] >= 8)[0], 4)],
                               p.nr_px_x, p.nr_px_y, rng)
    frames = [f.astype(dtype) if dtype != np.uint8 else np.clip(f, 0, 255).astype(np.uint8)
              for f in base + [other]]
    dense = np.clip(frames[0].astype(np.float64) + 2.0, 0, 255).astype(dtype)  # all positive
    frames.append(dense)
    with engine_for(p) as e:
        e.upload_db(c.records)
        singles, scales = [], []
        for f in frames:
            scales.append(e.load_image(0, f))
            e.match([0], p.min_nr_spots, p.min_intensity)
            singles.append(e.results(0))
        # previous content in every target slot
        for s in (1, 2, 5, 40, 63):
            e.load_image(s, other.astype(dtype) if dtype != np.uint8 else
                         np.clip(other, 0, 255).astype(np.uint8))
        got_sc = e.load_images([63, 1, 40, 2, 5], frames, want_scales=True)
        assert got_sc == scales
        e.match([1, 2, 5, 40, 63], p.min_nr_spots, p.min_intensity)
        res = e.results_batch([63, 1, 40, 2, 5])
        for i, s in enumerate([63, 1, 40, 2, 5]):
            assert res[s][1] == singles[i][1] and np.array_equal(res[s][0], singles[i][0])
        for k in (1, 2, 3):  # small batches: a frame split over scan segments
            e.load_images(list(range(10, 10 + k)), frames[:k])
            e.match(range(10, 10 + k), p.min_nr_spots, p.min_intensity)
            for i in range(k):
                r = e.results(10 + i)
                assert r[1] == singles[i][1] and np.array_equal(r[0], singles[i][0])
        with pytest.raises(LmbError):
            e.load_images([3, 3], frames[:2])


@pytest.mark.parametrize("share", [0.0, 0.34, 1.0])
def test_dense_share_of_pinned_frames_gives_same_results(share):
    """Pinned frames sent dense over the copy engine (a share of each batch)
    while the host scans the rest: same survivors as single loads."""
    from lauematching_b200.engine import PinnedBuffer
    c = golden_case("tilted_fcc")
    p = c.params
    npx = p.nr_px_x * p.nr_px_y
    rng = np.random.default_rng(12)
    frames = []
    for k in range(6):
        img = synth.render_image(c.records[rng.choice(np.nonzero(c.records[:, 0] >= 8)[0], 3)],
                                 p.nr_px_x, p.nr_px_y, rng)
        frames.append(np.clip(img, 0, 255).astype(np.uint8))
    pins = []
    for f in frames:
        pb = PinnedBuffer((npx,), np.uint8)
        pb.array[:] = f.ravel()
        pins.append(pb)
    with engine_for(p) as e:
        e.upload_db(c.records)
        singles = []
        for f in frames:
            e.load_image(0, f)
            e.match([0], p.min_nr_spots, p.min_intensity)
            singles.append(e.results(0))
        e.set_dense_share(share)
        for rep in range(2):  # slots reloaded: previous content replaced either way
            order = list(range(6))[::-1] if rep else list(range(6))
            e.load_images(list(range(10, 16)), [pins[k].array for k in order])
            e.match(range(10, 16), p.min_nr_spots, p.min_intensity)
            got = e.results_batch(range(10, 16))
            for i, k in enumerate(order):
                assert got[10 + i][1] == singles[k][1]
                assert np.array_equal(got[10 + i][0], singles[k][0])
    for pb in pins:
        pb.free()


def test_queued_passes_keep_each_slots_results():
    """A pass over other slots queued before the previous pass's results are
    read leaves those results intact; a slot's results are those of the last
    pass that included it; a slot never matched has none."""
    c = golden_case("tilted_dense")
    p = c.params
    scales = (1.0, 0.5, 2.0, 0.25)
    with engine_for(p) as e:
        e.upload_db(c.records)
        for k, s in enumerate(scales):
            e.load_image(k, c.image * s)
        alone = {}
        for k in range(4):
            e.match([k], p.min_nr_spots, p.min_intensity)
            alone[k] = e.results(k)
        for _ in range(3):  # more passes in flight than status entries are kept
            e.match([0, 1], p.min_nr_spots, p.min_intensity)
            e.match([2], p.min_nr_spots, p.min_intensity)
            e.match([3], p.min_nr_spots, p.min_intensity)
        got = e.results_batch([3, 0, 2, 1])
        for k in range(4):
            assert got[k][1] == alone[k][1] and np.array_equal(got[k][0], alone[k][0])
        e.match([2], p.min_nr_spots, 1e12)  # slot 2 again: nothing passes
        assert e.results(2)[1] == 0
        r0 = e.results(0)
        assert r0[1] == alone[0][1] and np.array_equal(r0[0], alone[0][0])
        e.load_image(9, c.image)
        with pytest.raises(LmbError):
            e.results(9)


def test_byte_counters_follow_the_copies():
    """lmb_engine_bytes: a dense frame adds its size, a sparse one its
    (index, value) pairs, a pass its status words, results their survivors."""
    c = golden_case("tilted_fcc")
    p = c.params
    npx = p.nr_px_x * p.nr_px_y
    nnz = int(np.count_nonzero(c.img_u8))
    with engine_for(p) as e:
        e.upload_db(c.records)
        h0, d0 = e.bytes_moved()
        assert h0 == c.records.nbytes
        e.set_sparse_uploads(False)
        e.load_image(0, c.img_u8, want_scale=False)
        h1, _ = e.bytes_moved()
        assert h1 - h0 == npx
        e.set_sparse_uploads(True)
        e.load_image(1, c.img_u8, want_scale=False)
        h2, _ = e.bytes_moved()
        assert 0 < h2 - h1 < npx and h2 - h1 >= 5 * nnz
        e.match([0, 1], p.min_nr_spots, p.min_intensity)
        _, d1 = e.bytes_moved()
        assert d1 - d0 == (2 * 64 + 1) * 4
        got = e.results_batch([0, 1])
        _, d2 = e.bytes_moved()
        assert d2 - d1 == sum(r.nbytes for r, _ in got.values())


def test_repeated_pass_replays_graph_with_same_results():
    """The first pass of a configuration runs eagerly, the second is captured
    into a CUDA graph, later ones replay it: results and timings stay valid."""
    c = golden_case("tilted_dense")
    p = c.params
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity)
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(2, c.image)
        e.load_image(9, c.image * 0.5)
        for it in range(5):
            e.match([2, 9], p.min_nr_spots, p.min_intensity)
            got, npass = e.results(2)
            assert npass == ref.n_pass
            assert_same_survivors(got, ref)
            cmp_ms, ord_ms = e.last_pass_ms()
            assert cmp_ms > 0 and ord_ms >= 0
        e.load_image(2, c.image * 0.25)  # new frame, same configuration: graph replays
        e.match([2, 9], p.min_nr_spots, p.min_intensity)
        got, npass = e.results(2)
        ref2 = O.compare(c.records, p.max_nr_spots, c.image * 0.25, p.nr_px_x, p.nr_px_y,
                         p.min_nr_spots, p.min_intensity)
        assert npass == ref2.n_pass
        assert_same_survivors(got, ref2)


def test_errors_are_reported_not_silent():
    c = golden_case("tilted_fcc")
    with engine_for(c.params) as e:
        with pytest.raises(LmbError):
            e.match([3], 5, 1.0)  # slot 3 holds no image
        with pytest.raises(LmbError):
            e.load_image(64, c.image)


def test_hexagonal_fundamental_zone_db_build():
    """Synthetic DB restricted to the hexagonal fundamental zone: each device
    rotation is the host reduction (synth.hexagonal_fundamental_zone) of the
    plain generator's rotation with the same ID, to rounding; it is one of
    the 12 equivalents of that rotation; and the records built from the zone
    rotations equal the oracle's forward simulation of them, byte for byte
    (hexagonal SG 194, 7790 HKLs)."""
    txt = synth.params_text(lattice=(0.295, 0.295, 0.468, 90, 90, 120), space_group=194,
                            max_nr_spots=30, min_nr_spots=5)
    p = P.parse_params_text(txt)
    hk = synth.hkls_hexagonal(10)
    n = 20000
    with engine_for(p) as e:
        om_fz = e.build_db_synthetic(seed=3, n=n, hkls=hk, return_orients=True, hex_fz=True)
        rec = e.download_db()
        assert np.array_equal(e.synth_orientations(3, 0, n), om_fz)
        plain = e.synth_orientations(3, 0, n, hex_fz=False)
    host = synth.hexagonal_fundamental_zone(plain)
    # the host reduction recovers the quaternion from the matrix (square roots
    # of small diagonal sums) and loses a few ulps more than the device's path
    assert np.max(np.abs(host - om_fz)) < 1e-10
    # an equivalent rotation: R_fz = R_plain . S for a symmetry operator S
    m_fz, m_pl = om_fz.reshape(-1, 3, 3), plain.reshape(-1, 3, 3)
    rel = np.einsum("nji,njk->nik", m_pl, m_fz)  # R_plain^T R_fz
    tr = np.clip((np.trace(rel, axis1=1, axis2=2) - 1) / 2, -1, 1)
    ang = np.degrees(np.arccos(tr))
    assert np.all(np.min(np.abs(ang[:, None] - np.array([0, 60, 120, 180])[None]), 1) < 1e-3)
    assert np.array_equal(rec, O.forward(p, om_fz, hk))


@pytest.mark.parametrize("variant", [2, 4])
def test_a_consumer_wait_that_runs_out_reports_a_timeout(variant):
    """The compare pass's waits are bounded.  A test wait (1 ms on a barrier
    nothing arrives at) makes the consumers give up; the producer's own wait
    for a free ring slot then runs out after its full bound and it waits for
    its own copies before returning.  The pass reports LMB_ERR_TIMEOUT (and
    keeps reporting it: the device error word is sticky), and the device
    stays usable: a new engine on it matches the oracle."""
    from lauematching_b200._lib import TimeoutError_
    c = golden_case("tilted_fcc")
    p = c.params
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity)
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(0, c.image)
        e.set_tuning(variant=variant, test_consumer_wait_us=1000)
        e.match([0], p.min_nr_spots, p.min_intensity)
        with pytest.raises(TimeoutError_):
            e.results(0)
        assert e.get_tuning()["last_variant"] == variant
    with engine_for(p) as e:
        e.upload_db(c.records)
        e.load_image(0, c.image)
        e.match([0], p.min_nr_spots, p.min_intensity)
        got, npass = e.results(0)
    assert npass == ref.n_pass
    assert_same_survivors(got, ref)
