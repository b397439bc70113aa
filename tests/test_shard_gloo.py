"""Multi-rank layout on CPU (gloo, world size 2): the DB split by ID range,
each rank matches its range, the gathered survivor list equals the
single-process list.  The per-rank matching runs on the oracle here (no GPU);
on B200 each rank runs the same split with its own engine."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, golden_case
from lauematching_b200.shard import merge_rank_survivors, shard_range


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            rs = [shard_range(n, r, w) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[i][1] == rs[i + 1][0] for i in range(w - 1))
            assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, name, out_path):
    import sys
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    import oracle as O
    from conftest import golden_case as gc
    from lauematching_b200.shard import gather_survivors, shard_range as sr
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    c = gc(name)
    p = c.params
    a, b = sr(c.records.shape[0], rank, world)
    s = O.compare(c.records[a:b], p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                  p.min_nr_spots, p.min_intensity, nthreads=1)
    local = np.zeros(len(s.ids), [("id", "<u8"), ("n_spots", "<i4"), ("score", "<f8")])
    local["id"], local["n_spots"], local["score"] = s.ids, s.n_spots, s.score
    merged, total = gather_survivors(local, s.n_pass, a)
    if rank == 0:
        np.savez(out_path, merged=merged, total=total)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name", ["tilted_dense"])
def test_two_rank_db_split_equals_single_process(tmp_path, name):
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), name, out), nprocs=2,
                       start_method="spawn")
    got = np.load(out)
    c = golden_case(name)
    p = c.params
    import oracle as O
    ref = O.compare(c.records, p.max_nr_spots, c.image, p.nr_px_x, p.nr_px_y,
                    p.min_nr_spots, p.min_intensity)
    m = got["merged"]
    assert int(got["total"]) == ref.n_pass
    assert np.array_equal(m["id"], ref.ids.astype(np.uint64))
    assert np.array_equal(m["n_spots"], ref.n_spots)
    assert np.array_equal(m["score"].view(np.uint64), ref.score.view(np.uint64))


def test_merge_rank_survivors_offsets():
    a = np.zeros(2, [("id", "<u8")])
    a["id"] = [1, 5]
    b = np.zeros(1, [("id", "<u8")])
    b["id"] = [0]
    m = merge_rank_survivors([a, b], [0, 10])
    assert m["id"].tolist() == [1, 5, 10]
