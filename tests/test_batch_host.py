"""Host logic of the batched form (no GPU): the seeded scene generator, the
world boxes of the segmented grid, and the split of scenes over ranks, run
as two gloo ranks."""

import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fluid_simulation_b200.batch import TANK, make_batch, shard_scenes, sub_batch


def test_generator_is_seeded_and_in_range():
    a = make_batch(n_scenes=16, seed=3)
    b = make_batch(n_scenes=16, seed=3)
    c = make_batch(n_scenes=16, seed=4)
    assert all(np.array_equal(x.x, y.x) for x, y in zip(a.scenes, b.scenes))
    assert not np.array_equal(a.scenes[0].x, c.scenes[0].x)
    for s in a.scenes:
        assert 0.2 <= s.column_fraction <= 0.6
        assert 0.8 * 2.5e5 <= s.stiffness <= 1.2 * 2.5e5
        assert 0.8e-6 <= s.viscosity <= 1.2e-6
        # a few lattice-rounding percent around the log-uniform draw range
        assert 0.8 * 2000 <= s.count <= 1.2 * 100000
        w, h, l = s.walls
        assert np.isclose(w / l, TANK[0] / TANK[2]) and np.isclose(h / l, TANK[1] / TANK[2])
        assert np.all(np.abs(s.x[:, 0]) <= w) and np.all(np.abs(s.x[:, 1]) <= h)
        assert np.all(s.x[:, 2] >= 0) and np.all(s.x[:, 2] <= 2 * l)
        # the column occupies the low-x fraction of the tank
        assert s.x[:, 0].max() <= -w + 2 * w * s.column_fraction + a.spacing


def test_default_batch_is_about_six_million_particles():
    b = make_batch()
    assert len(b.scenes) == 256
    assert 5.0e6 < b.total < 7.5e6
    assert b.world().shape == (b.total,)
    assert np.array_equal(np.bincount(b.world()), b.counts)


def test_world_boxes_cover_each_tank():
    """The cell coordinates int(x / h) of the tank's points span the box less
    its one-cell margin; points up to one cell width outside the tank (where
    DFSPH's mid-substep positions can lie) stay inside the box."""
    b = make_batch(n_scenes=8, seed=1)
    inv = np.float32(1.0) / np.float32(b.h)
    for s, (clo, dims, walls) in zip(b.scenes, b.boxes()):
        w, h, l = s.walls
        assert walls == s.walls
        for k, (a, e) in enumerate(((-w, w), (-h, h), (0.0, 2.0 * l))):
            pts = np.linspace(a, e, 1001).astype(np.float32)
            c = np.trunc(pts * inv).astype(np.int64)
            assert c.min() == clo[k] + 1 and c.max() == clo[k] + dims[k] - 2
            out = np.array([a - 0.999 * b.h, e + 0.999 * b.h], np.float32)
            c = np.trunc(out * inv).astype(np.int64)
            assert c.min() >= clo[k] and c.max() <= clo[k] + dims[k] - 1
    assert all(d == tuple(x - 2 for x in dm) for (_, d, _), (_, dm, _) in zip(b.boxes(margin=0), b.boxes()))


def test_shard_scenes_partitions_and_balances():
    counts = make_batch(n_scenes=64, seed=2).counts
    for ws in (1, 2, 3, 8):
        parts = shard_scenes(counts, ws)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(counts)))
        loads = [counts[p].sum() for p in parts]
        assert max(loads) - min(loads) <= counts.max()


def _rank_main(rank, world_size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        b = make_batch(n_scenes=24, seed=5, n_lo=500, n_hi=4000)
        mine = shard_scenes(b.counts, world_size)[rank]
        local = sub_batch(b, mine)
        # each rank owns whole scenes: its worlds are renumbered 0..k-1 locally
        assert np.array_equal(np.unique(local.world()), np.arange(len(mine)))
        t = torch.tensor([local.total, len(mine)], dtype=torch.int64)
        dist.all_reduce(t)
        ids = [None] * world_size
        dist.all_gather_object(ids, mine)
        if rank == 0:
            out.put((int(t[0]), int(t[1]), ids, b.total))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_scenes_without_overlap():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    total, nscenes, ids, want = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert total == want and nscenes == 24
    assert not set(ids[0]) & set(ids[1])
