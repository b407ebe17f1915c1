"""Sharding of a batch of independent worlds over ranks (the multi-GPU form of
the batched step): partitions are contiguous, complete, balanced by body
count, and each rank's slice is exactly its worlds' bodies.  The N>1 path is
exercised with world_size-2 gloo process groups on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nativeengine_b200 import scenes
from nativeengine_b200.bodies import concat, take_range
from nativeengine_b200.shard import partition_worlds, slice_bodies


def _batch():
    params, bodies, begin, _ = scenes.batch_mix(nworlds=9, lo=16, hi=200, seed=21)
    return params, bodies, begin


def test_partition_is_contiguous_complete_and_balanced():
    begin = np.array([0, 10, 30, 31, 80, 200, 260, 300], dtype=np.int64)
    for nranks in (1, 2, 3, 4, 7, 9):
        parts = partition_worlds(begin, nranks)
        assert len(parts) == nranks
        assert parts[0][0] == 0 and parts[-1][1] == len(begin) - 1
        for (a0, a1), (b0, b1) in zip(parts, parts[1:]):
            assert a1 == b0 and a0 <= a1
    loads = [begin[w1] - begin[w0] for w0, w1 in partition_worlds(begin, 2)]
    assert max(loads) <= begin[-1] // 2 + 120   # off by at most one world


def test_slices_reassemble_the_batch():
    params, bodies, begin = _batch()
    parts = [slice_bodies(bodies, begin, w0, w1) for w0, w1 in partition_worlds(begin, 3)]
    whole, shard_begin = concat([p for p, _ in parts])
    ranges = np.concatenate([pb[:-1].astype(np.int64) + sb for (_, pb), sb in zip(parts, shard_begin[:-1])]
                            + [np.array([bodies.n])])
    assert np.array_equal(ranges, begin.astype(np.int64))
    for k in ("x", "q", "v", "w", "inv_mass", "shape", "half_extents", "flags"):
        assert np.array_equal(getattr(whole, k), getattr(bodies, k)), k
    assert whole.n_verts == bodies.n_verts


def test_take_range_rebases_convex_vertices():
    from nativeengine_b200.scenes import mixed_shapes
    _, b = mixed_shapes(n=40, seed=3)
    part = take_range(b, 10, 30)
    for i in range(20):
        c = int(part.vert_count[i])
        if c:
            o = int(part.vert_offset[i])
            o0 = int(b.vert_offset[10 + i])
            assert np.array_equal(part.verts[o:o + c], b.verts[o0:o0 + c])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, bodies, begin = _batch()
        w0, w1 = partition_worlds(begin, world)[rank]
        part, pbegin = slice_bodies(bodies, begin, w0, w1)
        assert len(params[w0:w1]) == len(pbegin) - 1
        mine = torch.tensor([w0, w1, part.n, float(part.x.sum())], dtype=torch.float64)
        got = [torch.zeros(4, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(got, mine)
        # timing reduction used by the bench: max over ranks
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put(([g.tolist() for g in got], float(t[0])))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_shards_cover_the_batch_with_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got, tmax = out.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    params, bodies, begin = _batch()
    (a0, a1, an, ax), (b0, b1, bn, bx) = got
    assert a0 == 0 and a1 == b0 and b1 == len(begin) - 1
    assert an + bn == bodies.n
    assert abs((ax + bx) - float(bodies.x.sum())) < 1e-9 * max(1.0, abs(float(bodies.x.sum())))
    assert tmax == 2.0
