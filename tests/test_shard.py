"""Multi-GPU sharding logic, exercised on the CPU: two gloo ranks each run the
CPU oracle on their contiguous shard of a golden case's sky points; the
records gathered in rank order must equal the single-process run's."""
import os
import socket

import numpy as np
import pytest

from tdfstat_b200 import shard


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 1024):
        for w in (1, 2, 3, 8):
            rs = [shard.shard_range(n, r, w) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[i][1] == rs[i + 1][0] for i in range(w - 1))
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)


def test_balanced_ranges():
    costs = [1, 1, 1, 10, 1, 1, 1, 1]
    rs = shard.balanced_ranges(costs, 2)
    assert rs[0][0] == 0 and rs[-1][1] == len(costs) and rs[0][1] == rs[1][0]
    c = np.cumsum(costs)
    part0 = c[rs[0][1] - 1] if rs[0][1] else 0
    assert abs(part0 - (c[-1] - part0)) <= 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, ini, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, here)
    import torch.distributed as dist
    import refkit
    from tdfstat_b200 import host, shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    job = host.Job(ini, float_build=False)
    pm, mm, nn = job.sky_points()
    p, m, n = sh.shard_points(pm, mm, nn, rank, world)
    lib = refkit.load_oracle()
    st, rec, _ = refkit.search_points(lib.orc_search_points, job.segment(), job.search_opts(), p, m, n)
    part = (rec.hdr, np.array([len(x) for x in rec.pairs], np.int64),
            np.concatenate(rec.pairs) if rec.pairs else np.zeros(0, np.float32))
    parts = [None] * world
    dist.all_gather_object(parts, (st, part))
    if rank == 0:
        out_q.put(parts)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_merge_to_single_run(golden, oracle):
    import torch.multiprocessing as mp
    import refkit
    g = golden("g2_h1l1_inj")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, g.ini, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(st == 0 for st, _ in parts)
    hdr, lens, flat = shard.merge_records([p for _, p in parts])
    ref = g.ref["f64"]
    np.testing.assert_array_equal(hdr, ref.hdr)
    np.testing.assert_array_equal(lens, [len(x) for x in ref.pairs])
    np.testing.assert_array_equal(flat, np.concatenate(ref.pairs))


def test_assign_segments_partitions_and_balances():
    rng = np.random.default_rng(3)
    # the four segment sizes of the segmented workload, 64 segments, as costs
    sizes = [(86164, 131072), (129246, 131072), (172328, 262144), (258492, 262144)]
    costs = [shard.segment_cost(256 * 401, nf, 2, N) for N, nf in (sizes[k % 4] for k in range(64))]
    for world in (1, 2, 3, 4, 8):
        a = shard.assign_segments(costs, world)
        assert sorted(k for r in a for k in r) == list(range(64))
        assert all(r == sorted(r) for r in a)
        loads = [sum(costs[k] for k in r) for r in a]
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) + 1e-6
    rand = list(rng.uniform(1, 10, size=37))
    a = shard.assign_segments(rand, 5)
    loads = [sum(rand[k] for k in r) for r in a]
    assert max(loads) - min(loads) <= max(rand)
    assert shard.assign_segments([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.assign_segments([1.0], 0)


def _seg_worker(rank, world, port, costs, out_q):
    import torch.distributed as dist
    from tdfstat_b200 import shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = sh.assign_segments(costs, world)[rank]
    every = [None] * world
    dist.all_gather_object(every, mine)
    if rank == 0:
        out_q.put(every)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_disjoint_segments():
    """Every rank computes the same assignment on its own (no exchange); the
    ranks' segments are disjoint and cover all segments."""
    import torch.multiprocessing as mp
    costs = [shard.segment_cost(1000, 1 << (17 + (k % 2)), 2, 86164 * (1 + k % 3)) for k in range(11)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_seg_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    every = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(every[0] + every[1]) == list(range(11))
    assert not set(every[0]) & set(every[1])
