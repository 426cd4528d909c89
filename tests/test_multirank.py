"""The N>1 path without GPUs: two gloo ranks on the CPU partition a batched ensemble by scene
through pe_b200.shard (each scene on exactly one rank, loads balanced) and combine their timings
the way the benchmark does (max of the device times, sum of the spheres)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    from pe_b200 import scenes
    from pe_b200.shard import local_scenes, shard_scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ens = scenes.batched_ensemble(0, scenes=40, nmin=64, nmax=1024)
        mine = local_scenes(ens)
        assert [s.name for s in mine] == [s.name for s in shard_scenes(ens, rank, world)]
        names = [None] * world
        dist.all_gather_object(names, [s.name for s in mine])
        # the benchmark's reductions: max of the per-rank times, sum of the per-rank spheres
        t = torch.tensor([1.0 + rank], dtype=torch.float64)
        n = torch.tensor([float(sum(s.n for s in mine))], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        if rank == 0:
            out.put((names, float(t.item()), float(n.item()), [s.name for s in ens],
                     sum(s.n for s in ens), {s.name: s.n for s in ens}))
    finally:
        dist.destroy_process_group()


def test_ensemble_partition_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        names, tmax, ntot, all_names, all_n, sizes = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    a, b = set(names[0]), set(names[1])
    assert not (a & b) and (a | b) == set(all_names)
    assert tmax == 2.0 and ntot == all_n
    la, lb = sum(sizes[k] for k in a), sum(sizes[k] for k in b)
    assert abs(la - lb) <= max(sizes.values())   # greedy largest-first balance


def test_shard_scenes_single_rank_keeps_everything():
    import sys
    sys.path.insert(0, ROOT)
    from pe_b200 import scenes
    from pe_b200.shard import local_scenes, shard_scenes
    ens = scenes.batched_ensemble(1, scenes=10, nmin=64, nmax=256)
    want = [s.name for s in sorted(ens, key=lambda s: -s.n)]
    assert [s.name for s in shard_scenes(ens, 0, 1)] == want
    assert [s.name for s in local_scenes(ens)] == want   # no process group: everything
    with pytest.raises(ValueError):
        shard_scenes(ens, 2, 2)


def test_bench_uses_the_library_partition():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    from pe_b200 import shard
    assert bench.shard_scenes is shard.shard_scenes
