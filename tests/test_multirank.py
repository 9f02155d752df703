"""The multi-GPU form is replicas only: every rank refines its own meshes and
the only collectives are the timing reductions.  These run as two gloo ranks
on the CPU: max-over-ranks timing, and the partition of the batched workload
(every mesh on exactly one rank, the predicted work balanced)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    from slak_b200 import shard
    t = bench._max_over_ranks(dist, 1.5 + rank)
    bench._barrier(dist)
    sizes = [(it.kind, it.faces, it.levels, it.seed) for it in bench.batch_shard(2000, rank, ws)]
    # the library call a user makes: rank and world size from the process group
    r, w = shard.rank_and_world()
    mine = shard.shard_indices(_WORK, r, w)
    q.put((rank, t, sizes, (r, w, mine)))
    dist.destroy_process_group()


# predicted output of a small uneven batch (nnz x 4^(levels-1))
_WORK = [4000 * 4 ** 3, 120, 98_000, 98_000, 5, 0, 700 * 4 ** 2, 33_000 * 4, 1, 64_000]


def test_two_gloo_ranks_time_and_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [t for _, t, _, _ in res] == [2.5, 2.5]          # max over ranks, seen by both
    lib = [x for _, _, _, x in res]
    assert [(r, w) for r, w, _ in lib] == [(0, 2), (1, 2)]
    assert sorted(lib[0][2] + lib[1][2]) == list(range(len(_WORK)))
    assert all(x == sorted(x) for _, _, x in lib)
    loads = [sum(_WORK[k] for k in x) for _, _, x in lib]
    assert abs(loads[0] - loads[1]) <= max(_WORK)
    sys.path.insert(0, ROOT)
    import bench
    whole = [(it.kind, it.faces, it.levels, it.seed) for it in bench.batch_shard(2000)]
    shards = [s for _, _, s, _ in res]
    assert len(shards[0]) + len(shards[1]) == len(whole)
    assert sorted(shards[0] + shards[1]) == sorted(whole)          # a partition of the batch
    for sh in shards:                                               # each shard keeps batch order
        assert sh == [it for it in whole if it in sh]
    work = [sum(f * 4 ** (lv - 1) for _, f, lv, _ in sh) for sh in shards]
    biggest = max(f * 4 ** (lv - 1) for _, f, lv, _ in whole)
    assert abs(work[0] - work[1]) <= biggest                        # balanced to within one mesh


@pytest.mark.parametrize("ws", [3, 4, 8])
def test_partition_at_more_ranks(ws):
    """The 2,000-mesh batch split over ws ranks (as `bench.py --gpus ws` does):
    a partition, each shard in batch order, predicted work within one mesh."""
    sys.path.insert(0, ROOT)
    import bench
    key = lambda it: (it.kind, it.faces, it.levels, it.seed)
    whole = [key(it) for it in bench.batch_shard(2000)]
    shards = [[key(it) for it in bench.batch_shard(2000, r, ws)] for r in range(ws)]
    assert sorted(sum(shards, [])) == sorted(whole)
    for sh in shards:
        assert sh == [it for it in whole if it in set(sh)]
    work = [sum(f * 4 ** (lv - 1) for _, f, lv, _ in sh) for sh in shards]
    biggest = max(f * 4 ** (lv - 1) for _, f, lv, _ in whole)
    assert max(work) - min(work) <= biggest


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun, `bench.py --impl reference` does its work on rank 0;
    every other rank returns at once, with nothing to print."""
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    args = argparse.Namespace(scheme="slak", workload="mixed512", steps=1, warmup=3, cpu_budget=1.0,
                              crease_frac=0.0, batch_count=10)
    assert bench.run_reference(args, None, 1, 2) is None


def test_partition_edge_cases():
    sys.path.insert(0, ROOT)
    from slak_b200 import shard
    assert shard.partition([], 4) == []
    assert shard.partition([7, 7, 7], 5) == [0, 1, 2]            # more ranks than meshes: the rest idle
    assert shard.shard_indices([7, 7, 7], 4, 5) == []
    assert shard.partition([5, 9, 1], 1) == [0, 0, 0]
    assert shard.predicted_quads(1000, 1) == 1000 and shard.predicted_quads(1000, 3) == 16000
    assert shard.predicted_quads(1000, 0) == 0
    for bad in (lambda: shard.partition([1], 0), lambda: shard.partition([-1], 2),
                lambda: shard.shard_indices([1], 2, 2)):
        with pytest.raises(ValueError):
            bad()
