"""Sharding the batched workload over ranks (one process per GPU), on CPU.

Graphs are independent, so each rank takes a share computed on its own (no
collective on the data path) and only the timing is reduced, as the maximum
over ranks.  Two gloo ranks check that both compute the same split, that the
split covers every graph once and is balanced, and the max-over-ranks time
reduction that bench.py uses."""
import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_graph_once_and_balances():
    from gpugraphlayout_b200 import shard
    rng = np.random.default_rng(0)
    costs = list(rng.integers(50, 20000, 4096))
    for world in (1, 2, 3, 8):
        parts = shard.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-first greedy: within one item of the mean
        assert max(loads) - min(loads) <= max(costs)
        assert shard.partition(costs, world) == parts  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    import datetime

    import torch
    import torch.distributed as dist

    from gpugraphlayout_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        parts = shard.partition(costs, world)
        mine = parts[rank]
        # every rank's own view of the split, gathered for the check
        seen = [None] * world
        dist.all_gather_object(seen, mine)
        # the bench's timing reduction: max over ranks
        t = torch.tensor([float(100 + 10 * rank)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, seen, parts, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split_and_the_max_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    costs = [int(c) for c in np.random.default_rng(1).integers(50, 20000, 300)]
    port = _free_port()
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    (_, seen0, parts0, t0), (_, seen1, parts1, t1) = results
    assert parts0 == parts1
    assert seen0 == seen1 == parts0
    assert sorted(i for p in parts0 for i in p) == list(range(len(costs)))
    assert t0 == t1 == 110.0


def _batch_graphs():
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    sizes = [60, 420, 130, 800, 75, 300, 510, 90, 240, 660]
    out = []
    for i, n in enumerate(sizes):
        s, t = synth.sbm_edges(n, 2 + i % 5, 0.05, 0.002, 40.0, seed=70 + i)
        out.append(O.Graph(s, t))
    return out


def _layout(g, i, steps=4):
    """The oracle's iterations of graph i of the batch (weak gravity,
    scale 2, the batched workload's settings) from its own start."""
    from oracle import oracle as O
    xy = O.random_positions(g.n, 10000.0, 10000.0, 1234 + i)
    fo = O.FA2(g, xy, 2.0, 1.0, False)
    fo.step(steps)
    return fo.positions


def _rank_layouts(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from gpugraphlayout_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        graphs = _batch_graphs()
        costs = [g.n + g.m for g in graphs]
        mine = shard.partition(costs, world)[rank]
        # each rank lays out only its own graphs; positions travel once, at
        # the end (the only exchange of the sharded batch)
        local = {i: _layout(graphs[i], i).tobytes() for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        if rank == 0:
            union = {}
            for part in gathered:
                assert not set(part) & set(union)
                union.update(part)
            q.put(union)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_lay_out_their_shards_like_one_process():
    """Two ranks each run the oracle's iterations over their share of a
    batch; the gathered positions are bit for bit those of one process
    laying out every graph."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_layouts, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    union = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    graphs = _batch_graphs()
    assert sorted(union) == list(range(len(graphs)))
    for i, g in enumerate(graphs):
        assert union[i] == _layout(g, i).tobytes(), i
