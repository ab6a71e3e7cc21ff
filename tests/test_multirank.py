"""The multi-rank host logic on CPU: two `gloo` ranks, as bench.py runs them under torchrun.

The path has no cross-GPU exchange: independent problems are sharded across ranks by a
deterministic greedy rule that every rank evaluates on its own, and the only collectives are
the barrier and the max-over-ranks of the timing.  These tests check that both ranks compute
the same disjoint, covering, balanced assignment, and that the max reduction is correct.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    for p in (ROOT, os.path.join(ROOT, "computation-suite_b200")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from feab200 import cantilever
        from feab200.batched import problem_cost, shard_problems
        probs = cantilever.batch_cantilevers(256)
        costs = [problem_cost(len(p.mesh.nodes), p.F.shape[1]) for p in probs]
        shards = shard_problems(costs, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, [s.tolist() for s in shards])
        bench.barrier(world)
        t_max = bench.max_over_ranks(10.0 + rank, world)
        out.put((rank, gathered, shards[rank].tolist(), costs, t_max))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards_and_max():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    views = res[0][1]                       # every rank's assignment, gathered on rank 0
    assert res[1][1] == views and views[0] == views[1]                # same assignment on every rank
    shards = views[0]
    allidx = sorted(i for s in shards for i in s)
    assert allidx == list(range(256))                                 # covering and disjoint
    costs = np.asarray(res[0][3])
    loads = [costs[s].sum() for s in shards]
    assert max(loads) / min(loads) < 1.02                            # greedy balance
    assert res[0][2] == shards[0] and res[1][2] == shards[1]
    assert res[0][4] == res[1][4] == 11.0                            # max over ranks


@pytest.mark.parametrize("world", [1, 3, 8])
def test_shard_rule_properties(world):
    from feab200.batched import shard_problems
    rng = np.random.default_rng(7)
    costs = rng.integers(1, 1000, 57).astype(float)
    shards = shard_problems(costs, world)
    assert len(shards) == world
    assert sorted(np.concatenate(shards).tolist()) == list(range(57))
    # longest-processing-time bound: max load <= (4/3 - 1/(3w)) * optimum <= that * mean-or-max
    lower = max(costs.sum() / world, costs.max())
    assert max(costs[s].sum() for s in shards) <= (4 / 3) * lower + 1e-9
    assert all(np.array_equal(a, b) for a, b in zip(shards, shard_problems(costs, world)))   # deterministic
