"""Multi-rank host logic on CPU (gloo, world size 2): ensemble sharding and the timing reduction.

Each rank builds its shard of the seeded instance stream and advances it with the oracle; the
shards are disjoint, their union is the global stream, and the max-over-ranks reduction used
for timing returns the largest per-rank value on every rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_per_rank, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    from datetime import timedelta

    from summationbyparts_b200 import sharding, workloads
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    first, n = sharding.weak_shard(n_per_rank, rank)
    insts = workloads.ensemble_instances(n, seed=1, first=first)
    # advance the two smallest instances of this shard a few steps on the oracle
    from oracle import oracle as orc
    small = sorted(insts, key=lambda i: i.side)[:2]
    errs = []
    for inst in small:
        b = workloads.ensemble_blocks([inst])[0]
        s = orc.System([dict(x=b.x, y=b.y, op_xi=inst.op_id, op_eta=inst.op_id, bc=list(b.bc))])
        s.set_vortex([dict(x0=inst.x0, y0=inst.y0, rstar=workloads.ENSEMBLE_RSTAR, eps=inst.eps)], inst.mach)
        s.init_vortex(0.0)
        s.advance(3, inst.dt)
        errs.append(s.error())
    mx = sharding.max_over_ranks(float(rank + 1) * 1.5, dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, [(i.side, i.x0) for i in insts], errs, mx))


@pytest.mark.timeout(300)
def test_two_rank_weak_sharding():
    world, n = 2, 6
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    from summationbyparts_b200 import workloads
    allinst = [(i.side, i.x0) for i in workloads.ensemble_instances(world * n, seed=1)]
    assert res[0][1] + res[1][1] == allinst
    for rank, _, errs, mx in res:
        assert mx == 3.0
        assert all(np.isfinite(e) and 0 < e < 1 for e in errs)


def test_balanced_partition_lpt():
    from summationbyparts_b200 import sharding, workloads
    insts = workloads.ensemble_instances(512, seed=1)
    costs = [sharding.instance_cost(i) for i in insts]
    for world in (1, 2, 4, 8):
        bins = sharding.balanced_partition(costs, world)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(512))
        loads = [sum(costs[i] for i in b) for b in bins]
        # LPT is within 4/3 of optimal; on this many items it is near perfect
        assert max(loads) <= (sum(costs) / world) * 1.02 + max(costs)
    assert sharding.balanced_partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        sharding.balanced_partition([1.0], 0)
    assert sharding.weak_shard(512, 3) == (1536, 512)
