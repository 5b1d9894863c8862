"""Sharding of a quartet list over ranks (host logic), exercised with two
gloo ranks on CPU: shards are disjoint, cover every quartet, and carry
balanced cost; an all_gather of the per-rank costs agrees on every rank."""
import os

import numpy as np
import torch.multiprocessing as mp

from intception_b200 import basis, shard


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    b = basis.config_mixed_l2(nq=5000, seed=3, spherical=True)
    sub, idx = shard.shard_for_rank(b, rank, world)
    cost = float(shard.quartet_cost(b)[idx].sum())
    t = torch.tensor([len(idx), cost], dtype=torch.float64)
    out = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(out, t)
    ids = [torch.zeros(len(b.quartets), dtype=torch.int64) for _ in range(world)]
    mine = torch.zeros(len(b.quartets), dtype=torch.int64)
    mine[torch.as_tensor(idx)] = 1
    dist.all_gather(ids, mine)
    dist.destroy_process_group()
    cover = sum(x for x in ids)
    q.put((rank, [o.tolist() for o in out], int(cover.min()), int(cover.max()), sub.nq, sub.out_size))


def test_two_rank_partition_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, cmin, cmax, nq, size in res:
        assert cmin == 1 and cmax == 1          # every quartet on exactly one rank
        (n0, c0), (n1, c1) = gathered
        assert n0 + n1 == 5000
        assert abs(c0 - c1) / (c0 + c1) < 0.02  # cost-balanced
        assert nq == int(gathered[rank][0]) and size > 0


def test_partition_single_process_properties():
    b = basis.config_mixed_l2(nq=3000, seed=4, spherical=False)
    parts = shard.partition(b, 4)
    allidx = np.concatenate(parts)
    assert np.array_equal(np.sort(allidx), np.arange(b.nq))
    cost = shard.quartet_cost(b)
    loads = [cost[p].sum() for p in parts]
    assert max(loads) / min(loads) < 1.1
