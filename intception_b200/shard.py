"""Multi-GPU sharding of a quartet list (one process per GPU, no collective).

Every shell quartet is independent, so a batch is split into contiguous,
cost-balanced shards of the class-sorted quartet list; each rank evaluates its
shard with its own engine and writes its own output blocks.  The cost of a
quartet is the algorithmic FP64 work of its class times its primitive count
(the same per-class counts the roofline uses).
"""
import json
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))


def canonical_class(ls):
    """Canonical class id per quartet row of l values (la,lb,lc,ld)."""
    ls = np.asarray(ls, dtype=np.int64)
    la, lb, lc, ld = (ls[:, k].copy() for k in range(4))
    sw = la < lb
    la[sw], lb[sw] = lb[sw], la[sw].copy()
    sw = lc < ld
    lc[sw], ld[sw] = ld[sw], lc[sw].copy()
    pb = la * (la + 1) // 2 + lb
    pk = lc * (lc + 1) // 2 + ld
    hi, lo = np.maximum(pb, pk), np.minimum(pb, pk)
    return hi * (hi + 1) // 2 + lo


def quartet_cost(batch, stats=None):
    """Relative cost per quartet; classes without per-class counts (some l > 2)
    are costed by (L+1)^4 times the primitive count."""
    if stats is None:
        path = os.path.join(PKG, 'class_stats.json')
        stats = {}
        if os.path.exists(path):
            with open(path) as fh:
                stats = {s['cid']: s for s in json.load(fh)}
    ls = batch.shell_l[batch.quartets]
    kp = batch.shell_k[batch.quartets].astype(np.float64).prod(axis=1)
    cid = canonical_class(ls)
    L = ls.sum(axis=1)
    per = np.array([stats[c]['vrr_flops'] + 74 + 2 * stats[c]['L'] if c in stats else float((l + 1) ** 4)
                    for c, l in zip(cid, L)]) if len(cid) else np.zeros(0)
    return kp * per


def partition(batch, nranks, cost=None):
    """List of nranks index arrays (into batch.quartets): class-sorted,
    contiguous, balanced by cumulative cost.  Disjoint; their union is every
    quartet."""
    if cost is None:
        cost = quartet_cost(batch)
    order = np.lexsort((cost, canonical_class(batch.shell_l[batch.quartets])))
    c = np.cumsum(cost[order])
    total = c[-1] if len(c) else 0.0
    cuts = [0] + [int(np.searchsorted(c, total * r / nranks, side='left')) for r in range(1, nranks)] + [len(order)]
    return [np.sort(order[cuts[r]:cuts[r + 1]]) for r in range(nranks)]


def shard_for_rank(batch, rank, nranks):
    """The sub-batch of this rank (outputs repacked) and its indices."""
    idx = partition(batch, nranks)[rank]
    return batch.subset(idx), idx
