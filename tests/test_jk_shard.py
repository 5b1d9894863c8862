"""Multi-GPU J/K digestion, host logic (one process per rank, gloo on CPU):
each rank digests its share of every screened quartet chunk and one
all_reduce (sum) of the partial energies and forces follows.  The per-quartet
digestion is replaced by a CPU stand-in built on the oracle's ERI blocks (the
CUDA digestion has its own GPU tests); the sharded totals must equal the
single-rank totals to 1e-12."""
import os

import numpy as np
import torch
import torch.multiprocessing as mp

from intception_b200 import basis as B
from intception_b200 import jk


class OracleJK(jk.JKSystem):
    """JKSystem on the CPU: Schwarz factors and blocks from the oracle."""

    def _blocks(self, qt):
        from oracle import loader
        ns = self.ns
        l = self.shell_l[:ns].numpy()
        k = self.shell_k[:ns].numpy()
        ptr = self.shell_ptr[:ns].numpy()
        npr = int(k.sum())
        q = np.ascontiguousarray(qt.numpy().astype(np.int32))
        off, total = B.packed_offsets(l, q, False)
        sb = B.ShellBatch(l, k, ptr, self.shell_xyz[:ns].numpy(), self.prim_exp[:npr].numpy(),
                          self.prim_coef[:npr].numpy(), q, off, False, total)
        return loader.oracle_batch(sb), off, B.block_sizes(l, q, False)

    def schwarz(self):
        pr = self.pairs.numpy()
        qt = torch.from_numpy(np.stack([pr[:, 0], pr[:, 1], pr[:, 0], pr[:, 1]], axis=1).astype(np.int32))
        out, off, n = self._blocks(qt)
        return torch.tensor([np.sqrt(np.abs(out[o:o + m]).max()) for o, m in zip(off, n)], dtype=torch.float64)

    def _energy_chunk(self, qt, e):
        out, off, n = self._blocks(qt)
        q = qt.numpy()
        deg = (1.0 + (q[:, 0] != q[:, 1])) * (1.0 + (q[:, 2] != q[:, 3])) * \
            (1.0 + ((q[:, 0] != q[:, 2]) | (q[:, 1] != q[:, 3])))
        e[0] += float(sum(d * out[o:o + m].sum() for d, o, m in zip(deg, off, n)))
        e[1] -= float(sum(d * (out[o:o + m] ** 2).sum() for d, o, m in zip(deg, off, n)))

    def _force_chunk(self, qt, force):
        out, off, n = self._blocks(qt)
        atom = self.shell_atom_np[qt.numpy()[:, 0]]
        for a, o, m in zip(atom, off, n):
            force[3 * a:3 * a + 3] += torch.tensor([out[o:o + m].sum(), out[o:o + m].max(), -out[o:o + m].min()],
                                                   dtype=torch.float64)


def _system(**kw):
    xyz = np.array([[0.0, 0.0, 0.0], [1.4, 0.2, -0.3], [0.1, 2.1, 0.9]])
    ls = np.array([0, 1, 2] * 3, np.int32)
    ks = np.array([3, 2, 1] * 3, np.int32)
    atom = np.repeat(np.arange(3), 3).astype(np.int32)
    rng = np.random.default_rng(17)
    _, _, _, _, e, c = B.make_shells(rng, ls, ks, 0.2, 30.0, 1.0, centres=np.zeros((9, 3)))
    nbf = int((2 * ls + 1).sum())
    Cm = rng.normal(0.0, 0.1, (nbf, 3))
    return OracleJK(xyz, atom, ls, ks, e, c, Cm @ Cm.T, device='cpu', screen=1e-12, chunk=50, **kw), xyz


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    sys_, xyz = _system()
    assert sys_.rank == rank and sys_.world == world
    e = sys_.energy(xyz)
    g = sys_.gradient(xyz).numpy()
    nq = sum(int(sys_.shard(c).shape[0]) for c in sys_.quartet_chunks())
    dist.destroy_process_group()
    q.put((rank, e, g, nq))


def test_two_rank_jk_sums_equal_single_rank():
    one, xyz = _system(rank=0, world=1)
    e1 = one.energy(xyz)
    g1 = one.gradient(xyz).numpy()
    total = sum(int(c.shape[0]) for c in one.quartet_chunks())
    assert total > 100 and len(list(one.quartet_chunks())) > 2  # several chunks, each split
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][3] + res[1][3] == total and abs(res[0][3] - res[1][3]) <= len(list(one.quartet_chunks()))
    for _, e, g, _ in res:
        assert abs(e[0] - e1[0]) <= 1e-12 * max(1.0, abs(e1[0]))
        assert abs(e[1] - e1[1]) <= 1e-12 * max(1.0, abs(e1[1]))
        assert np.abs(g - g1).max() <= 1e-12 * max(1.0, np.abs(g1).max())


def test_partial_sums_without_reduce_add_up():
    """reduce=False returns each rank's partial sums; their sum is the total."""
    one, xyz = _system(rank=0, world=1)
    e1 = one.energy(xyz)
    parts = [_system(rank=r, world=3, reduce=False)[0] for r in range(3)]
    es = [p.energy(xyz) for p in parts]
    assert abs(sum(e[0] for e in es) - e1[0]) <= 1e-12 * max(1.0, abs(e1[0]))
    assert abs(sum(e[1] for e in es) - e1[1]) <= 1e-12 * max(1.0, abs(e1[1]))
