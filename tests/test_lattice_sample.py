"""Host logic of the lattice workload: the shells and the uniform sample of
screened unique quartets (checked against brute-force enumeration)."""
import numpy as np

from intception_b200 import basis


def test_lattice_shells_layout():
    rng, l_, k_, p_, xyz, e, c = basis.lattice_shells(natom=27, seed=5)
    assert len(l_) == 27 * 5
    assert list(l_[:5]) == [0, 0, 1, 2, 3] and list(k_[:5]) == [6, 3, 3, 1, 1]
    assert (np.diff(p_) == k_[:-1]).all() and len(e) == int(k_.sum())
    assert np.allclose(xyz[0], xyz[4])  # shells of one atom share its centre
    assert (e >= 0.1).all() and (e <= 1e3).all()


def test_sample_matches_enumeration():
    rng = np.random.default_rng(3)
    npair = 300
    q = np.exp(rng.uniform(np.log(1e-9), 0.0, npair))
    pairs = np.stack([np.arange(npair), np.arange(npair)], axis=1).astype(np.int32)
    order = np.argsort(-q, kind='stable')
    rank = np.empty(npair, np.int64)
    rank[order] = np.arange(npair)
    full = {(i, j) for i in range(npair) for j in range(npair)
            if rank[j] <= rank[i] and q[i] * q[j] >= 1e-12}
    qu, total = basis.sample_screened_quartets(q, pairs, 10 ** 9, np.random.default_rng(1), 1e-12)
    assert total == len(full)
    got = {(int(a), int(b)) for a, _, b, _ in qu}
    assert got == full  # asked for more than exist: every quartet once
    qu2, _ = basis.sample_screened_quartets(q, pairs, 500, np.random.default_rng(2), 1e-12)
    s2 = {(int(a), int(b)) for a, _, b, _ in qu2}
    assert len(s2) == 500 and s2 <= full
