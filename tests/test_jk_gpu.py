"""J/K energies and their nuclear gradient: energies against a dense
contraction of every ordered quartet evaluated by the CPU oracle, the adjoint
gradient against central finite differences of the GPU energy (h = 1e-4 bohr,
tolerance 1e-7), and the torch.autograd wiring."""
import numpy as np
import pytest

from intception_b200 import basis as B
from intception_b200 import jk
from oracle import loader

pytestmark = pytest.mark.gpu


def reference_energy(system, xyz):
    """(E_J, E_K) from all ordered shell quartets by the oracle, dense einsum."""
    ns = system.ns
    l = system.shell_l[:ns].cpu().numpy()
    k = system.shell_k[:ns].cpu().numpy()
    ptr = system.shell_ptr[:ns].cpu().numpy()
    npr = int(k.sum())
    e = system.prim_exp[:npr].cpu().numpy()
    c = system.prim_coef[:npr].cpu().numpy()
    shell_xyz = np.asarray(xyz, np.float64)[system.shell_atom_np]
    q = np.array([(a, b, cc, d) for a in range(ns) for b in range(ns) for cc in range(ns) for d in range(ns)],
                 np.int32)
    off, total = B.packed_offsets(l, q, False)
    sb = B.ShellBatch(l, k, ptr, shell_xyz, e, c, q, off, False, total)
    out = loader.oracle_batch(sb)
    nbf = system.nbf_cart
    fofs = system.fofs_np
    nc = (l + 1) * (l + 2) // 2
    I = np.zeros((nbf, nbf, nbf, nbf))
    for r, (a, b, cc, d) in enumerate(q):
        blk = out[off[r]:off[r] + nc[a] * nc[b] * nc[cc] * nc[d]].reshape(nc[d], nc[cc], nc[b], nc[a])
        I[fofs[a]:fofs[a] + nc[a], fofs[b]:fofs[b] + nc[b], fofs[cc]:fofs[cc] + nc[cc],
          fofs[d]:fofs[d] + nc[d]] = blk.transpose(3, 2, 1, 0)
    P = system.P.cpu().numpy()
    return 0.5 * np.einsum('ij,kl,ijkl->', P, P, I), -0.25 * np.einsum('ik,jl,ijkl->', P, P, I)


def small_system(natom=3, seed=7):
    return jk.lattice_system(natom=natom, seed=seed, shells=((0, 3), (1, 2), (2, 1)), alpha=(0.2, 30.0), nocc=4,
                             screen=1e-16)


def test_jk_energy_matches_dense_oracle_contraction():
    sys_, xyz = small_system()
    ej, ek = sys_.energy(xyz)
    rj, rk = reference_energy(sys_, xyz)
    assert abs(ej - rj) <= 1e-11 * max(1.0, abs(rj))
    assert abs(ek - rk) <= 1e-11 * max(1.0, abs(rk))
    assert abs(ej) > 1e-3 and abs(ek) > 1e-4


def test_jk_gradient_matches_central_differences():
    sys_, xyz = small_system()
    g = sys_.gradient(xyz).cpu().numpy()
    h = 1e-4
    fd = np.zeros_like(g)
    for a in range(xyz.shape[0]):
        for d in range(3):
            xp = xyz.copy()
            xm = xyz.copy()
            xp[a, d] += h
            xm[a, d] -= h
            fd[a, d] = (sum(sys_.energy(xp)) - sum(sys_.energy(xm))) / (2 * h)
    assert np.abs(g - fd).max() <= 1e-7
    assert np.abs(g.sum(axis=0)).max() <= 1e-9  # translational invariance
    assert np.abs(g).max() > 1e-4


def test_jk_autograd_function():
    import torch
    sys_, xyz = small_system()
    x = torch.tensor(xyz, dtype=torch.float64, requires_grad=True)
    e = jk.jk_energy(x, sys_)
    e.backward()
    g = sys_.gradient(xyz).cpu().numpy()
    assert np.allclose(x.grad.numpy(), g, atol=1e-13, rtol=0)
    assert abs(float(e) - sum(sys_.energy(xyz))) <= 1e-12


def test_jk_shards_add_up_on_one_gpu():
    """The two shards of a world-2 run, evaluated one after the other on this
    GPU with the all_reduce left out (reduce=False), add up to the one-rank
    energies and gradient to 1e-12."""
    one, xyz = small_system()
    e1 = one.energy(xyz)
    g1 = one.gradient(xyz).cpu().numpy()
    parts = [jk.lattice_system(natom=3, seed=7, shells=((0, 3), (1, 2), (2, 1)), alpha=(0.2, 30.0), nocc=4,
                               screen=1e-16, rank=r, world=2, reduce=False)[0] for r in range(2)]
    es = [p.energy(xyz) for p in parts]
    gs = [p.gradient(xyz).cpu().numpy() for p in parts]
    for k in range(2):
        assert abs(es[0][k] + es[1][k] - e1[k]) <= 1e-12 * max(1.0, abs(e1[k]))
    assert np.abs(gs[0] + gs[1] - g1).max() <= 1e-12 * max(1.0, np.abs(g1).max())


def test_jk_one_pass_digestion_equals_per_batch_launches():
    """The one-pass gradient digestion over the six auxiliary batches
    (intception_b200_jk_force_all, the default) against one launch per batch
    (intception_b200_jk_force), on a system with f shells so that the
    staged-density path and the gathering path both run."""
    sys_, xyz = jk.lattice_system(natom=4, seed=11, shells=((0, 3), (1, 2), (2, 2), (3, 1)), alpha=(0.2, 30.0),
                                  nocc=6, screen=1e-16)
    g_all = sys_.gradient(xyz).cpu().numpy()
    sys_.per_batch_digestion = True
    g_per = sys_.gradient(xyz).cpu().numpy()
    assert np.abs(g_all - g_per).max() <= 1e-12 * max(1.0, np.abs(g_per).max())
    assert np.abs(g_per).max() > 1e-4


def test_jk_energy_independent_of_chunking():
    """The energy sums are compensated and fixed-order: chunks of 97 quartets
    and one chunk give the same energies to 1e-15 relative (plain sums in a
    changing order move them by ~1e-13, which a central difference with
    h = 1e-4 would turn into a 1e-7 gradient error)."""
    sys_, xyz = small_system()
    e1 = sys_.energy(xyz)
    sys_.chunk = 97
    e2 = sys_.energy(xyz)
    for a, b in zip(e1, e2):
        assert abs(a - b) <= 1e-15 * abs(a)
