"""The primitive-screening bound of the class kernels, restated in numpy and
checked against the oracle: for primitive pairs of every l <= 3 combination,
Q bounds sqrt|(ab|ab)| of every element (Cartesian and spherical), so a
primitive quartet never exceeds Q_ab Q_cd (Cauchy-Schwarz)."""
from math import comb, sqrt

import numpy as np
import pytest

from intception_b200 import basis
from oracle import loader

# sqrt of the Coulomb self-energy of r^n exp(-r^2), n = 0..6 (the values the
# device code uses); n = 0 is sqrt(sqrt(2) pi^(5/2))
RN_NORM = [4.9738746919472297, 5.1652368552576019, 6.4612527577002005, 9.2648431767816622,
           14.794795287711256, 25.818805439099522, 48.591021989124202]
SPH_COLSUM = [1.0, 1.0, 2.0, 4.0]


def pair_bound(l0, l1, x0, c0, x1, c1, r, sph):
    z = x0 + x1
    K = abs(c0 * c1) * np.exp(-x0 * x1 / z * r * r)
    pa, pb = x1 / z * r, x0 / z * r
    s = 1.0 / sqrt(z)
    poly = sum(comb(l0, i) * comb(l1, j) * RN_NORM[i + j] * pa ** (l0 - i) * pb ** (l1 - j) * s ** (i + j)
               for i in range(l0 + 1) for j in range(l1 + 1))
    f = SPH_COLSUM[l0] * SPH_COLSUM[l1] if sph else 1.0
    return f * K * s * s * sqrt(s) * poly


def test_rn_norm_zero_is_closed_form():
    assert abs(RN_NORM[0] ** 2 - sqrt(2.0) * np.pi ** 2.5) < 1e-13


def test_sph_colsum_matches_library_matrices():
    for l in range(4):
        assert abs(np.abs(np.asarray(basis.sph_matrix(l))).sum(axis=0).max() - SPH_COLSUM[l]) < 1e-12


@pytest.mark.parametrize('sph', [False, True])
def test_pair_bound_covers_diagonal_integrals(sph):
    rng = np.random.default_rng(11 + sph)
    worst = 0.0
    for l0 in range(4):
        for l1 in range(4):
            for _ in range(12):
                x0, x1 = np.exp(rng.uniform(np.log(0.05), np.log(200.0), 2))
                c0, c1 = rng.uniform(-2.0, 2.0, 2)
                r = rng.choice([0.0, rng.uniform(0.1, 1.0), rng.uniform(1.0, 6.0)])
                A = np.zeros(3)
                u = rng.normal(size=3)
                B = r * u / np.linalg.norm(u)
                ls = np.array([l0, l1, l0, l1], np.int32)
                q = np.array([[0, 1, 2, 3]], np.int32)
                off, tot = basis.packed_offsets(ls, q, sph)
                b = basis.ShellBatch(ls, np.ones(4, np.int32), np.arange(4, dtype=np.int32),
                                     np.array([A, B, A, B]), np.array([x0, x1, x0, x1]),
                                     np.array([c0, c1, c0, c1]), q, off, sph, tot)
                v = loader.oracle_batch(b, basis.sph_matrices(6))
                n0 = 2 * l0 + 1 if sph else (l0 + 1) * (l0 + 2) // 2
                n1 = 2 * l1 + 1 if sph else (l1 + 1) * (l1 + 2) // 2
                blk = v.reshape(n1, n0, n1, n0)  # [d][c][b][a]
                diag = np.array([blk[j, i, j, i] for i in range(n0) for j in range(n1)])
                assert (diag >= -1e-14 * np.abs(diag).max()).all()  # (ab|ab) >= 0
                qb = pair_bound(l0, l1, x0, c0, x1, c1, r, sph)
                lhs = np.sqrt(np.abs(v).max())  # every element of (ab|ab), off-diagonal ones included
                assert lhs <= qb * (1 + 1e-12), (l0, l1, x0, x1, r, lhs, qb)
                if qb > 0.0:
                    worst = max(worst, lhs / qb)
    assert worst > 1e-3  # the bound is not vacuous


def _device_constants(name):
    """The literals of a constexpr chain `n == k ? v : ...` in the device header."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(__file__), '..', 'intception_b200', 'csrc', 'ib_eri_device.cuh')).read()
    body = src[src.index(name):]
    body = body[:body.index(';')]
    return [float(x) for x in re.findall(r'[0-9]+\.[0-9]+(?:e[-+]?[0-9]+)?', body)]


def test_device_norms_match_quadrature():
    """The device's N_n (sqrt of the Coulomb self-energy of r^n exp(-r^2)) for
    n = 0..12, against a direct quadrature of the spherical self-energy
    4 pi int g(r) V(r) r^2 dr, V(r) = 4 pi (int_0^r g s^2 ds / r + int_r^inf g s ds)."""
    from scipy import integrate
    vals = _device_constants('ib_rn_norm(int n)')
    assert len(vals) == 13
    assert np.allclose(vals[:7], RN_NORM, rtol=1e-15)
    for n in (0, 1, 3, 6, 9, 12):
        g = lambda r, n=n: r ** n * np.exp(-r * r)  # noqa: E731
        inner = lambda r: integrate.quad(lambda t: g(t) * t * t, 0, r, epsabs=0, epsrel=1e-13)[0]  # noqa: E731
        outer = lambda r: integrate.quad(lambda t: g(t) * t, r, np.inf, epsabs=0, epsrel=1e-13)[0]  # noqa: E731
        V = lambda r: 4 * np.pi * ((inner(r) / r if r > 0 else 0.0) + outer(r))  # noqa: E731
        u = integrate.quad(lambda r: g(r) * V(r) * 4 * np.pi * r * r, 0, 12, epsabs=0, epsrel=1e-11, limit=200)[0]
        assert abs(np.sqrt(u) - vals[n]) <= 1e-9 * vals[n], n


def test_device_sph_colsums_cover_library_matrices():
    vals = _device_constants('ib_sph_colsum(int l)')
    # the chain lists l <= 1, 2, 3, 4, 5 and the l = 6 fallback
    want = [float(np.abs(np.asarray(basis.sph_matrix(l))).sum(axis=0).max()) for l in range(1, 7)]
    assert len(vals) == 6
    for v, w in zip(vals, want):
        assert v >= w and v <= w * (1 + 1e-12)


@pytest.mark.parametrize('name', ['mixed_l2_sph_c2', 'mixed_l2_sph_compact', 'mixed_l2_cart_compact', 'l4_cart',
                                  'l4_sph', 'l6_cart', 'l6_sph', 'edge_cart', 'edge_sph'])
def test_oracle_quartet_bound_covers_reference_blocks(name):
    """The analytic screening bound (oracle/pair_bound.h, the restatement of
    intception_b200_quartet_bounds) is at least max |element| of every block
    the reference's emitted C99 wrote for the golden fixtures."""
    from conftest import load_batch
    b, T, ref = load_batch(name)
    bd = loader.quartet_bounds(b)
    sizes = basis.block_sizes(b.shell_l, b.quartets, b.spherical)
    for q in range(b.nq):
        m = float(np.abs(ref[b.out_off[q]:b.out_off[q] + sizes[q]]).max())
        assert m <= bd[q], (q, m, bd[q])


def test_oracle_quartet_bound_matches_numpy_restatement():
    """pair_bound.h against the numpy pair_bound above summed over primitives."""
    b = basis.config_mixed_l2(nq=200, seed=5, spherical=True)
    bd = loader.quartet_bounds(b)
    for q in range(b.nq):
        qs = []
        for side in range(2):
            s0, s1 = b.quartets[q, 2 * side], b.quartets[q, 2 * side + 1]
            r = float(np.linalg.norm(b.shell_xyz[s0] - b.shell_xyz[s1]))
            tot = 0.0
            for i in range(b.shell_k[s0]):
                for j in range(b.shell_k[s1]):
                    p0, p1 = b.shell_ptr[s0] + i, b.shell_ptr[s1] + j
                    tot += pair_bound(int(b.shell_l[s0]), int(b.shell_l[s1]), b.prim_exp[p0], b.prim_coef[p0],
                                      b.prim_exp[p1], b.prim_coef[p1], r, True)
            qs.append(tot)
        want = qs[0] * qs[1] * 1.000001 ** 5  # each stage widened by 1 + 1e-6, as on the device
        assert abs(bd[q] - want) <= 1e-12 * abs(bd[q]) + 1e-300
