"""The CPU oracle (C restatement of the reference's ERI path) against the
reference's own emitted C99: golden fixtures, live comparison when oracle/_ref
is built, and an independent McMurchie-Davidson cross-check."""
import numpy as np
import pytest

from conftest import BATCH_FIXTURES, load_batch, load_dropin_cases, tolerance, GOLDEN
from intception_b200 import basis
from oracle import loader, md_eri


@pytest.mark.parametrize('name', BATCH_FIXTURES)
def test_oracle_matches_golden(name):
    b, T, ref = load_batch(name)
    out = loader.oracle_batch(b, T)
    assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('k', range(12))
def test_oracle_dropin_cases(k):
    shells, ref, sph = load_dropin_cases()[k]
    out = np.full(ref.shape, -7.0)
    lib = loader.load_oracle()
    loader.call_main(lib, 'sph' if sph else 'cart', shells, np.zeros(1), out,
                     prefix='oracle_eri_cont_%s_main' % ('sph' if sph else 'cart'))
    assert np.array_equal(out == -7.0, ref == -7.0)  # same untouched elements
    assert np.abs(out - ref).max() <= tolerance(ref)


def test_oracle_boys_golden():
    """Same scheme as the reference; the tables are recomputed with mpmath, so
    only their last-digit rounding may differ."""
    z = np.load(GOLDEN + '/boys.npz')
    for x, F in zip(z['x'], z['F']):
        assert np.abs(loader.boys(int(z['nmax']), x) - F).max() <= 1e-15


def test_oracle_work_array_size_golden():
    t = np.load(GOLDEN + '/work_array_size.npz')['table']
    lib = loader.load_oracle()
    got = np.array([lib.oracle_eri_work_array_size(*map(int, r[:12])) for r in t])
    assert np.array_equal(got, t[:, 12])


def test_oracle_boys_accuracy():
    """The reference's Boys scheme against scipy's incomplete gamma."""
    for x in (0.0, 0.3, 3.7, 12.2, 15.05, 29.3, 40.0, 300.0):
        f = loader.boys(12, x)
        ex = np.array([md_eri.boys(m, x) for m in range(13)])
        assert np.abs(f - ex).max() < 2e-14


def test_oracle_accurate_boys_mode():
    """The oracle's accurate Boys mode (series + downward recursion below 50,
    exact upward recursion above) agrees with scipy to a few ulps in relative
    terms up to m = 24, where the reference's scheme loses digits (Taylor
    truncation on the 0.1 grid; exp(-x) dropped from x = 35); the default mode
    stays the reference's."""
    worst_acc = worst_ref = 0.0
    for x in np.concatenate([np.linspace(0.0, 70.0, 141), [1e-9, 1e-4, 34.99, 35.0, 35.5, 49.99, 50.0]]):
        ex = np.array([md_eri.boys(m, x) for m in range(25)])
        acc = loader.boys(24, x, exact=True)
        ref = loader.boys(24, x)
        worst_acc = max(worst_acc, float((np.abs(acc - ex) / ex).max()))
        worst_ref = max(worst_ref, float((np.abs(ref - ex) / ex).max()))
    assert worst_acc < 1e-13
    assert worst_ref > 1e-6  # the reference's own error at high m: the mode is a real switch
    z = np.load(GOLDEN + '/boys.npz')
    assert np.abs(loader.boys(int(z['nmax']), float(z['x'][0])) - z['F'][0]).max() <= 1e-15


@pytest.mark.parametrize('ls', [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 1, 1), (2, 1, 0, 1), (0, 2, 2, 1), (2, 2, 1, 1),
                                (3, 0, 1, 0), (0, 3, 0, 1), (3, 1, 1, 0), (1, 0, 3, 2)])
def test_oracle_vs_mcmurchie_davidson(ls):
    rng = np.random.default_rng(sum(ls) * 7 + 3)
    shells = []
    for l in ls:
        k = 2
        x = np.exp(rng.uniform(np.log(0.2), np.log(8.0), k))
        c = basis.normalize_shell(l, x, rng.uniform(0.2, 1.0, k))
        shells.append((l, x, c, rng.uniform(0.0, 2.5, 3)))
    ref = md_eri.contracted_eri(shells)
    ls_ = np.array(ls, np.int32)
    ks = np.full(4, 2, np.int32)
    ptr = np.arange(4, dtype=np.int32) * 2
    xyz = np.array([s[3] for s in shells])
    e = np.concatenate([s[1] for s in shells])
    c = np.concatenate([s[2] for s in shells])
    q = np.array([[0, 1, 2, 3]], np.int32)
    off, total = basis.packed_offsets(ls_, q, False)
    b = basis.ShellBatch(ls_, ks, ptr, xyz, e, c, q, off, False, total)
    out = loader.oracle_batch(b)
    assert np.abs(out - ref).max() < 1e-13 * max(1.0, np.abs(ref).max())


def test_oracle_vs_reference_live():
    """Fresh seeded inputs through both the restatement and the emitted C99."""
    if loader.load_ref('cart') is None:
        pytest.skip('oracle/_ref not built here')
    T = basis.sph_matrices(6)
    for sph in (False, True):
        b = basis.independent_quartet_batch(123, 50, [0, 1, 2, 3], [1, 2, 3], 0.1, 60.0, 5.0, sph)
        ref = loader.ref_batch(b, T)
        assert np.abs(loader.oracle_batch(b, T) - ref).max() <= tolerance(ref)


def test_quad_oracle_matches_golden_where_double_is_exact():
    """The binary128 build of the restatement (oracle_batch_quad) against the
    reference's golden values on well-conditioned (pp|pp) quartets, where
    double recurrences keep every digit: the two builds compute the same
    integrals."""
    b, T, ref = load_batch('pppp_k3_cart')
    sub = b.subset(np.arange(12))
    sizes = basis.block_sizes(b.shell_l, sub.quartets, False)
    gather = np.concatenate([np.arange(o, o + n) for o, n in zip(b.out_off[:12], sizes)])
    out = loader.oracle_batch_quad(sub, T)
    assert np.abs(out - ref[gather]).max() <= 1e-14 * max(1.0, float(np.abs(ref).max()))


def test_mixed_contraction_fixture_exact_values():
    """The fixture's exact values re-evaluated (its smallest quartets), and
    the reference's own error on its quartets, which the fixture records."""
    b, T, exact = load_batch('mixed_contraction_sph')
    sizes = basis.block_sizes(b.shell_l, b.quartets, True)
    cost = [int(np.prod(b.shell_k[s])) for s in b.quartets]
    for q in np.argsort(cost)[:3]:
        out = loader.oracle_batch_quad(b.subset(np.array([q])), T)
        assert np.array_equal(out, exact[b.out_off[q]:b.out_off[q] + sizes[q]])
    ref = np.load(GOLDEN + '/mixed_contraction_sph.npz')['ref_out']
    # the reference's double recurrences (bra HRR in the caller's shell order)
    # miss the exact values by more than the parity bar on some of these quartets
    assert np.abs(ref - exact).max() > tolerance(exact)


def test_generic_split_fixture_exact_values():
    """The generic-split fixture's exact values re-evaluated (its two cheapest
    quartets), and the double restatement against them: close, but off by
    more than the parity bar on its heavy quartets (3.1e-10)."""
    b, T, exact = load_batch('generic_split_sph')
    sizes = basis.block_sizes(b.shell_l, b.quartets, True)
    cost = [int(np.prod(b.shell_k[s])) for s in b.quartets]
    for q in np.argsort(cost, kind='stable')[:2]:
        out = loader.oracle_batch_quad(b.subset(np.array([q])), T)
        assert np.array_equal(out, exact[b.out_off[q]:b.out_off[q] + sizes[q]])
    err = np.abs(loader.oracle_batch(b, T) - exact).max()
    assert tolerance(exact) < err < 1e-9
