"""Primitive screening in the batch path (eri.set_prim_tol), on a B200: every
element stays within Ka Kb Kc Kd x tol of the unscreened result (plus the
rounding of the shortened sums), the parity tests still hold at the bench
tolerance, and 0 restores the exact path bit for bit."""
import numpy as np
import pytest

from conftest import tolerance
from intception_b200 import basis, eri
from oracle import loader

pytestmark = pytest.mark.gpu


def _run(b, tol):
    import torch
    eri.set_prim_tol(tol)
    try:
        eng = eri.EriEngine(b)
        out = eng.compute()
        torch.cuda.synchronize()
        assert eng.device_status() == 0
        return out.cpu().numpy()
    finally:
        eri.set_prim_tol(0.0)


def _allowed(b, exact, tol):
    """Per element: Ka Kb Kc Kd tol (the skipped primitive quartets) plus
    1e-12 of the block's largest element (the shortened sums round
    differently, and the HRRs carry that rounding as they carry the FP64
    path's own)."""
    sizes = basis.block_sizes(b.shell_l, b.quartets, b.spherical)
    kp = b.shell_k[b.quartets].prod(axis=1).astype(np.float64)
    seg = np.repeat(np.arange(b.nq), sizes)
    bmax = np.zeros(b.nq)
    np.maximum.at(bmax, seg, np.abs(exact))
    return np.repeat(kp * tol + 1e-12 * bmax, sizes)


@pytest.mark.parametrize('sph', [False, True])
@pytest.mark.parametrize('tol', [1e-18, 1e-13, 1e-10])
def test_screened_within_bound(sph, tol):
    """The bench's l <= 2 distribution (30-bohr cube, K 1..6): per element
    |screened - exact| <= Ka Kb Kc Kd tol; large tolerances actually move
    results (the screening runs) and stay inside the bound."""
    b = basis.config_mixed_l2(nq=30000, seed=5, spherical=sph)
    exact = _run(b, 0.0)
    scr = _run(b, tol)
    assert (np.abs(scr - exact) <= _allowed(b, exact, tol)).all()
    if tol >= 1e-13:
        assert (scr != exact).any()


def test_zero_tolerance_is_exact_path():
    b = basis.config_mixed_l2(nq=5000, seed=6, spherical=True)
    a1 = _run(b, 0.0)
    _run(b, 1e-10)
    a2 = _run(b, 0.0)
    assert np.array_equal(a1, a2)


def _orderings(seed, lmax, sph, lo, hi, box, kmax):
    rng = np.random.default_rng(seed)
    quartets, ls = [], []
    for la in range(lmax + 1):
        for lb in range(lmax + 1):
            for lc in range(lmax + 1):
                for ld in range(lmax + 1):
                    base = len(ls)
                    ls += [la, lb, lc, ld]
                    quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.integers(1, kmax + 1, len(ls)).astype(np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, lo, hi, box)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    return basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)


@pytest.mark.parametrize('sph', [False, True])
def test_screened_l2_classes_vs_oracle(sph):
    """Every (la,lb,lc,ld) ordering with l <= 2, three copies (exponents
    0.05..1e4 in a 6-bohr box, K 1..6), screened at the bench tolerance,
    against the oracle at the parity bar."""
    b = _orderings(131 + sph, 2, sph, 0.05, 1e4, 6.0, 6)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    out = _run(b, 1e-18)
    assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('sph', [False, True])
def test_screened_f_classes(sph):
    """Every ordering with l <= 3 (the 128-lane (ff|ff) groups and the 64-lane
    f groups build their lists the same way): at the bench tolerance the
    screened blocks meet the parity bar against the oracle; at 1e-12, which
    drops many more primitive quartets, they stay within Ka Kb Kc Kd tol of
    the unscreened ones (plus 1e-13 of rounding)."""
    b = _orderings(141 + sph, 3, sph, 0.3, 40.0, 5.0, 5)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    assert np.abs(_run(b, 1e-18) - ref).max() <= tolerance(ref)
    exact = _run(b, 0.0)
    scr = _run(b, 1e-12)
    kp = np.repeat(b.shell_k[b.quartets].prod(axis=1).astype(np.float64),
                   basis.block_sizes(b.shell_l, b.quartets, b.spherical))
    assert (np.abs(scr - exact) <= kp * 1e-12 + 1e-13).all()
    assert (scr != exact).any()


def test_prim_tol_rejects_out_of_range():
    for bad in (-1e-20, 1e-5, float('nan')):
        with pytest.raises(Exception):
            eri.set_prim_tol(bad)
    eri.set_prim_tol(0.0)


def test_schwarz_factors_ignore_prim_tol():
    """The Schwarz factors bound the quartets that screening zeroes, so they
    are computed without primitive screening whatever the setting."""
    import torch
    b = basis.config_mixed_l2(nq=4000, seed=8, spherical=True)
    eng = eri.EriEngine(b)
    q0 = eng.quartet_bounds()
    eri.set_prim_tol(1e-6)
    try:
        q1 = eng.quartet_bounds()
        torch.cuda.synchronize()
    finally:
        eri.set_prim_tol(0.0)
    assert torch.equal(q0, q1)


def test_screened_with_fp32_tier_meets_error_bar():
    """Primitive screening together with the FP32 tier (every class's FP32
    kernel on, all quartets in the tier): within 1e-10 of the oracle."""
    import torch
    b = _orderings(151, 2, True, 0.05, 1e4, 6.0, 6)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    eri.set_prim_tol(1e-18)
    eri.set_class_fp32(True)
    try:
        eng = eri.EriEngine(b)
        bounds = torch.ones(b.nq, dtype=torch.float64, device='cuda')
        out = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, fp32_below=2.0, mixed_tol=5e-11)
        torch.cuda.synchronize()
        assert eng.device_status() == 0
    finally:
        eri.set_prim_tol(0.0)
        eri.set_class_fp32(None)
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-10
