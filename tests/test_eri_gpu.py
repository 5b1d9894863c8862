"""CUDA path parity: the drop-ins and the batch API against the reference's
emitted C99 (golden fixtures) and the oracle, on a B200."""
import numpy as np
import pytest

from conftest import BATCH_FIXTURES, load_batch, load_dropin_cases, tolerance, GOLDEN
from intception_b200 import basis, eri
from oracle import loader

pytestmark = pytest.mark.gpu


def run_batch(b, **kw):
    import torch
    eng = eri.EriEngine(b)
    out = eng.compute(**kw)
    torch.cuda.synchronize()
    assert eng.device_status() == 0
    return out.cpu().numpy()


@pytest.mark.parametrize('name', BATCH_FIXTURES)
def test_batch_matches_reference_golden(name):
    b, T, ref = load_batch(name)
    out = run_batch(b)
    assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('k', range(12))
def test_dropin_matches_reference_golden(k):
    shells, ref, sph = load_dropin_cases()[k]
    out = np.full(ref.shape, -7.0)
    (eri.cont_sph_main if sph else eri.cont_cart_main)(shells, out)
    assert np.array_equal(out == -7.0, ref == -7.0)  # elements outside the strided block untouched
    assert np.abs(out - ref).max() <= tolerance(ref)


def _all_l2_orderings(seed, sph, kmax=4, copies=1, box=3.0):
    """copies x the 81 (la,lb,lc,ld) orderings with l <= 2, fresh shells each."""
    rng = np.random.default_rng(seed)
    quartets = []
    ls = []
    for _ in range(copies):
        for la in range(3):
            for lb in range(3):
                for lc in range(3):
                    for ld in range(3):
                        base = len(ls)
                        ls += [la, lb, lc, ld]
                        quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.integers(1, kmax + 1, len(ls)).astype(np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, 0.1, 40.0, box)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    return basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)


@pytest.mark.parametrize('cap', [1, 2, 4, 8, 16, 32, 64, 0])
@pytest.mark.parametrize('sph', [False, True])
def test_slices_every_l2_class_vs_oracle(cap, sph):
    """Every slice count (lane groups sharing one quartet, forced by the cap;
    0 = as many as the grid allows, up to a whole block) gives the oracle's
    blocks: 3 x 81 orderings, K up to 6 so that slices get uneven shares of
    the primitive quartets."""
    b = _all_l2_orderings(71 + sph, sph, kmax=6, copies=3)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    eri.set_slice_cap(cap)
    try:
        out = run_batch(b)
    finally:
        eri.set_slice_cap(0)
    assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('sph', [False, True])
def test_long_contractions_span_pair_tiles(sph):
    """K up to 20 per shell (up to 400 primitive pairs a side): the live-pair
    lists run over several 64 x 64 tiles of a quartet; every l <= 2 ordering,
    FP64, against the oracle; slices forced both ways."""
    rng = np.random.default_rng(97 + sph)
    quartets, ls = [], []
    for la in range(3):
        for lb in range(3):
            for lc in range(3):
                for ld in range(3):
                    base = len(ls)
                    ls += [la, lb, lc, ld]
                    quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.choice(np.array([1, 7, 9, 13, 20], np.int32), len(ls))
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, 0.1, 30.0, 2.5)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    b = basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)
    assert (k_[q[:, 0]] * k_[q[:, 1]] > 64).any() and (k_[q[:, 2]] * k_[q[:, 3]] > 64).any()
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    for cap in (1, 0):
        eri.set_slice_cap(cap)
        try:
            out = run_batch(b)
        finally:
            eri.set_slice_cap(0)
        assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('minb', [1, 3, 4, 5])
def test_every_register_budget_vs_oracle(minb):
    """Each register budget the class kernels are compiled with (minimum
    resident blocks per SM) gives the oracle's blocks, FP64 Cartesian and
    spherical, and the FP32 tier stays within 1e-10 of FP64."""
    import torch
    from intception_b200.emit.eri_emitter import canonical_classes
    classes = canonical_classes(2)
    try:
        eri.set_class_fp32(True)  # every class's FP32 kernel, also where the tuned default skips it
        for cls in classes:
            for v4 in range(4):
                eri.set_class_minb(cls, v4, minb)
        for sph in (False, True):
            b = _all_l2_orderings(91 + sph, sph, kmax=5, copies=2)
            ref = loader.oracle_batch(b, basis.sph_matrices(6))
            eng = eri.EriEngine(b)
            out = eng.compute()
            bounds = torch.ones(b.nq, dtype=torch.float64, device='cuda')
            mix = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, fp32_below=2.0, mixed_tol=5e-11)
            torch.cuda.synchronize()
            assert eng.device_status() == 0
            assert np.abs(out.cpu().numpy() - ref).max() <= tolerance(ref)
            assert np.abs(mix.cpu().numpy() - ref).max() <= 1e-10
    finally:
        eri.set_class_fp32(None)
        for cls in classes:
            for v4 in range(4):
                eri.set_class_minb(cls, v4, 0)


@pytest.mark.parametrize('cap', [1, 4, 0])
def test_slices_mixed_tier_meets_error_bar(cap):
    """The FP32 tier sums its rounding-error bound over the slices: the
    rejected quartets are redone in FP64, the rest stay within 1e-10."""
    import torch
    b = _all_l2_orderings(81, True, kmax=6, copies=4, box=2.0)
    eng = eri.EriEngine(b)
    eri.set_slice_cap(cap)
    eri.set_class_fp32(True)
    try:
        ref = eng.compute().clone()
        bounds = eng.quartet_bounds()
        mix = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, skip_below=1e-14, fp32_below=1e-2,
                          mixed_tol=5e-11).clone()
        torch.cuda.synchronize()
    finally:
        eri.set_slice_cap(0)
        eri.set_class_fp32(None)
    assert eng.device_status() == 0
    assert np.abs(mix.cpu().numpy() - ref.cpu().numpy()).max() <= 1e-10


def test_fp32_switch_per_class():
    """With every class's FP32 kernel switched off the FP32 tier reproduces the
    FP64 path bit for bit; switched on for one class only, only that class's
    blocks move (within the error bar)."""
    import torch
    b = _all_l2_orderings(83, True, kmax=4, copies=2, box=2.0)
    eng = eri.EriEngine(b)
    bounds = torch.ones(b.nq, dtype=torch.float64, device='cuda')
    ref = eng.compute().cpu().numpy()
    try:
        eri.set_class_fp32(False)
        off = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, fp32_below=2.0, mixed_tol=1e300).cpu().numpy()
        assert np.array_equal(off, ref)
        eri.set_class_fp32(True, (2, 2, 2, 1))
        # every FP32 result accepted (no error-bound rejection), so they show
        one = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, fp32_below=2.0, mixed_tol=1e300).cpu().numpy()
        torch.cuda.synchronize()
    finally:
        eri.set_class_fp32(None)
    assert eng.device_status() == 0
    assert np.abs(one - ref).max() <= 1e-5 * np.abs(ref).max()  # FP32-VRR rounding, nothing else
    moved = np.nonzero(one != ref)[0]
    assert len(moved) > 0
    ls = b.shell_l[b.quartets]
    sizes = basis.block_sizes(b.shell_l, b.quartets, True)
    q_of = np.searchsorted(b.out_off, moved, side='right') - 1
    for q in np.unique(q_of):
        assert sorted(ls[q]) == [1, 2, 2, 2], ls[q]
    assert np.all(moved < b.out_off[q_of] + sizes[q_of])


@pytest.mark.parametrize('sph', [False, True])
def test_every_l2_class_vs_oracle(sph):
    """All 81 (la,lb,lc,ld) orderings with l <= 2, i.e. every canonical class
    reached through every permutation of shells and strides."""
    rng = np.random.default_rng(31 + sph)
    quartets = []
    ls = []
    for la in range(3):
        for lb in range(3):
            for lc in range(3):
                for ld in range(3):
                    base = len(ls)
                    ls += [la, lb, lc, ld]
                    quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.integers(1, 5, len(ls)).astype(np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, 0.1, 40.0, 3.0)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    b = basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    out = run_batch(b)
    assert np.abs(out - ref).max() <= tolerance(ref)


# (exponent range, box edge in bohr, max abs error allowed).  The 0.1..40
# range three bohr apart is the hard case: with the diffuse shell of an
# equal-l pair first, the contracted [e0|f0] intermediates reach 2e3 for
# blocks of 1e-2 and the HRRs cancel six digits (5.5e-12 error measured);
# the batch entries put the more compact shell first (4e-14 measured).
F_DISTS = [(0.3, 5.0, 3.0, 1e-12), (0.3, 5.0, 6.0, 1e-12), (0.1, 40.0, 1.0, 1e-12), (0.5, 20.0, 4.0, 1e-12),
           (0.1, 40.0, 3.0, 1e-12), (0.3, 40.0, 5.0, 1e-12)]


@pytest.mark.parametrize('sph', [False, True])
@pytest.mark.parametrize('dist', range(len(F_DISTS)))
def test_every_f_class_vs_oracle(dist, sph):
    """All 175 (la,lb,lc,ld) orderings with l <= 3 and at least one f shell,
    (ff|ff) included, two copies each with fresh shells and K 1..3."""
    lo, hi, box, tol = F_DISTS[dist]
    rng = np.random.default_rng(57 + sph + 10 * dist)
    quartets = []
    ls = []
    for _ in range(2):
        for la in range(4):
            for lb in range(4):
                for lc in range(4):
                    for ld in range(4):
                        if max(la, lb, lc, ld) < 3:
                            continue
                        base = len(ls)
                        ls += [la, lb, lc, ld]
                        quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.integers(1, 4, len(ls)).astype(np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, lo, hi, box)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    b = basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    out = run_batch(b)
    assert np.abs(out - ref).max() <= tol * max(1.0, float(np.abs(ref).max()))


G_DISTS = [(0.3, 5.0, 3.0), (0.3, 5.0, 6.0), (0.5, 20.0, 4.0), (0.1, 40.0, 3.0)]


@pytest.mark.parametrize('sph', [False, True])
@pytest.mark.parametrize('dist', range(len(G_DISTS)))
def test_every_g_class_vs_oracle(dist, sph):
    """All 369 (la,lb,lc,ld) orderings with l <= 4 and at least one g shell:
    the unrolled lane-group kernels (61 canonical classes) and the generic
    kernel for (gf|gf), (gg|gf), (gg|gg) and (gg|ss); K 1..2, fresh shells.

    The one exception to the flat 1e-12 bar: 2e-12 here.  In the two settings
    with shells 3 bohr apart, four-level horizontal recurrences on both sides
    cancel two to three digits (HRR growth factors of 1e2 to 2e4 measured on
    the worst quartets), and the measured maximum is 1.21e-12 on blocks of
    1e-2 (the reference builds the ket by vertical recurrences on c and d and
    has no ket HRR to amplify its rounding)."""
    lo, hi, box = G_DISTS[dist]
    rng = np.random.default_rng(157 + sph + 10 * dist)
    quartets, ls = [], []
    for la in range(5):
        for lb in range(5):
            for lc in range(5):
                for ld in range(5):
                    if max(la, lb, lc, ld) < 4:
                        continue
                    base = len(ls)
                    ls += [la, lb, lc, ld]
                    quartets.append([base, base + 1, base + 2, base + 3])
    ks = rng.integers(1, 3, len(ls)).astype(np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, np.array(ls, np.int32), ks, lo, hi, box)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    b = basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)
    ref = loader.oracle_batch(b, basis.sph_matrices(6))
    out = run_batch(b)
    assert np.abs(out - ref).max() <= 2e-12


def test_boys_dropin_vs_reference():
    z = np.load(GOLDEN + '/boys.npz')
    nmax = int(z['nmax'])
    for x, F in zip(z['x'], z['F']):
        f = eri.boys(nmax, x)
        # the reference drops exp(-x) above x = 35; both are below 1e-14 there
        assert np.abs(f - F).max() <= 2e-14, x


def test_boys_batch_accuracy():
    import torch
    from oracle import md_eri
    xs = np.concatenate([np.linspace(0, 40, 801), [1e-13, 35.999, 36.0, 36.001, 60.0, 500.0]])
    nmax = 16
    x = torch.tensor(xs, dtype=torch.float64, device='cuda')
    f = torch.empty(len(xs) * (nmax + 1), dtype=torch.float64, device='cuda')
    lib = eri.load()
    st = lib.intception_b200_boys_batch(x.data_ptr(), len(xs), nmax, f.data_ptr(), None)
    assert st == 0
    lib.intception_b200_synchronize()
    torch.cuda.synchronize()
    f = f.cpu().numpy().reshape(len(xs), nmax + 1)
    ex = np.array([[md_eri.boys(m, v) for m in range(nmax + 1)] for v in xs])
    assert np.abs(f - ex).max() < 5e-15


def test_dropin_rejects_bad_l_and_n():
    shells, ref, sph = load_dropin_cases()[0]
    bad = [dict(s) for s in shells]
    bad[0]['l'] = 7
    out = np.full(ref.shape, -7.0)
    with pytest.raises(eri.IntceptionError):
        eri.cont_cart_main(bad, out)
    assert np.all(out == -7.0)
    bad = [dict(s) for s in shells]
    bad[2]['n'] = bad[2]['n'] + 1
    with pytest.raises(eri.IntceptionError):
        eri.cont_cart_main(bad, out)
    assert np.all(out == -7.0)
    # a good call afterwards still works
    eri.cont_cart_main(shells, out)
    assert np.abs(out - ref).max() <= tolerance(ref)


def test_batch_reports_l_above_basis_lmax():
    import torch
    b, T, ref = load_batch('pppp_k3_cart')
    eng = eri.EriEngine(b)
    eng._basis.lmax = 0  # declared lmax below the shells' l
    eng.compute()
    torch.cuda.synchronize()
    assert eng.device_status() == eri.IB_ERR_ARG


def test_permutational_symmetry_large():
    """(ab|cd) = (ba|cd) = (cd|ab) through different canonicalisation paths,
    at 100k quartets of the l<=2 spherical workload."""
    b = basis.config_mixed_l2(nq=100_000, seed=17, spherical=True)
    out = run_batch(b)
    q2 = b.quartets[:, [2, 3, 0, 1]].copy()
    b2 = basis.ShellBatch(b.shell_l, b.shell_k, b.shell_ptr, b.shell_xyz, b.prim_exp, b.prim_coef, q2,
                          *basis.packed_offsets(b.shell_l, q2, True)[:1], True, b.out_size)
    out2 = run_batch(b2)
    # compare block by block: (cd|ab)[ic,id,ia,ib] == (ab|cd)[ia,ib,ic,id]
    ls = b.shell_l[b.quartets]
    n = 2 * ls + 1
    for q in range(0, b.nq, 997):
        na, nb, nc, nd = n[q]
        x = out[b.out_off[q]:b.out_off[q] + na * nb * nc * nd].reshape(nd, nc, nb, na)
        y = out2[b2.out_off[q]:b2.out_off[q] + na * nb * nc * nd].reshape(nb, na, nd, nc)
        assert np.abs(x - y.transpose(2, 3, 0, 1)).max() <= 1e-13 * max(1.0, np.abs(x).max())


def _block_max(b, x):
    sizes = basis.block_sizes(b.shell_l, b.quartets, b.spherical)
    seg = np.repeat(np.arange(b.nq), sizes)
    m = np.zeros(b.nq)
    np.maximum.at(m, seg, np.abs(x))
    return m


def test_schwarz_bounds_hold():
    """|(ab|cd)| <= q_ab q_cd for every element (compact 8-bohr box, so most
    bounds are far from zero)."""
    import torch
    b = basis.independent_quartet_batch(51, 20000, [0, 1, 2], [1, 2, 3, 4], 0.05, 1e4, 8.0, True)
    eng = eri.EriEngine(b)
    ref = eng.compute()
    bounds = eng.quartet_bounds()
    torch.cuda.synchronize()
    m = _block_max(b, ref.cpu().numpy())
    bd = bounds.cpu().numpy()
    assert np.all(m <= bd * (1 + 1e-10) + 1e-300)
    # the factors match an explicit diagonal evaluation for a few pairs
    for p in (0, 7, 1234):
        a, bb = b.quartets[p, 0], b.quartets[p, 1]
        q = np.array([[a, bb, a, bb]], np.int32)
        off, tot = basis.packed_offsets(b.shell_l, q, True)
        sub = basis.ShellBatch(b.shell_l, b.shell_k, b.shell_ptr, b.shell_xyz, b.prim_exp, b.prim_coef, q, off,
                               True, tot)
        blk = loader.oracle_batch(sub, basis.sph_matrices(6))
        na, nb = 2 * b.shell_l[a] + 1, 2 * b.shell_l[bb] + 1
        diag = max(abs(blk[i + na * (j + nb * (i + na * j))]) for i in range(na) for j in range(nb))
        qab = float(eng.schwarz(torch.tensor([[a, bb]], dtype=torch.int32, device='cuda'))[0])
        assert abs(qab - np.sqrt(diag)) <= 1e-12 * max(1.0, np.sqrt(diag))


def test_screened_and_mixed_paths_meet_error_bar():
    """l<=2 spherical workload (30-bohr cube): screening writes zeros below
    1e-12 (error <= bound), the mixed path keeps the max abs error <= 1e-10."""
    import torch
    b = basis.config_mixed_l2(nq=50000, seed=21, spherical=True)
    eng = eri.EriEngine(b)
    ref = eng.compute().clone()
    bounds = eng.quartet_bounds()
    scr = eng.compute(bounds=bounds, skip_below=1e-12).clone()
    mix = eng.compute(precision=eri.PREC_MIXED, bounds=bounds, skip_below=1e-12, fp32_below=1e-4,
                      mixed_tol=5e-11).clone()
    torch.cuda.synchronize()
    assert eng.device_status() == 0
    r = ref.cpu().numpy()
    assert np.abs(scr.cpu().numpy() - r).max() <= 1e-12
    assert np.abs(mix.cpu().numpy() - r).max() <= 1e-10
    kept = (bounds >= 1e-12).double().mean().item()
    assert 0.0 < kept < 1.0


def test_cuda_graph_replay_matches_direct_batch():
    """The captured pipeline (sort, items, every class kernel, side-stream
    fork/join) replays to the same blocks, also after the inputs change."""
    import torch
    b = basis.config_mixed_l2(nq=20000, seed=61, spherical=True)
    eng = eri.EriEngine(b)
    ref = eng.compute().clone()
    out = torch.full_like(ref, float('nan'))
    g = eng.graph(out)
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    # replay reads the current inputs: move every shell and compare again
    eng.shell_xyz.add_(0.25)
    ref2 = eng.compute().clone()
    out.fill_(float('nan'))
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(out, ref2)
    g.close()


def test_host_pipeline_matches_direct_batches():
    """Three batches queued back to back through the host pipeline (two device
    buffer sets, so the third reuses the first's) give the same blocks, bit for
    bit, as the direct batch entry; a screened batch with bounds as well."""
    import torch
    batches = [basis.config_mixed_l2(nq=n, seed=s, spherical=True) for n, s in ((3000, 41), (5000, 42), (2000, 43))]
    refs = []
    for b in batches:
        eng = eri.EriEngine(b)
        refs.append(eng.compute().cpu().numpy())
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    pipe = eri.HostPipeline(True, depth=2)
    outs = []
    for b in batches:
        h = {'shell_l': pin(b.shell_l), 'shell_k': pin(b.shell_k), 'shell_ptr': pin(b.shell_ptr),
             'shell_xyz': pin(b.shell_xyz), 'prim_exp': pin(b.prim_exp), 'prim_coef': pin(b.prim_coef),
             'quartets': pin(b.quartets.reshape(-1)), 'out_off': pin(b.out_off)}
        o = torch.full((b.out_size,), float('nan'), dtype=torch.float64).pin_memory()
        pipe.submit(h, o)
        outs.append(o)
    pipe.synchronize()
    for o, r in zip(outs, refs):
        assert np.array_equal(o.numpy(), r)
    # screened: bounds travel with the batch
    b = batches[1]
    eng = eri.EriEngine(b)
    bounds = eng.quartet_bounds()
    ref = eng.compute(bounds=bounds, skip_below=1e-12).cpu().numpy()
    h = {'shell_l': pin(b.shell_l), 'shell_k': pin(b.shell_k), 'shell_ptr': pin(b.shell_ptr),
         'shell_xyz': pin(b.shell_xyz), 'prim_exp': pin(b.prim_exp), 'prim_coef': pin(b.prim_coef),
         'quartets': pin(b.quartets.reshape(-1)), 'out_off': pin(b.out_off), 'bounds': bounds.cpu().pin_memory()}
    o = torch.empty(b.out_size, dtype=torch.float64).pin_memory()
    pipe.submit(h, o, skip_below=1e-12)
    pipe.synchronize()
    assert np.array_equal(o.numpy(), ref)


def test_fp32_rejection_count_covers_only_the_last_batch():
    """intception_b200_last_fp32_rejections counts the flags of the last mixed
    batch only: a large batch whose every FP32 attempt is rejected, then a
    smaller one that rejects nothing, must report 0 (the flag buffer still
    holds the large batch's flags past the small batch's end)."""
    import torch
    big = _all_l2_orderings(123, True, kmax=4, copies=4)
    small = big.subset(np.arange(40))
    try:
        eri.set_class_fp32(True)
        for b, tol, want_any in ((big, 1e-300, True), (small, 1.0, False)):
            eng = eri.EriEngine(b)
            bounds = torch.ones(b.nq, dtype=torch.float64, device='cuda')
            eng.compute(precision=eri.PREC_MIXED, bounds=bounds, fp32_below=2.0, mixed_tol=tol)
            torch.cuda.synchronize()
            assert eng.device_status() == 0
            n = eng.fp32_rejected()
            assert (n > 0) if want_any else (n == 0), n
            assert n <= b.nq
    finally:
        eri.set_class_fp32(None)


def test_c1_every_quartet_through_the_dropin():
    """The (pp|pp) K=3 Cartesian configuration at its full size (4096
    quartets, seed 0): every quartet through the drop-in
    intception_integral_eri_abcd_m_cont_cart_main, one call per quartet as the
    reference's caller makes them, against the reference's emitted C99 at a
    flat 1e-12 absolute; the batch entry covers the same fixture in
    test_batch_matches_reference_golden."""
    b, T, ref = load_batch('c1_pppp_k3_cart_4096')
    assert b.nq == 4096
    worst = 0.0
    for q in range(b.nq):
        shells = []
        for i, s in enumerate(b.quartets[q]):
            p0, k = int(b.shell_ptr[s]), int(b.shell_k[s])
            shells.append(dict(x=b.prim_exp[p0:p0 + k], cen=b.shell_xyz[s], coef=b.prim_coef[p0:p0 + k], l=1, n=3,
                               iskip=3 ** i, nprim=k, ncont=1, iskip_cont=81))
        out = np.zeros(81)
        eri.cont_cart_main(shells, out)
        r = ref[b.out_off[q]:b.out_off[q] + 81]
        worst = max(worst, float(np.abs(out - r).max()))
    assert worst <= 1e-12, worst


@pytest.mark.parametrize('sph', [False, True])
def test_analytic_quartet_bounds_match_oracle_and_cover_blocks(sph):
    """intception_b200_quartet_bounds against its C restatement (oracle/pair_bound.h,
    FP64): the device evaluates the primitive-pair terms in float and widens
    them by 1.001, so it must lie in [1, 1.01] x the restatement, l <= 6; every
    block of the batch path stays within its bound, and screening with it errs
    by no more than the threshold."""
    import torch
    b = basis.independent_quartet_batch(131 + sph, 600, [0, 1, 2, 3, 4, 5, 6], [1, 2, 3, 6], 0.05, 1e4, 8.0, sph)
    eng = eri.EriEngine(b)
    dev = eng.analytic_bounds().cpu().numpy()
    ora = loader.quartet_bounds(b)
    assert np.all(dev >= ora)
    assert np.all(dev <= 1.01 * ora)
    out = run_batch(b)
    sizes = basis.block_sizes(b.shell_l, b.quartets, b.spherical)
    for q in range(b.nq):
        assert np.abs(out[b.out_off[q]:b.out_off[q] + sizes[q]]).max() <= dev[q]
    thr = float(np.quantile(dev, 0.5))
    scr = eng.compute(bounds=torch.from_numpy(dev).cuda(), skip_below=thr)
    torch.cuda.synchronize()
    assert np.abs(scr.cpu().numpy() - out).max() <= thr


@pytest.mark.parametrize('sph', [False, True])
def test_ill_conditioned_pairs_built_on_the_compact_shell(sph):
    """Bra pairs of a diffuse higher-l shell and a tight lower-l shell a few
    bohr apart: built on the higher-l shell, their horizontal recurrence would
    cancel up to ~10 digits, so the batch entry routes them to the generic
    kernel built on the tight shell.  Checked at a flat 1e-12 against the
    oracle evaluated in the stable order (the tight shell first, its block
    transposed back); K 1..3, l up to 6."""
    rng = np.random.default_rng(211 + sph)
    lpairs = [(2, 1), (3, 1), (3, 2), (4, 1), (4, 2), (4, 3), (5, 2), (6, 4)]
    ls, xs, cs, cens, ks, quartets = [], [], [], [], [], []
    for rep in range(3):
        for la, lb in lpairs:
            lc, ld = int(rng.integers(0, 3)), int(rng.integers(0, 3))
            A = rng.uniform(0, 1, 3)
            u = rng.normal(size=3)
            B = A + rng.uniform(2.0, 5.0) * u / np.linalg.norm(u)
            for l, lo, hi, cen in ((la, 0.05, 0.3, A), (lb, 1e3, 1e5, B), (lc, 0.3, 10.0, A + 0.5),
                                   (ld, 0.3, 10.0, B - 0.4)):
                k = int(rng.integers(1, 4))
                e = np.exp(rng.uniform(np.log(lo), np.log(hi), k))
                ls.append(l)
                ks.append(k)
                xs.append(e)
                cs.append(basis.normalize_shell(l, e, rng.uniform(0.1, 1.0, k)))
                cens.append(cen)
            n = len(ls)
            quartets.append([n - 4, n - 3, n - 2, n - 1])
    l_ = np.array(ls, np.int32)
    k_ = np.array(ks, np.int32)
    p_ = np.concatenate([[0], np.cumsum(k_)[:-1]]).astype(np.int32)
    q = np.array(quartets, np.int32)
    off, total = basis.packed_offsets(l_, q, sph)
    b = basis.ShellBatch(l_, k_, p_, np.array(cens), np.concatenate(xs), np.concatenate(cs), q, off, sph, total)
    out = run_batch(b)
    # the oracle with each quartet's bra shells swapped (built on the tight shell)
    qs = q[:, [1, 0, 2, 3]].copy()
    offs, tots = basis.packed_offsets(l_, qs, sph)
    bs = basis.ShellBatch(l_, k_, p_, np.array(cens), np.concatenate(xs), np.concatenate(cs), qs, offs, sph, tots)
    refs = loader.oracle_batch(bs, basis.sph_matrices(6))
    worst = 0.0
    for i in range(b.nq):
        n = [2 * l_[s] + 1 if sph else (l_[s] + 1) * (l_[s] + 2) // 2 for s in q[i]]
        blk = refs[offs[i]:offs[i] + np.prod(n)].reshape(n[3], n[2], n[0], n[1]).transpose(0, 1, 3, 2).ravel()
        worst = max(worst, float(np.abs(out[off[i]:off[i] + np.prod(n)] - blk).max()))
    assert worst <= tolerance(refs), worst


@pytest.mark.parametrize('sph', [False, True])
def test_df_class_kernels_for_ill_conditioned_fd_pairs(sph):
    """(f d) pairs of a diffuse f and a tight d shell 2-4 bohr apart, in the
    bra, the ket or both, against partners up to f: the (d f| class kernels
    (the d shell built on) must match, at the flat bar, the oracle evaluated
    with every such pair swapped (its stable order), block transposed back."""
    rng = np.random.default_rng(311 + sph)
    ls, xs, cs, cens, ks, quartets, swaps = [], [], [], [], [], [], []

    def shell(l, lo, hi, cen):
        k = int(rng.integers(1, 3))
        e = np.exp(rng.uniform(np.log(lo), np.log(hi), k))
        ls.append(l)
        ks.append(k)
        xs.append(e)
        cs.append(basis.normalize_shell(l, e, rng.uniform(0.1, 1.0, k)))
        cens.append(cen)
        return len(ls) - 1

    def fd_pair():
        A = rng.uniform(0, 1, 3)
        u = rng.normal(size=3)
        return shell(3, 0.08, 0.3, A), shell(2, 2e3, 5e4, A + rng.uniform(2.0, 4.0) * u / np.linalg.norm(u))

    for rep in range(4):
        for kind in ('bra', 'ket', 'both'):
            for lp in [(0, 0), (1, 0), (2, 1), (3, 3), (3, 1)]:
                if kind == 'both':
                    a, b = fd_pair()
                    c, d = fd_pair()
                    quartets.append([a, b, c, d])
                    swaps.append((True, True))
                else:
                    a, b = fd_pair()
                    C = rng.uniform(0, 3, 3)
                    c = shell(lp[0], 0.3, 20.0, C)
                    d = shell(lp[1], 0.3, 20.0, C + 0.7)
                    quartets.append([a, b, c, d] if kind == 'bra' else [c, d, a, b])
                    swaps.append((kind == 'bra', kind == 'ket'))
    l_ = np.array(ls, np.int32)
    k_ = np.array(ks, np.int32)
    p_ = np.concatenate([[0], np.cumsum(k_)[:-1]]).astype(np.int32)
    q = np.array(quartets, np.int32)
    def mk(qq):
        off, total = basis.packed_offsets(l_, qq, sph)
        return basis.ShellBatch(l_, k_, p_, np.array(cens), np.concatenate(xs), np.concatenate(cs), qq, off, sph,
                                total)

    b = mk(q)
    out = run_batch(b)
    qs = q.copy()
    for i, (sb, sk) in enumerate(swaps):
        if sb:
            qs[i, [0, 1]] = qs[i, [1, 0]]
        if sk:
            qs[i, [2, 3]] = qs[i, [3, 2]]
    bs = mk(qs)
    refs = loader.oracle_batch(bs, basis.sph_matrices(6))
    worst = 0.0
    for i in range(b.nq):
        n = [2 * l_[s] + 1 if sph else (l_[s] + 1) * (l_[s] + 2) // 2 for s in q[i]]
        ns = [n[1], n[0], n[2], n[3]] if swaps[i][0] else list(n)
        if swaps[i][1]:
            ns[2], ns[3] = ns[3], ns[2]
        blk = refs[bs.out_off[i]:bs.out_off[i] + np.prod(n)].reshape(ns[3], ns[2], ns[1], ns[0])
        if swaps[i][0]:
            blk = blk.transpose(0, 1, 3, 2)
        if swaps[i][1]:
            blk = blk.transpose(1, 0, 2, 3)
        worst = max(worst, float(np.abs(out[b.out_off[i]:b.out_off[i] + np.prod(n)] - blk.ravel()).max()))
    assert worst <= tolerance(refs), worst
