"""Generate the golden ERI fixtures from the reference's own emitted C99.

Run in a container that has the reference tree (it builds oracle/_ref first):
    python oracle/gen_ref.py && python tests/golden/make_golden.py
(``make_golden.py twoidx`` writes only twoidx.npz, ``make_golden.py c1`` only
c1_pppp_k3_cart_4096.npz, ``make_golden.py mixed`` only
mixed_contraction_sph.npz, whose ``out`` is exact (binary128) and whose
``ref_out`` is the reference's.)

Every fixture stores seeded inputs (shell table, quartets, spherical matrices)
and the outputs of intception_integral_eri_abcd_m_cont_{cart,sph}_main as
emitted by the reference generator for oracle/eri_input.py.  The GPU box has
no reference tree; the tests read these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from intception_b200 import basis  # noqa: E402
from oracle import loader  # noqa: E402


def save_batch(name, b, T, out, **extra):
    np.savez_compressed(os.path.join(HERE, name), shell_l=b.shell_l, shell_k=b.shell_k, shell_ptr=b.shell_ptr,
                        shell_xyz=b.shell_xyz, prim_exp=b.prim_exp, prim_coef=b.prim_coef, quartets=b.quartets,
                        out_off=b.out_off, spherical=np.int32(b.spherical), out_size=np.int64(b.out_size),
                        sph=np.concatenate([t.ravel(order='F') for t in T]), out=out, **extra)
    print(name, b.nq, 'quartets, max |I| = %.3e' % np.abs(out).max())


def ref(b, T):
    out = loader.ref_batch(b, T, nthreads=0)
    assert out is not None, 'oracle/_ref not built (python oracle/gen_ref.py)'
    return out


def edge_batch(spherical):
    """Hand-built edge cases: coincident centres (T = 0), a far ket pair (T
    above every table), very tight and very diffuse exponents, K = 1 and mixed
    K, one shell repeated four times in a quartet.  Shell j = kind*3 + l."""
    rng = np.random.default_rng(11)
    origin = np.zeros(3)
    kinds = [(1, origin, (1.0, 1.0)),                       # 0: single primitive at the origin
             (3, origin, (0.02, 0.05)),                     # 1: diffuse
             (2, np.array([0.0, 0.0, 25.0]), (1e4, 1e5)),   # 2: tight, 25 bohr away
             (4, origin + 0.3, (0.1, 100.0))]               # 3: generic
    ls, ks, cen, exps, coefs = [], [], [], [], []
    for k, c, (lo, hi) in kinds:
        for l in range(3):
            e = np.exp(rng.uniform(np.log(lo), np.log(hi), k))
            ls.append(l)
            ks.append(k)
            cen.append(c)
            exps.append(e)
            coefs.append(basis.normalize_shell(l, e, rng.uniform(0.1, 1.0, k)))

    def sh(kind, l):
        return kind * 3 + l

    quartets = []
    for la in range(3):
        for lb in range(3):
            for lc in range(3):
                for ld in range(3):
                    quartets.append([sh(0, la), sh(0, lb), sh(0, lc), sh(0, ld)])  # all at the origin, T = 0
                    quartets.append([sh(3, la), sh(1, lb), sh(2, lc), sh(2, ld)])  # far ket pair
                    quartets.append([sh(3, la), sh(3, lb), sh(3, lc), sh(3, ld)])  # repeated shells
    q = np.array(quartets, np.int32)
    l_arr = np.array(ls, np.int32)
    k_arr = np.array(ks, np.int32)
    ptr = np.zeros(len(ls), np.int32)
    ptr[1:] = np.cumsum(k_arr)[:-1]
    off, total = basis.packed_offsets(l_arr, q, spherical)
    return basis.ShellBatch(l_arr, k_arr, ptr, np.array(cen), np.concatenate(exps), np.concatenate(coefs), q,
                            off, spherical, total)


def main():
    T = basis.sph_matrices(6)
    # C1 shape: (pp|pp) K=3, 10-bohr cube, Cartesian
    b = basis.config_pppp_k3(nq=256, seed=0)
    save_batch('pppp_k3_cart.npz', b, T, ref(b, T))
    # C2 distribution (30-bohr cube) and a compact 6-bohr variant with larger values
    b = basis.config_mixed_l2(nq=400, seed=1, spherical=True)
    save_batch('mixed_l2_sph_c2.npz', b, T, ref(b, T))
    b = basis.independent_quartet_batch(5, 400, [0, 1, 2], [1, 2, 3, 4, 5, 6], 0.05, 1.0e4, 6.0, True)
    save_batch('mixed_l2_sph_compact.npz', b, T, ref(b, T))
    b = basis.independent_quartet_batch(6, 300, [0, 1, 2], [1, 2, 3], 0.1, 50.0, 5.0, False)
    save_batch('mixed_l2_cart_compact.npz', b, T, ref(b, T))
    # higher angular momentum through the generic kernel
    b = basis.independent_quartet_batch(7, 40, [0, 1, 2, 3, 4], [1, 2], 0.1, 30.0, 4.0, False)
    save_batch('l4_cart.npz', b, T, ref(b, T))
    b = basis.independent_quartet_batch(8, 24, [2, 3, 4], [1, 2], 0.1, 30.0, 4.0, True)
    save_batch('l4_sph.npz', b, T, ref(b, T))
    # l up to 6 (the reference's global_user_lmax): one shell per l, chosen quartets
    rng = np.random.default_rng(9)
    ls = np.arange(7, dtype=np.int32)
    l_, k_, p_, xyz, e, c = basis.make_shells(rng, ls, np.array([1, 2, 1, 2, 1, 1, 1], np.int32), 0.3, 3.0, 3.0)
    q = np.array([[6, 0, 0, 0], [5, 1, 2, 0], [6, 6, 0, 0], [4, 5, 1, 1], [6, 2, 3, 0], [0, 3, 6, 1]], np.int32)
    for sph in (False, True):
        off, total = basis.packed_offsets(l_, q, sph)
        b = basis.ShellBatch(l_, k_, p_, xyz, e, c, q, off, sph, total)
        save_batch('l6_%s.npz' % ('sph' if sph else 'cart'), b, T, ref(b, T))
    for sph in (False, True):
        b = edge_batch(sph)
        save_batch('edge_%s.npz' % ('sph' if sph else 'cart'), b, T, ref(b, T))
    # drop-in cases: general contraction (cases 4, 5: K = 6, three contracted
    # functions on b), caller strides with gaps, caller matrices (case 3: random)
    rng = np.random.default_rng(12)
    cases = []
    ref_cart = loader.load_ref('cart')
    ref_sph = loader.load_ref('sph')
    for case in range(12):
        sph = case % 2 == 1
        ls = rng.integers(0, 4 if case < 8 else 5, 4)
        shells = []
        for i in range(4):
            l = int(ls[i])
            nprim = int(rng.integers(1, 4)) if case not in (4, 5) else 6
            ncont = int(rng.integers(1, 3)) if case not in (4, 5) else (3 if i == 1 else 1)
            x = np.exp(rng.uniform(np.log(0.1), np.log(20.0), nprim))
            coef = rng.uniform(-1.0, 1.0, (nprim, ncont))
            for k in range(ncont):
                coef[:, k] = basis.normalize_shell(l, x, np.abs(coef[:, k]) + 0.1)
            ncart = (l + 1) * (l + 2) // 2
            nn = 2 * l + 1 if sph else ncart
            Tm = rng.normal(size=(ncart, 2 * l + 1)) if case == 3 else T[l]
            shells.append(dict(x=x, cen=rng.uniform(0, 4.0, 3), l=l, n=nn, nprim=nprim, ncont=ncont,
                               coef=coef.ravel(order='F'), T=Tm))
        # strides: a fastest with a padded gap between blocks of b, and cont strides outermost
        dims = [s['n'] for s in shells]
        cont = [s['ncont'] for s in shells]
        st = [1, dims[0] + 1, (dims[0] + 1) * dims[1] + 2, ((dims[0] + 1) * dims[1] + 2) * dims[2]]
        blk = st[3] * dims[3] + 3
        cst = [blk, blk * cont[0], blk * cont[0] * cont[1], blk * cont[0] * cont[1] * cont[2]]
        for i in range(4):
            shells[i]['iskip'] = st[i]
            shells[i]['iskip_cont'] = cst[i]
        size = cst[3] * cont[3]
        out = np.full(size, -7.0)  # untouched elements must stay -7
        work = np.zeros(loader.load_ref('cart').ref_work_array_size(*ls, *[s['nprim'] for s in shells],
                                                                     *cont) + 16)
        loader.call_main(ref_sph if sph else ref_cart, 'sph' if sph else 'cart', shells, work, out)
        cases.append((shells, out, sph))
    flat = {}
    for k, (shells, out, sph) in enumerate(cases):
        flat['case%d_sph' % k] = np.int32(sph)
        flat['case%d_out' % k] = out
        for i, s in enumerate(shells):
            for key in ('x', 'cen', 'coef'):
                flat['case%d_%d_%s' % (k, i, key)] = s[key]
            flat['case%d_%d_T' % (k, i)] = np.asarray(s['T']).ravel(order='F')
            flat['case%d_%d_int' % (k, i)] = np.array([s['l'], s['n'], s['iskip'], s['nprim'], s['ncont'],
                                                       s['iskip_cont']], np.int64)
    flat['ncases'] = np.int32(len(cases))
    np.savez_compressed(os.path.join(HERE, 'dropin_cases.npz'), **flat)
    print('dropin_cases.npz', len(cases), 'cases')
    # Boys function of the reference at edge arguments
    xs = np.array([0.0, 1e-12, 1e-6, 0.05, 0.049999, 1.0, 7.77, 14.95, 15.0, 15.000001, 20.5, 34.99, 35.0,
                   35.01, 50.0, 123.4, 1000.0])
    nmax = 24
    F = np.array([loader.boys(nmax, x, loader.load_ref('cart')) for x in xs])
    np.savez_compressed(os.path.join(HERE, 'boys.npz'), x=xs, nmax=np.int32(nmax), F=F)
    print('boys.npz', len(xs), 'arguments')
    # work_array_size table
    import itertools
    rows = []
    for la, lb, lc, ld in itertools.product(range(5), repeat=4):
        for kp, kc in (((1, 1, 1, 1), (1, 1, 1, 1)), ((3, 2, 4, 1), (1, 2, 1, 1)), ((6, 6, 6, 6), (2, 2, 2, 2))):
            rows.append([la, lb, lc, ld, *kp, *kc, ref_cart.ref_work_array_size(la, lb, lc, ld, *kp, *kc)])
    np.savez_compressed(os.path.join(HERE, 'work_array_size.npz'), table=np.array(rows, np.int64))
    print('work_array_size.npz', len(rows), 'rows')


def twoidx_pairs(seed, n, lmax):
    """Seeded pair set for the two-index classes: random pairs over every
    (la, lb) <= lmax, then hand-built edges (A = B, A = B = C so T = 0, a far
    charge with T above the Boys table, tight and diffuse exponents)."""
    rng = np.random.default_rng(seed)
    la = rng.integers(0, lmax + 1, n)
    lb = rng.integers(0, lmax + 1, n)
    xa = np.exp(rng.uniform(np.log(0.05), np.log(200.0), n))
    xb = np.exp(rng.uniform(np.log(0.05), np.log(200.0), n))
    ca = rng.uniform(0.0, 3.0, (n, 3))
    cb = rng.uniform(0.0, 3.0, (n, 3))
    cc = rng.uniform(0.0, 3.0, (n, 3))
    edges = []
    for l1 in range(lmax + 1):
        for l2 in range(lmax + 1):
            c0 = rng.uniform(0, 1, 3)
            edges.append((l1, l2, 0.8, 1.3, c0, c0, c0 + 0.4))             # A = B
            edges.append((l1, l2, 2.0, 0.7, c0, c0, c0))                   # A = B = C: T = 0
            edges.append((l1, l2, 1.5, 2.5, c0, c0 + 0.2, c0 + 30.0))      # T >= 36
            edges.append((l1, l2, 5e3, 0.02, c0, c0 + 1.0, c0 - 0.5))      # tight with diffuse
    la = np.concatenate([la, [e[0] for e in edges]]).astype(np.int32)
    lb = np.concatenate([lb, [e[1] for e in edges]]).astype(np.int32)
    xa = np.concatenate([xa, [e[2] for e in edges]])
    xb = np.concatenate([xb, [e[3] for e in edges]])
    ca = np.concatenate([ca, [e[4] for e in edges]])
    cb = np.concatenate([cb, [e[5] for e in edges]])
    cc = np.concatenate([cc, [e[6] for e in edges]])
    sizes = ((la + 1) * (la + 2) // 2) * ((lb + 1) * (lb + 2) // 2)
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    return dict(xa=xa, ca=ca.ravel(), la=la, xb=xb, cb=cb.ravel(), lb=lb, cc=cc.ravel(), off=off,
                size=np.int64(sizes.sum()))


def twoidx():
    """twoidx.npz: the reference-emitted overlap_2idx and nuclear_2idx of its
    example script over a seeded pair set, and their work-array sizes."""
    lib = loader.load_ref_2idx()
    assert lib is not None, 'oracle/_ref/libref_2idx.so not built (python oracle/gen_ref.py)'
    pairs = twoidx_pairs(21, 250, 6)
    ov = loader.twoidx_batch(0, pairs, lib)
    nu = loader.twoidx_batch(1, pairs, lib)
    rows = [[k, la, lb, lib.ref_2idx_work_array_size(k, la, lb)] for k in (0, 1) for la in range(7)
            for lb in range(7)]
    np.savez_compressed(os.path.join(HERE, 'twoidx.npz'), overlap=ov, nuclear=nu,
                        work_array_size=np.array(rows, np.int64), **pairs)
    print('twoidx.npz', len(pairs['xa']), 'pairs, max |S| = %.3e, max |V| = %.3e'
          % (np.abs(ov).max(), np.abs(nu).max()))


def c1():
    """c1_pppp_k3_cart_4096.npz: the (pp|pp) K=3 Cartesian configuration at its
    full size, 4096 quartets of four fresh shells, seed 0, through the
    reference's emitted _cont_cart function."""
    T = basis.sph_matrices(6)
    b = basis.config_pppp_k3(nq=4096, seed=0)
    save_batch('c1_pppp_k3_cart_4096.npz', b, T, ref(b, T))


def pair_kappa(b, s0, s1, l_moved, build_first):
    """Growth bound of a pair's HRR (the library's ib_hrr_kappa restated):
    max over primitive pairs of ((sig + |PA| + R) / (sig + |PB|))^l_moved,
    A the shell the recurrences build on."""
    e = lambda s: b.prim_exp[b.shell_ptr[s]:b.shell_ptr[s] + b.shell_k[s]]  # noqa: E731
    x0, x1 = (e(s0), e(s1)) if build_first else (e(s1), e(s0))
    R = float(np.linalg.norm(b.shell_xyz[s0] - b.shell_xyz[s1]))
    a, c = x0[:, None], x1[None, :]
    z = a + c
    sig = 1.0 / np.sqrt(z)
    return float((((sig + c / z * R + R) / (sig + a / z * R)) ** l_moved).max())


def compact_batch(picks):
    """One ShellBatch (spherical) holding only the shells of the given
    (batch, quartet index) picks, four fresh shells per quartet."""
    ls, ks, xyz, ex, co = [], [], [], [], []
    for b, q in picks:
        for s in b.quartets[q]:
            ls.append(b.shell_l[s])
            ks.append(b.shell_k[s])
            xyz.append(b.shell_xyz[s])
            ex.append(b.prim_exp[b.shell_ptr[s]:b.shell_ptr[s] + b.shell_k[s]])
            co.append(b.prim_coef[b.shell_ptr[s]:b.shell_ptr[s] + b.shell_k[s]])
    ls, ks = np.array(ls, np.int32), np.array(ks, np.int32)
    ptr = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int32)
    quart = np.arange(len(ls), dtype=np.int32).reshape(-1, 4)
    off, size = basis.packed_offsets(ls, quart, True)
    return basis.ShellBatch(ls, ks, ptr, np.array(xyz), np.concatenate(ex), np.concatenate(co), quart, off, True,
                            size)


def mixed():
    """mixed_contraction_sph.npz: quartets of the l <= 4, K <= 8 workload
    (exponents log-uniform in [0.02, 1e5], centres in a 10-bohr cube) with a
    pair whose HRR growth bound exceeds 1e6 in both shell orders -- their
    contractions mix tight and diffuse exponents on both shells -- plus the
    (fg|gg) quartet 13409 of the 50000-quartet draw with seed 4.  out holds
    exact values (the C restatement in binary128, oracle_batch_quad); ref_out
    the reference's emitted C99 on the same quartets, whose own double
    recurrences lose digits on some of them."""
    T = basis.sph_matrices(6)
    b = basis.independent_quartet_batch(4, 20000, [0, 1, 2, 3, 4], [1, 2, 3, 4, 5, 6, 7, 8], 0.02, 1.0e5, 10.0, True)
    bnd = loader.quartet_bounds(b)
    pick, total = [], 0
    for q in range(b.nq):
        if bnd[q] < 1e-12:
            continue
        s = b.quartets[q]
        l = b.shell_l[s]
        if np.prod(b.shell_k[s]) > 1500:  # keeps the binary128 evaluation to seconds per quartet
            continue
        hard = False
        for i in (0, 2):
            if min(l[i], l[i + 1]) == 0:
                continue
            k0 = pair_kappa(b, s[i], s[i + 1], l[i + 1], True)
            k1 = pair_kappa(b, s[i], s[i + 1], l[i], False)
            hard = hard or min(k0, k1) > 1e6
        n = int(np.prod(2 * l + 1))
        if hard and total + n <= 60000:
            pick.append(q)
            total += n
        if len(pick) == 40:
            break
    big = basis.independent_quartet_batch(4, 50000, [0, 1, 2, 3, 4], [1, 2, 3, 4, 5, 6, 7, 8], 0.02, 1.0e5, 10.0,
                                          True)
    mb = compact_batch([(b, q) for q in pick] + [(big, 13409)])
    from multiprocessing import Pool
    with Pool(os.cpu_count() or 1) as p:
        parts = p.map(_quad_one, [(mb, q, T) for q in range(mb.nq)], chunksize=1)
    exact = np.concatenate(parts)
    save_batch('mixed_contraction_sph', mb, T, exact, ref_out=ref(mb, T))


def _quad_one(args):
    b, q, T = args
    return loader.oracle_batch_quad(b.subset(np.array([q])), T)


def generic_split():
    """generic_split_sph.npz: l 3..4 quartets (exponents log-uniform in
    [0.1, 1e3], centres in a 3-bohr cube), 16 with K = 5 on every shell (625
    primitive quartets each: the generic kernel splits those of its classes
    over a cluster) and 16 with K drawn from 1, 2, 5 (light and heavy mixed).
    out holds exact values (the C restatement in binary128)."""
    T = basis.sph_matrices(6)
    heavy = basis.independent_quartet_batch(11, 16, [3, 4], [5], 0.1, 1.0e3, 3.0, True)
    mixed_k = basis.independent_quartet_batch(11, 16, [3, 4], [1, 2, 5], 0.1, 1.0e3, 3.0, True)
    mb = compact_batch([(heavy, q) for q in range(heavy.nq)] + [(mixed_k, q) for q in range(mixed_k.nq)])
    from multiprocessing import Pool
    with Pool(os.cpu_count() or 1) as p:
        parts = p.map(_quad_one, [(mb, q, T) for q in range(mb.nq)], chunksize=1)
    save_batch('generic_split_sph', mb, T, np.concatenate(parts))


if __name__ == '__main__':
    if sys.argv[1:] == ['twoidx']:
        twoidx()
    elif sys.argv[1:] == ['c1']:
        c1()
    elif sys.argv[1:] == ['mixed']:
        mixed()
    elif sys.argv[1:] == ['generic_split']:
        generic_split()
    else:
        main()
        twoidx()
        c1()
        mixed()
        generic_split()
