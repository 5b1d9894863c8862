"""Shell data model, normalisation and Cartesian->spherical matrices.

Conventions (the ones the reference's emitted code and its DSL fix):

* Cartesian components of one shell are ordered x-descending, then
  y-descending (``dsl.py:988-1001``): l=2 -> xx, xy, xz, yy, yz, zz.  The index
  inside a level is ``mz + (my+mz)(my+mz+1)/2`` (``dsl.py:1029-1041``).
* Contraction coefficients already include primitive normalisation: the
  reference never normalises (``contracted_general.py:42-68`` passes
  ``contract_array_?[iprim + icont*n_prim]`` straight into the contraction).
  ``normalize_shell`` produces such coefficients from raw ones, normalising every
  Cartesian component with the norm of the axis-aligned x^l function.
* A spherical matrix is stored ``T[icart + isph*ncart]`` (column-major
  ncart x nsph), the layout of ``sph_trans_array_?``
  (``generator_sph_trans_function.py:69-125``).  ``sph_matrix(l)`` returns real
  solid harmonics ordered m = -l..l, each scaled to the norm of x^l.

Batch layout (segmented shells, n_cont = 1): quartet q writes its block at
``out[out_off[q]:]`` with a fastest, ``ia + na*(ib + nb*(ic + nc*id))``.
"""
from dataclasses import dataclass
from math import comb, factorial, sqrt, pi

import numpy as np

LMAX = 6  # generator_options(global_user_lmax) default, generator.py:206


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nsph(l):
    return 2 * l + 1


def cart_components(l):
    """[(mx, my, mz), ...] in the reference's order for one level l."""
    out = []
    for mx in range(l, -1, -1):
        for my in range(l - mx, -1, -1):
            out.append((mx, my, l - mx - my))
    return out


def cart_index(mx, my, mz):
    """Index of (mx,my,mz) inside its level (``dsl.py:1029-1041`` minus the offset)."""
    return mz + (my + mz) * (my + mz + 1) // 2


def _dfact(n):
    """(n)!! with (-1)!! = 0!! = 1."""
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def prim_norm(alpha, l):
    """Norm of x^l exp(-alpha r^2)."""
    alpha = np.asarray(alpha, dtype=np.float64)
    return (2.0 * alpha / pi) ** 0.75 * (4.0 * alpha) ** (l / 2.0) / sqrt(_dfact(2 * l - 1))


def normalize_shell(l, exps, coefs):
    """Return coefficients with primitive norms folded in and the contracted
    x^l function renormalised to 1."""
    exps = np.asarray(exps, dtype=np.float64)
    c = np.asarray(coefs, dtype=np.float64)
    a = exps[:, None] + exps[None, :]
    ov = (2.0 * np.sqrt(exps[:, None] * exps[None, :]) / a) ** (l + 1.5)
    s = float(c @ ov @ c)
    return c / sqrt(s) * prim_norm(exps, l)


def _solid_harmonic_monomials(l, m):
    """Real regular solid harmonic S_lm as {(i,j,k): coefficient} (unnormalised)."""
    am = abs(m)
    vm = 0.5 if m < 0 else 0.0
    out = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            v = vm
            while v <= (am / 2.0 - vm) // 1 + vm + 1e-9:
                two_v = int(round(2 * v))
                c = ((-1) ** int(round(t + v - vm)) * (0.25 ** t) * comb(l, t) * comb(l - t, am + t)
                     * comb(t, u) * comb(am, two_v))
                i = 2 * t + am - 2 * u - two_v
                j = 2 * u + two_v
                k = l - 2 * t - am
                if c != 0:
                    out[(i, j, k)] = out.get((i, j, k), 0.0) + c
                v += 1.0
    return out


def sph_matrix(l):
    """ncart x nsph matrix T (Fortran order, ``T[icart + isph*ncart]``), m = -l..l."""
    comps = cart_components(l)
    idx = {c: n for n, c in enumerate(comps)}
    nc = len(comps)
    T = np.zeros((nc, 2 * l + 1))
    # overlap of monomials with a common Gaussian, up to a factor depending only on l
    S = np.zeros((nc, nc))
    for p, (i1, j1, k1) in enumerate(comps):
        for q, (i2, j2, k2) in enumerate(comps):
            n = (i1 + i2, j1 + j2, k1 + k2)
            if all(x % 2 == 0 for x in n):
                S[p, q] = _dfact(n[0] - 1) * _dfact(n[1] - 1) * _dfact(n[2] - 1)
    for col, m in enumerate(range(-l, l + 1)):
        for mono, c in _solid_harmonic_monomials(l, m).items():
            T[idx[mono], col] += c
        nrm = T[:, col] @ S @ T[:, col]
        T[:, col] *= sqrt(_dfact(2 * l - 1) / nrm)
    return T


_SPH_CACHE = {}


def sph_matrices(lmax=LMAX):
    """List of Fortran-ordered T matrices for l = 0..lmax (cached)."""
    if lmax not in _SPH_CACHE:
        _SPH_CACHE[lmax] = [np.asfortranarray(sph_matrix(l)) for l in range(lmax + 1)]
    return _SPH_CACHE[lmax]


@dataclass
class ShellBatch:
    """A shell table plus a list of shell quartets (segmented contraction).

    shell_l, shell_k, shell_ptr : int32 [nshell]
    shell_xyz                   : float64 [nshell, 3]
    prim_exp, prim_coef         : float64 [nprim] (coefficients normalised)
    quartets                    : int32 [nq, 4] shell indices (a, b, c, d)
    out_off                     : int64 [nq] block offsets into the output
    spherical                   : output 2l+1 (True) or Cartesian components
    """
    shell_l: np.ndarray
    shell_k: np.ndarray
    shell_ptr: np.ndarray
    shell_xyz: np.ndarray
    prim_exp: np.ndarray
    prim_coef: np.ndarray
    quartets: np.ndarray
    out_off: np.ndarray
    spherical: bool
    out_size: int = 0

    @property
    def nq(self):
        return int(self.quartets.shape[0])

    @property
    def nshell(self):
        return int(self.shell_l.shape[0])

    def block_dims(self, q):
        ls = self.shell_l[self.quartets[q]]
        return tuple((2 * l + 1) if self.spherical else ncart(l) for l in ls)

    def subset(self, idx):
        """Batch with the quartets idx (shell table shared), outputs packed."""
        idx = np.asarray(idx)
        qs = np.ascontiguousarray(self.quartets[idx])
        off, total = packed_offsets(self.shell_l, qs, self.spherical)
        return ShellBatch(self.shell_l, self.shell_k, self.shell_ptr, self.shell_xyz, self.prim_exp,
                          self.prim_coef, qs, off, self.spherical, total)


def block_sizes(shell_l, quartets, spherical):
    ls = shell_l[quartets]
    n = (2 * ls + 1) if spherical else (ls + 1) * (ls + 2) // 2
    return np.prod(n.astype(np.int64), axis=1)


def packed_offsets(shell_l, quartets, spherical):
    sz = block_sizes(shell_l, quartets, spherical)
    off = np.zeros(len(sz), dtype=np.int64)
    if len(sz):
        off[1:] = np.cumsum(sz)[:-1]
    return off, int(sz.sum())


def make_shells(rng, ls, ks, alpha_lo, alpha_hi, box, coef_lo=0.1, coef_hi=1.0, centres=None):
    """Random shells: exponents log-uniform in [alpha_lo, alpha_hi], raw
    coefficients uniform in [coef_lo, coef_hi] then normalised, centres uniform
    in [0, box]^3 unless given."""
    ls = np.asarray(ls, dtype=np.int32)
    ks = np.asarray(ks, dtype=np.int32)
    n = len(ls)
    ptr = np.zeros(n, dtype=np.int32)
    if n:
        ptr[1:] = np.cumsum(ks)[:-1]
    nprim = int(ks.sum())
    exps = np.exp(rng.uniform(np.log(alpha_lo), np.log(alpha_hi), nprim))
    raw = rng.uniform(coef_lo, coef_hi, nprim)
    coefs = np.empty(nprim)
    # vectorised normalisation, grouped by (l, K)
    for l in np.unique(ls):
        for k in np.unique(ks[ls == l]):
            sel = np.nonzero((ls == l) & (ks == k))[0]
            if len(sel) == 0:
                continue
            pidx = ptr[sel][:, None] + np.arange(k)[None, :]
            e = exps[pidx]
            c = raw[pidx]
            a = e[:, :, None] + e[:, None, :]
            ov = (2.0 * np.sqrt(e[:, :, None] * e[:, None, :]) / a) ** (l + 1.5)
            s = np.einsum('si,sij,sj->s', c, ov, c)
            coefs[pidx] = c / np.sqrt(s)[:, None] * prim_norm(e, int(l))
    if centres is None:
        centres = rng.uniform(0.0, box, (n, 3))
    return ls, ks, ptr, np.ascontiguousarray(centres, dtype=np.float64), exps, coefs


def independent_quartet_batch(seed, nq, lchoices, kchoices, alpha_lo, alpha_hi, box, spherical,
                              fixed_l=None, fixed_k=None):
    """nq quartets, each over four fresh shells (no shell reuse): l drawn
    uniformly from lchoices and K from kchoices per shell unless fixed."""
    rng = np.random.default_rng(seed)
    ns = 4 * nq
    ls = np.full(ns, fixed_l, np.int32) if fixed_l is not None else \
        rng.choice(np.asarray(lchoices, np.int32), ns)
    ks = np.full(ns, fixed_k, np.int32) if fixed_k is not None else \
        rng.choice(np.asarray(kchoices, np.int32), ns)
    l, k, ptr, xyz, e, c = make_shells(rng, ls, ks, alpha_lo, alpha_hi, box)
    quartets = np.arange(ns, dtype=np.int32).reshape(nq, 4)
    off, total = packed_offsets(l, quartets, spherical)
    return ShellBatch(l, k, ptr, xyz, e, c, quartets, off, spherical, total)


def config_pppp_k3(nq=4096, seed=0):
    """(pp|pp), K=3 per shell, exponents log-uniform [0.1,100], coefficients
    uniform [0.1,1] then normalised, centres uniform in a 10-bohr cube, Cartesian."""
    return independent_quartet_batch(seed, nq, None, None, 0.1, 100.0, 10.0, False, fixed_l=1, fixed_k=3)


def config_mixed_l2(nq=1_000_000, seed=1, spherical=True):
    """l in {0,1,2} per shell (class uniform over the 81 classes), K uniform in
    {1..6}, exponents log-uniform [0.05,1e4], centres in a 30-bohr cube,
    spherical output."""
    return independent_quartet_batch(seed, nq, [0, 1, 2], [1, 2, 3, 4, 5, 6], 0.05, 1.0e4, 30.0,
                                     spherical)


def lattice_shells(natom=200, seed=2, spacing=2.6, jitter=0.3,
                   shells=((0, 6), (0, 3), (1, 3), (2, 1), (3, 1)), alpha=(0.1, 1e3)):
    """Jittered cubic lattice: the first natom sites (row-major) of the smallest
    cube holding them, spacing bohr apart, each moved by a uniform +-jitter;
    per atom the given (l, K) shells, exponents log-uniform in alpha,
    coefficients uniform [0.1, 1] then normalised.  Returns (rng, shell_l,
    shell_k, shell_ptr, shell_xyz, prim_exp, prim_coef); rng continues the
    seeded stream for sampling."""
    rng = np.random.default_rng(seed)
    n = int(np.ceil(natom ** (1.0 / 3.0) - 1e-9))
    sites = np.array([(i, j, k) for i in range(n) for j in range(n) for k in range(n)][:natom], np.float64)
    xyz = sites * spacing + rng.uniform(-jitter, jitter, (natom, 3))
    ls = np.array([l for _ in range(natom) for (l, _) in shells], np.int32)
    ks = np.array([k for _ in range(natom) for (_, k) in shells], np.int32)
    centres = np.repeat(xyz, len(shells), axis=0)
    return (rng,) + make_shells(rng, ls, ks, alpha[0], alpha[1], 1.0, centres=centres)


def sample_screened_quartets(q, pairs, nq, rng, threshold=1e-12):
    """Uniform sample of nq of the unique quartets (pair i, pair j), j <= i in
    the order of decreasing Schwarz factor q, whose bound q_i q_j reaches the
    threshold.  q: per pair factor, pairs: [npair, 2] shell indices.  Returns
    (quartets [n, 4] int32, number of such quartets)."""
    order = np.argsort(-q, kind='stable')
    qs, pr = q[order], pairs[order]
    # row i pairs with the rows j <= i whose q_j >= threshold / q_i (a prefix: q sorted)
    cnt = np.searchsorted(-qs, -(threshold / np.maximum(qs, 1e-300)), side='right')
    m = np.minimum(cnt, np.arange(1, len(qs) + 1))
    cm = np.cumsum(m)
    total = int(cm[-1]) if len(cm) else 0
    pos = np.sort(rng.choice(total, size=min(nq, total), replace=False))
    row = np.searchsorted(cm, pos, side='right')
    col = pos - (cm[row] - m[row])
    quartets = np.concatenate([pr[row], pr[col]], axis=1).astype(np.int32)
    return np.ascontiguousarray(quartets), total

