"""ctypes access to the CPU oracle and to the reference-emitted C99.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg.  The product (intception_b200) never imports this module.

* ``liberi_oracle.so`` (built from oracle/eri_oracle.c by oracle/Makefile) is the
  C restatement of the reference's path.  It is built on demand with gcc.
* ``_ref/libref_eri_{cart,sph}.so`` (built by oracle/gen_ref.py where the
  reference tree exists) is the reference generator's own emitted C99 plus an
  OpenMP batch driver.  It may be absent; callers must handle ``None``.
* ``_ref/libref_2idx.so`` (also gen_ref.py) is the reference's emitted C99 of
  its example script's two-index classes (overlap, nuclear attraction).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, '_gen', 'liberi_oracle.so')
_REF_SO = {v: os.path.join(HERE, '_ref', 'libref_eri_%s.so' % v) for v in ('cart', 'sph')}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)

_oracle = None
_ref = {}


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(_ORACLE_SO):
            subprocess.run(['make', '-s', '-C', HERE], check=True)
        lib = C.CDLL(_ORACLE_SO)
        lib.oracle_boys.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double]
        lib.oracle_boys.restype = None
        lib.oracle_set_boys_exact.argtypes = [C.c_int]
        lib.oracle_set_boys_exact.restype = None
        lib.oracle_eri_work_array_size.argtypes = [C.c_int] * 12
        lib.oracle_eri_work_array_size.restype = C.c_int
        lib.oracle_eri_batch.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, C.POINTER(_dp), _lp, _dp]
        lib.oracle_eri_batch.restype = None
        lib.oracle_quartet_bounds.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, C.c_int, _dp]
        lib.oracle_quartet_bounds.restype = None
        idx = [C.c_int] * 6
        per_cart = [_dp, _dp] + idx + [_dp]
        per_sph = per_cart + [_dp]
        lib.oracle_eri_cont_cart_main.argtypes = per_cart * 4 + [_dp, _dp]
        lib.oracle_eri_cont_cart_main.restype = None
        lib.oracle_eri_cont_sph_main.argtypes = per_sph * 4 + [_dp, _dp]
        lib.oracle_eri_cont_sph_main.restype = None
        lib.oracle_2idx_batch.argtypes = [C.c_int, C.c_int, _dp, _dp, _ip, _dp, _dp, _ip, _dp, _lp, _dp]
        lib.oracle_2idx_batch.restype = None
        lib.oracle_2idx_work_array_size.argtypes = [C.c_int] * 3
        lib.oracle_2idx_work_array_size.restype = C.c_int
        pair = [C.c_double, _dp, C.c_int, C.c_int, C.c_int] * 2
        lib.oracle_overlap_2idx_ab_prim_cart_main.argtypes = pair + [_dp, _dp]
        lib.oracle_overlap_2idx_ab_prim_cart_main.restype = None
        lib.oracle_nuclear_2idx_ab_m_cC_prim_cart_main.argtypes = pair + [_dp, _dp, _dp]
        lib.oracle_nuclear_2idx_ab_m_cC_prim_cart_main.restype = None
        _oracle = lib
    return _oracle


def load_ref(variant):
    """The reference-emitted C99 for 'cart' or 'sph', or None if not built."""
    if variant not in _ref:
        path = _REF_SO[variant]
        if not os.path.exists(path):
            _ref[variant] = None
        else:
            lib = C.CDLL(path)
            lib.ref_eri_batch.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, C.POINTER(_dp), _lp,
                                          _dp, C.c_int]
            lib.ref_eri_batch.restype = C.c_int
            lib.ref_eri_batch_screened.argtypes = lib.ref_eri_batch.argtypes + [C.c_double]
            lib.ref_eri_batch_screened.restype = C.c_int
            lib.ref_work_array_size.argtypes = [C.c_int] * 12
            lib.ref_work_array_size.restype = C.c_int
            main = getattr(lib, 'intception_integral_eri_abcd_m_cont_%s_main' % variant)
            idx = [C.c_int] * 6
            per = [_dp, _dp] + idx + [_dp] + ([_dp] if variant == 'sph' else [])
            main.argtypes = per * 4 + [_dp, _dp]
            main.restype = None
            lib.intception_boys.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double]
            lib.intception_boys.restype = None
            _ref[variant] = lib
    return _ref[variant]


_REF_2IDX_SO = os.path.join(HERE, '_ref', 'libref_2idx.so')
_ref2 = []


def load_ref_2idx():
    """The reference-emitted two-index classes (ref_2idx_batch), or None."""
    if not _ref2:
        if not os.path.exists(_REF_2IDX_SO):
            _ref2.append(None)
        else:
            lib = C.CDLL(_REF_2IDX_SO)
            lib.ref_2idx_batch.argtypes = [C.c_int, C.c_int, _dp, _dp, _ip, _dp, _dp, _ip, _dp, _lp, _dp]
            lib.ref_2idx_batch.restype = None
            lib.ref_2idx_work_array_size.argtypes = [C.c_int] * 3
            lib.ref_2idx_work_array_size.restype = C.c_int
            _ref2.append(lib)
    return _ref2[0]


def twoidx_batch(kind, pairs, lib=None):
    """Two-index primitive blocks of a pair set (dict with xa, ca, la, xb, cb,
    lb, cc, off, size; kind 0 overlap, 1 nuclear) with the C restatement, or
    with the reference's emitted C99 when lib is load_ref_2idx()."""
    lib = lib or load_oracle()
    fn = lib.oracle_2idx_batch if hasattr(lib, 'oracle_2idx_batch') else lib.ref_2idx_batch
    a = {k: np.ascontiguousarray(pairs[k], dtype=np.int32 if k in ('la', 'lb') else
                                 (np.int64 if k == 'off' else np.float64))
         for k in ('xa', 'ca', 'la', 'xb', 'cb', 'lb', 'cc', 'off')}
    out = np.zeros(int(pairs['size']))
    fn(int(kind), len(a['xa']), _ptr(a['xa']), _ptr(a['ca']), _ptr(a['la'], _ip), _ptr(a['xb']), _ptr(a['cb']),
       _ptr(a['lb'], _ip), _ptr(a['cc']), _ptr(a['off'], _lp), _ptr(out))
    return out


def boys(nmax, x, lib=None, exact=False):
    lib = lib or load_oracle()
    f = np.zeros(nmax + 1)
    if hasattr(lib, 'oracle_boys'):
        lib.oracle_set_boys_exact(1 if exact else 0)
        try:
            lib.oracle_boys(_ptr(f), 1, 0, nmax, float(x))
        finally:
            lib.oracle_set_boys_exact(0)
    else:
        lib.intception_boys(_ptr(f), 1, 0, nmax, float(x))
    return f


def _sph_table(sphT, lmax=6):
    keep = [np.ascontiguousarray(np.asarray(T, dtype=np.float64).ravel(order='F')) for T in sphT]
    arr = (_dp * len(keep))(*[_ptr(k) for k in keep])
    return arr, keep


def _batch_args(b):
    q = np.ascontiguousarray(b.quartets, dtype=np.int32)
    sl = np.ascontiguousarray(b.shell_l, dtype=np.int32)
    sk = np.ascontiguousarray(b.shell_k, dtype=np.int32)
    sp = np.ascontiguousarray(b.shell_ptr, dtype=np.int32)
    xyz = np.ascontiguousarray(b.shell_xyz, dtype=np.float64)
    e = np.ascontiguousarray(b.prim_exp, dtype=np.float64)
    c = np.ascontiguousarray(b.prim_coef, dtype=np.float64)
    off = np.ascontiguousarray(b.out_off, dtype=np.int64)
    return q, sl, sk, sp, xyz, e, c, off


def oracle_batch(b, sphT=None, exact_boys=False):
    """Evaluate a ShellBatch with the C restatement (single thread).
    exact_boys: an accurate Boys function in place of the reference's (see
    oracle_set_boys_exact in eri_oracle.c)."""
    lib = load_oracle()
    q, sl, sk, sp, xyz, e, c, off = _batch_args(b)
    out = np.zeros(b.out_size)
    tab, keep = _sph_table(sphT) if b.spherical else (None, None)
    lib.oracle_set_boys_exact(1 if exact_boys else 0)
    try:
        lib.oracle_eri_batch(b.nq, _ptr(q, _ip), _ptr(sl, _ip), _ptr(sk, _ip), _ptr(sp, _ip), _ptr(xyz),
                             _ptr(e), _ptr(c), tab, _ptr(off, _lp), _ptr(out))
    finally:
        lib.oracle_set_boys_exact(0)
    return out


_oracle_quad = None


def oracle_batch_quad(b, sphT=None):
    """Evaluate a ShellBatch with the C restatement computed in binary128
    (eri_oracle.c built with ORACLE_QUAD, accurate Boys function): exact to
    double precision even where double-precision recurrences cancel digits.
    Slow (software binary128): for a few quartets."""
    global _oracle_quad
    if _oracle_quad is None:
        so = os.path.join(os.path.dirname(_ORACLE_SO), 'liberi_oracle_quad.so')
        if not os.path.exists(so):
            subprocess.run(['make', '-s', '-C', HERE], check=True)
        lib = C.CDLL(so)
        lib.oracle_eri_batch.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, C.POINTER(_dp), _lp, _dp]
        lib.oracle_eri_batch.restype = None
        _oracle_quad = lib
    q, sl, sk, sp, xyz, e, c, off = _batch_args(b)
    out = np.zeros(b.out_size)
    tab, keep = _sph_table(sphT) if b.spherical else (None, None)
    _oracle_quad.oracle_eri_batch(b.nq, _ptr(q, _ip), _ptr(sl, _ip), _ptr(sk, _ip), _ptr(sp, _ip), _ptr(xyz),
                                  _ptr(e), _ptr(c), tab, _ptr(off, _lp), _ptr(out))
    return out


def quartet_bounds(b):
    """The library's analytic screening bound of every quartet (pair_bound.h),
    with the C restatement."""
    lib = load_oracle()
    q, sl, sk, sp, xyz, e, c, off = _batch_args(b)
    out = np.zeros(b.nq)
    lib.oracle_quartet_bounds(b.nq, _ptr(q, _ip), _ptr(sl, _ip), _ptr(sk, _ip), _ptr(sp, _ip), _ptr(xyz), _ptr(e),
                              _ptr(c), 1 if b.spherical else 0, _ptr(out))
    return out


def ref_batch_screened(b, sphT, skip_below, nthreads=0, out=None):
    """The reference-emitted C99 behind the library's analytic screening:
    quartets whose bound is below skip_below get zero blocks.  Returns (out,
    number evaluated), or (None, 0) when oracle/_ref was not built."""
    lib = load_ref('sph' if b.spherical else 'cart')
    if lib is None:
        return None, 0
    q, sl, sk, sp, xyz, e, c, off = _batch_args(b)
    if out is None:
        out = np.zeros(b.out_size)
    tab, keep = _sph_table(sphT) if b.spherical else (None, None)
    n = lib.ref_eri_batch_screened(b.nq, _ptr(q, _ip), _ptr(sl, _ip), _ptr(sk, _ip), _ptr(sp, _ip), _ptr(xyz),
                                   _ptr(e), _ptr(c), tab, _ptr(off, _lp), _ptr(out), int(nthreads),
                                   float(skip_below))
    return out, n


def ref_batch(b, sphT=None, nthreads=0, out=None):
    """Evaluate a ShellBatch with the reference-emitted C99 (OpenMP).  Returns
    None when oracle/_ref was not built."""
    lib = load_ref('sph' if b.spherical else 'cart')
    if lib is None:
        return None
    q, sl, sk, sp, xyz, e, c, off = _batch_args(b)
    if out is None:
        out = np.zeros(b.out_size)
    tab, keep = _sph_table(sphT) if b.spherical else (None, None)
    lib.ref_eri_batch(b.nq, _ptr(q, _ip), _ptr(sl, _ip), _ptr(sk, _ip), _ptr(sp, _ip), _ptr(xyz), _ptr(e),
                      _ptr(c), tab, _ptr(off, _lp), _ptr(out), int(nthreads))
    return out


def call_main(lib, variant, shells, work, out, prefix=None):
    """Call a per-quartet main (oracle or reference) with the emitted argument
    list.  shells: four dicts with keys x, cen, l, n, iskip, nprim, ncont,
    iskip_cont, coef and (sph) T."""
    fn = getattr(lib, prefix or ('intception_integral_eri_abcd_m_cont_%s_main' % variant))
    args = []
    keep = []
    for s in shells:
        x = np.ascontiguousarray(s['x'], dtype=np.float64)
        cen = np.ascontiguousarray(s['cen'], dtype=np.float64)
        coef = np.ascontiguousarray(s['coef'], dtype=np.float64)
        keep += [x, cen, coef]
        args += [_ptr(x), _ptr(cen), s['l'], s['n'], s['iskip'], s['nprim'], s['ncont'], s['iskip_cont'],
                 _ptr(coef)]
        if variant == 'sph':
            T = np.ascontiguousarray(np.asarray(s['T'], dtype=np.float64).ravel(order='F'))
            keep.append(T)
            args.append(_ptr(T))
    fn(*args, _ptr(work), _ptr(out))
    return out
