"""Generator back end 'cuda': keep the input-script API, emit CUDA-backed files.

An input script builds its integral classes with the reference's DSL and calls
``generator(...).out()``, which writes C99 (``generator.py:1352-1502``): per
class ``<full_name>.c/.h``, plus ``global_data``, ``boys_function`` and
``global_functions`` files, into ``generator_options(output_directory=...)``.

With this module installed (``install(generator)``, once, with the
reference's generator class), ``gen.out(backend='cuda')`` writes into the same
directory, under the same names, the files a Makefile-flow user links instead:

* ``<header_filename>`` -- the class's prototypes (the emitted argument lists of
  ``contracted_general.py:42-68`` / ``primitive_general.py:31-97``), now
  implemented by libintception_b200.so;
* ``<full_name>_cuda.c`` -- only when the class's name differs from the
  library's: a forwarding shim from the class's symbols to the library's;
* ``boys_function.h`` -- ``intception_boys``, implemented by the library;
* ``intception_cuda.mk`` -- include and link flags for the library.

Supported classes, recognised by shape and then verified numerically:

* four-index electron-repulsion integrals (four Cartesian-Gaussian indices,
  one auxiliary index, a Boys function in the base), contracted, Cartesian or
  spherical;
* the example script's two-index overlap (two indices, no auxiliary index, no
  Boys function) and nuclear attraction (two indices, one auxiliary index, one
  position argument, a Boys function), primitive Cartesian
  (``examples/example_input.py:83-107``).

Verification (``verify=True``, the default): the reference back end writes the
class's own C99 into a temporary directory, the C compiler builds it, and the
class is run on fixed probe inputs; the checksums must match those of the
known integral (``fingerprints.json``, recorded from the reference's emitted
code).  A class of the right shape but different algebra therefore raises
``UnsupportedClass`` instead of being replaced by a different integral.
Anything else raises ``UnsupportedClass`` too (pass ``fallback=True`` to have
the reference back end write C99 for the whole generator instead).
"""
import contextlib
import ctypes as C
import io
import json
import math
import os
import shutil
import subprocess
import tempfile

PKG = os.path.dirname(os.path.abspath(__file__))
FINGERPRINTS = os.path.join(PKG, 'fingerprints.json')
ROOT = os.path.dirname(PKG)
LIB_NAME = 'intception_b200'


class UnsupportedClass(ValueError):
    pass


_PER_INDEX = ('const double * x{i}, const double c{I}[3], const int l{i}, const int n{i}, const int iskip{i}, '
              'const int n{i}_prim, const int n{i}_cont, const int iskip{i}_cont, const double * contract_array_{i}')
_SPH = ', const double * sph_trans_array_{i}'
_WSIZE = ('const int la, const int lb, const int lc, const int ld, const int na_prim, const int nb_prim, '
          'const int nc_prim, const int nd_prim, const int na_cont, const int nb_cont, const int nc_cont, '
          'const int nd_cont')


def _main_args(spherical, names=('a', 'b', 'c', 'd')):
    parts = []
    for i in names:
        p = _PER_INDEX.format(i=i, I=i.upper())
        if spherical:
            p += _SPH.format(i=i)
        parts.append(p)
    return ', '.join(parts) + ', double * work_array, double * output_array'


def _call_args(spherical, names=('a', 'b', 'c', 'd')):
    parts = []
    for i in names:
        p = ('x{i}, c{I}, l{i}, n{i}, iskip{i}, n{i}_prim, n{i}_cont, iskip{i}_cont, contract_array_{i}'
             .format(i=i, I=i.upper()))
        if spherical:
            p += ', sph_trans_array_{i}'.format(i=i)
        parts.append(p)
    return ', '.join(parts) + ', work_array, output_array'


_PAIR_ARGS = ('const double xa, const double cA[3], const int la, const int na, const int iskipa, '
              'const double xb, const double cB[3], const int lb, const int nb, const int iskipb')
_PAIR_CALL = 'xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb'

# mode -> the library's implementation of that class
LIBRARY_CLASS = {
    'eri_cont_cart': 'intception_integral_eri_abcd_m_cont_cart',
    'eri_cont_sph': 'intception_integral_eri_abcd_m_cont_sph',
    'overlap_2idx_prim_cart': 'intception_integral_overlap_2idx_ab_prim_cart',
    'nuclear_2idx_prim_cart': 'intception_integral_nuclear_2idx_ab_m_cC_prim_cart',
}


def _has_boys(base):
    seen, stack = set(), [base]
    while stack:
        node = stack.pop()
        if id(node) in seen or node is None:
            continue
        seen.add(id(node))
        if type(node).__name__ == 'boys_f':
            return True
        for attr in ('_left', '_right', '_arg', '_expr'):
            child = getattr(node, attr, None)
            if child is not None and hasattr(child, '__dict__'):
                stack.append(child)
    return False


def _shape(integral):
    """'eri', 'overlap_2idx', 'nuclear_2idx' or None, from the class's indices,
    auxiliary indices, arguments and whether its base holds a Boys function."""
    idx, aux, args = integral.index_list(), integral.aux_list(), integral.arg_list()
    if not all(type(i).__name__ == 'dsl_cartesian_gaussian' for i in idx):
        return None
    boys = _has_boys(integral.base())
    if len(idx) == 4 and len(aux) == 1 and not args and boys:
        return 'eri'
    if (len(idx) == 2 and len(aux) == 1 and len(args) == 1 and boys
            and type(args[0]).__name__ == 'dsl_position'):
        return 'nuclear_2idx'
    if len(idx) == 2 and not aux and not args and not boys:
        return 'overlap_2idx'
    return None


def _mode(shape, contracted, spherical):
    mode = '%s_%s_%s' % (shape, 'cont' if contracted else 'prim', 'sph' if spherical else 'cart')
    return mode if mode in LIBRARY_CLASS else None


# ---------------------------------------------------------------- probes
def _ncart(l):
    return (l + 1) * (l + 2) // 2


_ERI_PROBES = [(0, 0, 0, 0), (1, 0, 1, 0), (1, 1, 1, 1), (2, 1, 2, 0), (2, 2, 1, 1)]
_PAIR_PROBES = [(0, 0), (1, 0), (0, 2), (1, 1), (2, 1), (3, 2)]
_dp = C.POINTER(C.c_double)


def _checksum(out):
    return math.fsum(v * (1.0 + k / 7.0) for k, v in enumerate(out))


def _arr(vals):
    return (C.c_double * max(1, len(vals)))(*vals)


def _eri_probe(lib, full, spherical, ls, keep):
    """One contracted quartet through <full>_main; returns the output list."""
    main = getattr(lib, full + '_main')
    wsize = getattr(lib, full + '_work_array_size')
    wsize.restype = C.c_int
    wsize.argtypes = [C.c_int] * 12
    main.restype = None
    nprim = [2, 2, 1, 2]
    ncont = [1, 2 if ls == (1, 1, 1, 1) else 1, 1, 1]
    n = [2 * l + 1 if spherical else _ncart(l) for l in ls]
    st = [1, n[0], n[0] * n[1], n[0] * n[1] * n[2]]
    blk = st[3] * n[3]
    cst = [blk, blk * ncont[0], blk * ncont[0] * ncont[1], blk * ncont[0] * ncont[1] * ncont[2]]
    size = cst[3] * ncont[3]
    args, types = [], []
    for i, l in enumerate(ls):
        x = _arr([0.45 * (2.9 ** k) * (1.0 + 0.13 * i) for k in range(nprim[i])])
        cen = _arr([0.1 * i, 0.35 - 0.2 * i, 0.05 * i * i - 0.2])
        coef = _arr([0.4 + 0.25 * k + 0.1 * c + 0.05 * i for c in range(ncont[i]) for k in range(nprim[i])])
        keep += [x, cen, coef]
        args += [x, cen, l, n[i], st[i], nprim[i], ncont[i], cst[i], coef]
        types += [_dp, _dp] + [C.c_int] * 6 + [_dp]
        if spherical:
            nc = _ncart(l)
            T = _arr([math.cos(0.9 * r + 0.4 * c + 0.3 * l) for c in range(2 * l + 1) for r in range(nc)])
            keep.append(T)
            args.append(T)
            types.append(_dp)
    work = _arr([0.0] * (wsize(*ls, *nprim, *ncont) + 16))
    out = _arr([0.0] * size)
    keep += [work, out]
    main.argtypes = types + [_dp, _dp]
    main(*args, work, out)
    return list(out)


def _pair_probe(lib, full, nuclear, la, lb, keep):
    main = getattr(lib, full + '_main')
    wsize = getattr(lib, full + '_work_array_size')
    wsize.restype = C.c_int
    wsize.argtypes = [C.c_int, C.c_int]
    main.restype = None
    na, nb = _ncart(la), _ncart(lb)
    A, B, Cc = _arr([0.1, -0.2, 0.3]), _arr([-0.3, 0.25, 0.05]), _arr([0.4, 0.1, -0.35])
    work = _arr([0.0] * (wsize(la, lb) + 16))
    out = _arr([0.0] * (na * nb))
    keep += [A, B, Cc, work, out]
    types = [C.c_double, _dp, C.c_int, C.c_int, C.c_int] * 2
    if nuclear:
        main.argtypes = types + [_dp, _dp, _dp]
        main(0.9, A, la, na, 1, 1.7, B, lb, nb, na, Cc, work, out)
    else:
        main.argtypes = types + [_dp, _dp]
        main(0.9, A, la, na, 1, 1.7, B, lb, nb, na, work, out)
    return list(out)


def probe_checksums(lib, mode, full):
    """Checksums of the class <full> (symbols <full>_main and
    <full>_work_array_size in the loaded library lib) on the fixed probes of
    mode."""
    keep = []
    if mode.startswith('eri_'):
        return [_checksum(_eri_probe(lib, full, mode.endswith('_sph'), ls, keep)) for ls in _ERI_PROBES]
    nuclear = mode.startswith('nuclear_')
    return [_checksum(_pair_probe(lib, full, nuclear, la, lb, keep)) for la, lb in _PAIR_PROBES]


def _c99_out(gen):
    out = type(gen).out
    return getattr(out, '_intception_b200_c99', out)


def _verify(gen, classes):
    """Write the reference back end's C99 for gen into a temporary directory,
    compile it, and compare each class's probe checksums with the recorded
    ones.  Raises UnsupportedClass on any mismatch or build failure."""
    with open(FINGERPRINTS) as fh:
        want_all = json.load(fh)
    tmp = tempfile.mkdtemp(prefix='intception_b200_verify_')
    try:
        opt = gen.generator_options()
        saved = opt._output_directory
        opt._output_directory = tmp
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                _c99_out(gen)(gen)
        finally:
            opt._output_directory = saved
        unity = os.path.join(tmp, '_verify_unity.c')
        with open(unity, 'w') as fh:
            fh.write('#include <math.h>\n')
            for f in sorted(os.listdir(tmp)):
                if f.endswith('.c') and f != '_verify_unity.c':
                    fh.write('#include "%s"\n' % f)
        so = os.path.join(tmp, '_verify.so')
        cc = os.environ.get('CC', 'gcc')
        r = subprocess.run([cc, '-std=gnu99', '-O1', '-fPIC', '-shared', '-w', '-I', tmp, unity, '-o', so, '-lm'],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise UnsupportedClass('cannot build the C99 of the classes to verify them (%s): %s'
                                   % (cc, r.stderr.strip()[-400:]))
        lib = C.CDLL(so)
        for wi, mode in classes:
            got = probe_checksums(lib, mode, wi.full_name())
            want = want_all[mode]
            for g, w in zip(got, want):
                if not abs(g - w) <= 1e-9 * max(1.0, abs(w)):
                    raise UnsupportedClass('class %s has the shape of %s but not its values (probe checksum %r, '
                                           'expected %r)' % (wi.full_name(), mode, g, w))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# ---------------------------------------------------------------- files
def _write_header(path, full, mode, guard):
    with open(path, 'w') as fh:
        fh.write('/* %s: implemented by lib%s.so (sm_100a); written by the cuda back end. */\n' % (full, LIB_NAME))
        fh.write('#ifndef %s\n#define %s\n#ifdef __cplusplus\nextern "C" {\n#endif\n' % (guard, guard))
        if mode.startswith('eri_'):
            sph = mode.endswith('_sph')
            fh.write('void %s_main( %s );\n' % (full, _main_args(sph)))
            fh.write('int %s_work_array_size( %s );\n' % (full, _WSIZE))
        else:
            extra = ', const double cC[3]' if mode.startswith('nuclear_') else ''
            fh.write('void %s_main( %s%s, double * work_array, double * output_array );\n'
                     % (full, _PAIR_ARGS, extra))
            fh.write('int %s_work_array_size( const int la, const int lb );\n' % full)
        fh.write('int intception_b200_last_status(void);\nconst char *intception_b200_last_error(void);\n')
        fh.write('#ifdef __cplusplus\n}\n#endif\n#endif\n')


def _write_shim(path, header, full, ours, mode):
    with open(path, 'w') as fh:
        fh.write('/* Forwards %s to the library implementation %s. */\n' % (full, ours))
        fh.write('#include "%s"\n' % header)
        if mode.startswith('eri_'):
            sph = mode.endswith('_sph')
            fh.write('void %s_main( %s );\n' % (ours, _main_args(sph)))
            fh.write('int %s_work_array_size( %s );\n' % (ours, _WSIZE))
            fh.write('void %s_main( %s ) {\n  %s_main( %s );\n}\n' % (full, _main_args(sph), ours, _call_args(sph)))
            fh.write('int %s_work_array_size( %s ) {\n  return %s_work_array_size( la, lb, lc, ld, na_prim, '
                     'nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont );\n}\n' % (full, _WSIZE, ours))
        else:
            nuc = mode.startswith('nuclear_')
            args = _PAIR_ARGS + (', const double cC[3]' if nuc else '') + ', double * work_array, double * output_array'
            call = _PAIR_CALL + (', cC' if nuc else '') + ', work_array, output_array'
            fh.write('void %s_main( %s );\n' % (ours, args))
            fh.write('int %s_work_array_size( const int la, const int lb );\n' % ours)
            fh.write('void %s_main( %s ) {\n  %s_main( %s );\n}\n' % (full, args, ours, call))
            fh.write('int %s_work_array_size( const int la, const int lb ) {\n  return %s_work_array_size( la, lb );'
                     '\n}\n' % (full, ours))


def cuda_out(gen, fallback=False, verify=True):
    """Write the CUDA-backed files for every class of ``gen`` (a reference
    ``generator``).  Returns the list of written paths."""
    opt = gen.generator_options()
    outdir = opt.output_directory()
    contracted = bool(opt.contracted())
    spherical = bool(opt.spherical_transformed())
    classes = []
    for wi in gen._wi_list:
        shape = _shape(wi.integral())
        mode = _mode(shape, contracted, spherical) if shape else None
        if mode is None:
            if fallback:
                _c99_out(gen)(gen)
                return []
            if shape is None:
                raise UnsupportedClass('class %s is not a supported integral class' % wi.full_name())
            raise UnsupportedClass('class %s: the CUDA back end implements %s only as %s' % (
                wi.full_name(), shape, 'contracted' if shape == 'eri' else 'primitive Cartesian'))
        classes.append((wi, mode))
    if verify:
        try:
            _verify(gen, classes)
        except UnsupportedClass:
            if fallback:
                _c99_out(gen)(gen)
                return []
            raise
    written = []
    os.makedirs(outdir, exist_ok=True)
    for wi, mode in classes:
        full, ours = wi.full_name(), LIBRARY_CLASS[mode]
        hdr = os.path.join(outdir, wi.header_filename())
        guard = ''.join(ch if ch.isalnum() else '_' for ch in wi.header_filename()).upper()
        _write_header(hdr, full, mode, guard)
        written.append(hdr)
        if full != ours:
            shim = os.path.join(outdir, full + '_cuda.c')
            _write_shim(shim, wi.header_filename(), full, ours, mode)
            written.append(shim)
    boys = os.path.join(outdir, 'boys_function.h')
    with open(boys, 'w') as fh:
        fh.write('/* intception_boys: implemented by lib%s.so. */\n' % LIB_NAME)
        fh.write('#ifndef INTCEPTION_BOYS_FUNCTION_H\n#define INTCEPTION_BOYS_FUNCTION_H\n')
        fh.write('void intception_boys( double * f, const int ifskip, const int nmin, const int nmax, '
                 'const double x );\n#endif\n')
    written.append(boys)
    mk = os.path.join(outdir, 'intception_cuda.mk')
    with open(mk, 'w') as fh:
        fh.write('# Include from a Makefile that builds against the CUDA back end.\n')
        fh.write('INTCEPTION_B200_DIR ?= %s\n' % ROOT)
        fh.write('INTCEPTION_CFLAGS += -I$(INTCEPTION_B200_DIR)/include\n')
        fh.write('INTCEPTION_LDFLAGS += -L$(INTCEPTION_B200_DIR)/intception_b200 -l%s '
                 '-Wl,-rpath,$(INTCEPTION_B200_DIR)/intception_b200\n' % LIB_NAME)
        shims = ' '.join(os.path.basename(p) for p in written if p.endswith('_cuda.c'))
        fh.write('INTCEPTION_CUDA_SOURCES = %s\n' % shims)
    written.append(mk)
    return written


def install(generator_cls):
    """Give the reference's generator class an ``out(backend=...)`` keyword:
    backend='c99' (default) keeps the reference behaviour, 'cuda' calls
    cuda_out."""
    if getattr(generator_cls.out, '_intception_b200', False):
        return
    original = generator_cls.out

    def out(self, use_stdout=False, backend='c99'):
        if backend == 'cuda':
            return cuda_out(self)
        if backend != 'c99':
            raise ValueError('backend must be "c99" or "cuda"')
        return original(self, use_stdout)

    out._intception_b200 = True
    out._intception_b200_c99 = original
    generator_cls.out = out
