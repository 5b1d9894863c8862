"""Generator back end 'cuda': keep the input-script API, emit CUDA-backed files.

An input script builds its integral classes with the reference's DSL and calls
``generator(...).out()``, which writes C99 (``generator.py:1352-1502``): per
class ``<full_name>.c/.h``, plus ``global_data``, ``boys_function`` and
``global_functions`` files, into ``generator_options(output_directory=...)``.

With this module installed (``install(generator)``, once, with the
reference's generator class), ``gen.out(backend='cuda')`` writes into the same
directory, under the same names, the files a Makefile-flow user links instead:

* ``<header_filename>`` -- the class's prototypes (the emitted argument lists of
  ``contracted_general.py:42-68``), now implemented by libintception_b200.so;
* ``<full_name>_cuda.c`` -- only when the class is not named ``eri``: a
  forwarding shim from the class's symbols to the library's;
* ``boys_function.h`` -- ``intception_boys``, implemented by the library;
* ``intception_cuda.mk`` -- include and link flags for the library.

Supported classes: contracted four-index electron-repulsion integrals (four
Cartesian-Gaussian indices, one auxiliary index, a Boys function in the base
expression), Cartesian or spherical.  Anything else raises
``UnsupportedClass`` (pass ``fallback=True`` to have the reference back end
write C99 for the whole generator instead).
"""
import os

PKG = os.path.dirname(os.path.abspath(__file__))
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


def _is_eri_class(integral):
    """Four Cartesian-Gaussian indices, one auxiliary index, no extra
    arguments, and a Boys function in the base expression."""
    idx, aux, args = integral.index_list(), integral.aux_list(), integral.arg_list()
    if len(idx) != 4 or len(aux) != 1 or len(args) != 0:
        return False
    if not all(type(i).__name__ == 'dsl_cartesian_gaussian' for i in idx):
        return False
    base = integral.base()
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


def cuda_out(gen, fallback=False):
    """Write the CUDA-backed files for every class of ``gen`` (a reference
    ``generator``).  Returns the list of written paths."""
    opt = gen.generator_options()
    outdir = opt.output_directory()
    if not opt.contracted():
        if fallback:
            gen.out()
            return []
        raise UnsupportedClass('the CUDA back end implements contracted integrals (contracted=True)')
    spherical = bool(opt.spherical_transformed())
    variant = 'sph' if spherical else 'cart'
    ours = 'intception_integral_eri_abcd_m_cont_%s' % variant
    written = []
    os.makedirs(outdir, exist_ok=True)
    for wi in gen._wi_list:
        if not _is_eri_class(wi.integral()):
            if fallback:
                gen.out()
                return []
            raise UnsupportedClass('class %s is not an electron-repulsion integral' % wi.full_name())
        full = wi.full_name()
        hdr = os.path.join(outdir, wi.header_filename())
        guard = ''.join(ch if ch.isalnum() else '_' for ch in wi.header_filename()).upper()
        with open(hdr, 'w') as fh:
            fh.write('/* %s: implemented by lib%s.so (sm_100a); written by the cuda back end. */\n'
                     % (full, LIB_NAME))
            fh.write('#ifndef %s\n#define %s\n#ifdef __cplusplus\nextern "C" {\n#endif\n' % (guard, guard))
            fh.write('void %s_main( %s );\n' % (full, _main_args(spherical)))
            fh.write('int %s_work_array_size( %s );\n' % (full, _WSIZE))
            fh.write('int intception_b200_last_status(void);\nconst char *intception_b200_last_error(void);\n')
            fh.write('#ifdef __cplusplus\n}\n#endif\n#endif\n')
        written.append(hdr)
        if full != ours:
            shim = os.path.join(outdir, full + '_cuda.c')
            with open(shim, 'w') as fh:
                fh.write('/* Forwards %s to the library implementation %s. */\n' % (full, ours))
                fh.write('#include "%s"\n' % wi.header_filename())
                fh.write('void %s_main( %s );\n' % (ours, _main_args(spherical)))
                fh.write('int %s_work_array_size( %s );\n' % (ours, _WSIZE))
                fh.write('void %s_main( %s ) {\n  %s_main( %s );\n}\n'
                         % (full, _main_args(spherical), ours, _call_args(spherical)))
                fh.write('int %s_work_array_size( %s ) {\n  return %s_work_array_size( la, lb, lc, ld, na_prim, '
                         'nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont );\n}\n'
                         % (full, _WSIZE, ours))
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
    generator_cls.out = out
