"""Build the reference's own CPU implementation of the ERI path into oracle/_ref/.

Test infrastructure only (the oracle is the checker, never the product).

The reference is a Python code generator; its CPU implementation of the hot path
is the C99 it emits for an ERI input script.  This recipe
  1. imports the reference generator from its source tree (read-only),
     with ``time.clock`` restored (removed in Python 3.8; the reference's
     ``timer.py:31,36`` still calls it),
  2. runs ``oracle/eri_input.py`` for the contracted Cartesian and contracted
     spherical variants, writing C99 into ``oracle/_ref/gen_{cart,sph}/``,
  3. compiles each variant as one translation unit (``#include`` of every emitted
     ``.c``; the emitted ``boys_function.h`` declares its tables without
     ``extern``, ``generator.py:1608-1612``, which gcc>=10 rejects at link time
     across several objects) together with the OpenMP batch driver
     ``oracle/ref_batch.c`` into ``oracle/_ref/libref_eri_{cart,sph}.so``.

Usage:  python oracle/gen_ref.py [--reference PATH] [--lmax 6]
The reference tree is --reference, else $INTCEPTION_REFERENCE, else the
read-only mount this recipe was written for (``reference_root()``).  Nothing
here runs on the GPU box: the built ``oracle/_ref`` travels with the tree.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, '_ref')
_DEFAULT_REFERENCE = '/root/reference'  # where this recipe reads the reference tree unless told otherwise


def reference_root():
    """The reference source tree: $INTCEPTION_REFERENCE, else the default
    mount.  Callers check os.path.isdir(<root>/src/intception) themselves."""
    return os.environ.get('INTCEPTION_REFERENCE', _DEFAULT_REFERENCE)


def generate(reference, variant, lmax):
    outdir = os.path.join(REF_OUT, 'gen_' + variant)
    os.makedirs(outdir, exist_ok=True)
    env = dict(os.environ)
    env['ERI_CONTRACTED'] = '1'
    env['ERI_SPHERICAL'] = '1' if variant == 'sph' else '0'
    env['ERI_OUTDIR'] = outdir
    env['ERI_LMAX'] = str(lmax)
    shim = ("import sys, time, runpy; time.clock = time.perf_counter; "
            "sys.path.insert(0, %r); runpy.run_path(%r, run_name='__main__')"
            % (os.path.join(reference, 'src'), os.path.join(HERE, 'eri_input.py')))
    subprocess.run([sys.executable, '-c', shim], check=True, env=env, cwd=outdir)
    return outdir


def compile_variant(outdir, variant):
    srcs = sorted(f for f in os.listdir(outdir) if f.endswith('.c') and f != 'unity.c')
    unity = os.path.join(outdir, 'unity.c')
    with open(unity, 'w') as fh:
        fh.write('#include <math.h>\n')
        for s in srcs:
            fh.write('#include "%s"\n' % s)
        # OpenMP batch driver: the emitted per-quartet function called from C,
        # no Python in the timed loop
        fh.write('#include "ref_batch.c"\n')
    so = os.path.join(REF_OUT, 'libref_eri_%s.so' % variant)
    cmd = ['gcc', '-std=gnu99', '-O3', '-march=native', '-fPIC', '-shared', '-fopenmp', '-w',
           '-DREF_VARIANT_%s' % variant.upper(), '-I', outdir, '-I', HERE, unity, '-o', so, '-lm']
    subprocess.run(cmd, check=True)
    return so


def build_example(reference):
    """The reference's own example script (2-index overlap and nuclear
    attraction, primitive Cartesian), run from oracle/_ref/gen_2idx so that its
    output_directory './output' lands there, compiled with ref_batch_2idx.c."""
    work = os.path.join(REF_OUT, 'gen_2idx')
    outdir = os.path.join(work, 'output')
    os.makedirs(outdir, exist_ok=True)
    shim = ("import sys, time, runpy; time.clock = time.perf_counter; "
            "sys.path.insert(0, %r); runpy.run_path(%r, run_name='__main__')"
            % (os.path.join(reference, 'src'), os.path.join(reference, 'examples', 'example_input.py')))
    subprocess.run([sys.executable, '-c', shim], check=True, cwd=work, stdout=subprocess.DEVNULL)
    srcs = sorted(f for f in os.listdir(outdir) if f.endswith('.c') and f != 'unity.c')
    unity = os.path.join(outdir, 'unity.c')
    with open(unity, 'w') as fh:
        fh.write('#include <math.h>\n')
        for s in srcs:
            fh.write('#include "%s"\n' % s)
        fh.write('#include "ref_batch_2idx.c"\n')
    so = os.path.join(REF_OUT, 'libref_2idx.so')
    subprocess.run(['gcc', '-std=gnu99', '-O3', '-march=native', '-fPIC', '-shared', '-fopenmp', '-w', '-I', outdir,
                    '-I', HERE, unity, '-o', so, '-lm'], check=True)
    return so


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=reference_root())
    ap.add_argument('--lmax', type=int, default=6)
    args = ap.parse_args()
    if not os.path.isdir(os.path.join(args.reference, 'src', 'intception')):
        print('reference tree not found at %s; skipping oracle/_ref build' % args.reference)
        return 1
    os.makedirs(REF_OUT, exist_ok=True)
    for variant in ('cart', 'sph'):
        outdir = generate(args.reference, variant, args.lmax)
        print(compile_variant(outdir, variant))
    print(build_example(args.reference))
    return 0


if __name__ == '__main__':
    sys.exit(main())
