"""Generator back end 'cuda': runs the reference generator (when its source
tree is present) on the ERI input script and on the reference's example
script, writes the CUDA-backed files with gen.out(backend='cuda'), and
compiles and links a C caller against them and libintception_b200.so -- the
Makefile-flow switch, checked at link time.  Classes of a supported shape but
different algebra must be refused by the numerical verification."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import gen_ref  # noqa: E402

REF_SRC = os.path.join(gen_ref.reference_root(), 'src')

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_SRC, 'intception')),
                                reason='reference generator not available here')

def _run_script(tmp, name, spherical):
    """Build the ERI class of oracle/eri_input.py (optionally renamed) and
    call out(backend='cuda')."""
    src = open(os.path.join(ROOT, 'oracle', 'eri_input.py')).read()
    src = src.replace("name='eri'", "name=%r" % name)
    src = src.replace('gen.out()', "gen.out(backend='cuda')")
    pre = ('import sys, time\ntime.clock = time.perf_counter\nsys.path.insert(0, %r)\nsys.path.insert(0, %r)\n'
           'from intception.generator.generator import generator as _g\nfrom intception_b200 import frontend\n'
           'frontend.install(_g)\n' % (REF_SRC, ROOT))
    path = os.path.join(tmp, 'input_%s.py' % name)
    open(path, 'w').write(pre + src)
    env = dict(os.environ, ERI_OUTDIR=tmp, ERI_SPHERICAL='1' if spherical else '0', ERI_CONTRACTED='1')
    subprocess.run([sys.executable, path], check=True, env=env, cwd=tmp)


CALLER = r'''
#include <stdio.h>
#include "%(header)s"
int main(void) {
  double x[1] = {1.0}, c[1] = {1.0}, cen[3] = {0, 0, 0}, T[1] = {1.0}, work[1], out[1];
  int n = %(full)s_work_array_size(0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1);
  if (0) %(full)s_main(%(args)s);
  printf("%%d\n", n);
  return n > 0 ? 0 : 1;
}
'''


@pytest.mark.parametrize('name,spherical', [('eri', False), ('eri', True), ('coulomb', False)])
def test_cuda_backend_links(tmp_path, name, spherical):
    tmp = str(tmp_path)
    _run_script(tmp, name, spherical)
    v = 'sph' if spherical else 'cart'
    full = 'intception_integral_%s_abcd_m_cont_%s' % (name, v)
    header = full + '.h'
    files = os.listdir(tmp)
    assert header in files and 'boys_function.h' in files and 'intception_cuda.mk' in files
    assert (full + '_cuda.c' in files) == (name != 'eri')
    per = 'x, cen, 0, 1, 1, 1, 1, 0, c' + (', T' if spherical else '')
    caller = os.path.join(tmp, 'caller.c')
    open(caller, 'w').write(CALLER % dict(header=header, full=full, args=', '.join([per] * 4) + ', work, out'))
    srcs = [caller] + ([os.path.join(tmp, full + '_cuda.c')] if name != 'eri' else [])
    exe = os.path.join(tmp, 'caller')
    libdir = os.path.join(ROOT, 'intception_b200')
    subprocess.run(['gcc', '-std=c99', '-I', tmp] + srcs + ['-L', libdir, '-lintception_b200',
                                                            '-Wl,-rpath,' + libdir, '-o', exe], check=True)
    # the work-array size needs no GPU: run it
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and int(r.stdout.strip()) > 0


def _example_script(tmp, rename=None):
    """The reference's example script with out(backend='cuda'), run in tmp."""
    src = open(os.path.join(REF_SRC, '..', 'examples', 'example_input.py')).read()
    src = src.replace('output_directory = "./output"', 'output_directory = %r' % tmp)
    src = src.replace('gen.out()', "gen.out(backend='cuda')")
    if rename:
        src = src.replace("name='nuclear_2idx'", "name=%r" % rename)
    pre = ('import sys, time\ntime.clock = time.perf_counter\nsys.path.insert(0, %r)\nsys.path.insert(0, %r)\n'
           'from intception.generator.generator import generator as _g\nfrom intception_b200 import frontend\n'
           'frontend.install(_g)\n' % (REF_SRC, ROOT))
    path = os.path.join(tmp, 'example_cuda.py')
    open(path, 'w').write(pre + src)
    subprocess.run([sys.executable, path], check=True, cwd=tmp, stdout=subprocess.DEVNULL)


PAIR_CALLER = r'''
#include <stdio.h>
#include "intception_integral_overlap_2idx_ab_prim_cart.h"
#include "%(nuc)s.h"
int main(void) {
  double c[3] = {0, 0, 0}, work[1], out[1];
  int n = intception_integral_overlap_2idx_ab_prim_cart_work_array_size(2, 1) + %(nuc)s_work_array_size(2, 1);
  if (0) intception_integral_overlap_2idx_ab_prim_cart_main(1.0, c, 0, 1, 1, 1.0, c, 0, 1, 1, work, out);
  if (0) %(nuc)s_main(1.0, c, 0, 1, 1, 1.0, c, 0, 1, 1, c, work, out);
  printf("%%d\n", n);
  return 0;
}
'''


@pytest.mark.parametrize('rename', [None, 'attraction'])
def test_cuda_backend_example_script(tmp_path, rename):
    """The example's two primitive classes verify, and a caller links against
    the written headers (a renamed class gets a forwarding shim)."""
    tmp = str(tmp_path)
    _example_script(tmp, rename)
    nuc = 'intception_integral_%s_ab_m_cC_prim_cart' % (rename or 'nuclear_2idx')
    files = os.listdir(tmp)
    assert 'intception_integral_overlap_2idx_ab_prim_cart.h' in files and nuc + '.h' in files
    assert (nuc + '_cuda.c' in files) == bool(rename)
    assert not any(f.endswith('.c') and not f.endswith('_cuda.c') for f in files)
    caller = os.path.join(tmp, 'caller.c')
    open(caller, 'w').write(PAIR_CALLER % dict(nuc=nuc))
    srcs = [caller] + ([os.path.join(tmp, nuc + '_cuda.c')] if rename else [])
    exe = os.path.join(tmp, 'caller')
    libdir = os.path.join(ROOT, 'intception_b200')
    subprocess.run(['gcc', '-std=c99', '-I', tmp] + srcs + ['-L', libdir, '-lintception_b200',
                                                            '-Wl,-rpath,' + libdir, '-o', exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    # 2 idx: overlap ncum(2)*ncum(1) = 40; nuclear 2*(40 + 4) = 88
    assert r.returncode == 0 and int(r.stdout.strip()) == 40 + 88


def _overlap_class(tmp_path, contracted, full_vrr):
    sys.path.insert(0, REF_SRC)
    import time
    time.clock = time.perf_counter
    from intception import dsl_cartesian_gaussian, dsl_integral, dsl_scalar, dsl_position, exp, sqrt, dsl_value
    from intception.generator.generator import generator, generator_options
    from math import pi
    ga = dsl_cartesian_gaussian('a', constant=True)
    gb = dsl_cartesian_gaussian('b', constant=True)
    xa, xb, A, B = ga.exp(), gb.exp(), ga.cen(), gb.cen()
    xp = dsl_scalar('xp', xa + xb)
    o_o_xp = dsl_scalar('o_o_xp', 1.0 / xp)
    o_o_2xp = dsl_scalar('o_o_2xp', 0.5 * o_o_xp)
    AB = dsl_position('AB', A - B)
    PA = dsl_position('PA', xb * o_o_xp * -AB)
    PB = dsl_position('PB', xa * o_o_xp * AB)
    RAB2 = dsl_scalar('RAB2', AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2])
    pi3 = dsl_value(name='pi3', value=pi ** 3, vartype='double')
    ov = dsl_integral(ga, gb, name='overlap_2idx')
    ov.set_base(sqrt(pi3 * o_o_xp * o_o_xp * o_o_xp) * exp(-xa * xb * o_o_xp * RAB2))
    if full_vrr:
        ov.add_vrr('vrr1', ga, PA * ov.int(ga - 1, gb) + o_o_2xp * (ga - 1) * ov.int(ga - 2, gb)
                   + o_o_2xp * gb * ov.int(ga - 1, gb - 1))
        ov.add_vrr('vrr2', gb, PB * ov.int(ga, gb - 1) + o_o_2xp * (gb - 1) * ov.int(ga, gb - 2)
                   + o_o_2xp * ga * ov.int(ga - 1, gb - 1))
    else:  # the recurrence terms in a-1 / b-2 left out: a different integral
        ov.add_vrr('vrr1', ga, PA * ov.int(ga - 1, gb))
        ov.add_vrr('vrr2', gb, PB * ov.int(ga, gb - 1))
    return generator(ov, opt=generator_options(output_directory=str(tmp_path), silent=True, contracted=contracted))


def test_unsupported_options_rejected(tmp_path):
    from intception_b200 import frontend
    gen = _overlap_class(tmp_path, contracted=True, full_vrr=True)
    with pytest.raises(frontend.UnsupportedClass, match='primitive'):
        frontend.cuda_out(gen)


def test_different_algebra_rejected(tmp_path):
    """Right shape, wrong recurrences: the numerical verification refuses it;
    with fallback=True the reference back end writes C99 instead."""
    from intception_b200 import frontend
    gen = _overlap_class(tmp_path, contracted=False, full_vrr=False)
    with pytest.raises(frontend.UnsupportedClass, match='not its values'):
        frontend.cuda_out(gen)
    assert frontend.cuda_out(gen, fallback=True) == []
    assert any(f.endswith('.c') for f in os.listdir(str(tmp_path)))


def test_same_algebra_other_names_verifies(tmp_path):
    """The overlap written with other variable names is the same integral."""
    from intception_b200 import frontend
    gen = _overlap_class(tmp_path, contracted=False, full_vrr=True)
    written = frontend.cuda_out(gen)
    assert any(p.endswith('intception_integral_overlap_2idx_ab_prim_cart.h') for p in written)
