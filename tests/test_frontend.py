"""Generator back end 'cuda': runs the reference generator (when its source
tree is present) on the ERI input script, writes the CUDA-backed files with
gen.out(backend='cuda'), and compiles and links a C caller against them and
libintception_b200.so -- the Makefile-flow switch, checked at link time."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = '/root/reference/src'

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


def test_unsupported_class_rejected(tmp_path):
    sys.path.insert(0, REF_SRC)
    import time
    time.clock = time.perf_counter
    from intception import dsl_cartesian_gaussian, dsl_integral, dsl_scalar, dsl_position, exp, sqrt, dsl_value
    from intception.generator.generator import generator, generator_options
    from intception_b200 import frontend
    from math import pi
    ga = dsl_cartesian_gaussian('a', constant=True)
    gb = dsl_cartesian_gaussian('b', constant=True)
    xp = dsl_scalar('xp', ga.exp() + gb.exp())
    ov = dsl_integral(ga, gb, name='overlap_2idx')
    pi3 = dsl_value(name='pi3', value=pi ** 3, vartype='double')
    ov.set_base(sqrt(pi3 / (xp * xp * xp)) * exp(-ga.exp() * gb.exp() / xp))
    ov.add_vrr('vrr1', ga, dsl_position('PA', gb.exp() / xp * (gb.cen() - ga.cen())) * ov.int(ga - 1, gb))
    ov.add_vrr('vrr2', gb, dsl_position('PB', ga.exp() / xp * (ga.cen() - gb.cen())) * ov.int(ga, gb - 1))
    gen = generator(ov, opt=generator_options(output_directory=str(tmp_path), silent=True))
    with pytest.raises(frontend.UnsupportedClass):
        frontend.cuda_out(gen)
