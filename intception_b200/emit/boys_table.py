"""Device Boys-function table, regenerated with mpmath at build time.

The device evaluates F_L(T) for T < BOYS_TMAX by a 7-term Taylor expansion about
the nearest grid point T_i = i*h (h = 1/16, |T - T_i| <= 1/32), then walks down
to F_0 with F_m = (2T F_{m+1} + e^{-T}) / (2m+1).  The same scheme the reference
uses (``generator_boys_function.py:140-163``) on a grid 1.6x finer, so the
truncation error (1/32)^7/7! F_{L+7} stays below 1e-16 absolute.

Row i of the table holds g_k = F_k(T_i) for k = 0..BOYS_NCOL-1.  The device code
stages, per angular-momentum class, the seven columns L..L+6 divided by k! into
shared memory.
"""
import os
import sys

import mpmath

BOYS_H_INV = 16          # grid points per unit T
BOYS_TMAX = 36.0         # table range [0, TMAX]; above it: asymptotic + upward recursion
BOYS_NPTS = int(BOYS_TMAX * BOYS_H_INV) + 2
BOYS_NCOL = 4 * 6 + 7 + 1  # F_0..F_31: L <= 24 (l <= 6 per shell) plus 7 Taylor terms


def boys(m, x):
    x = mpmath.mpf(x)
    if x == 0:
        return mpmath.mpf(1) / (2 * m + 1)
    return mpmath.hyp1f1(m + mpmath.mpf(1) / 2, m + mpmath.mpf(3) / 2, -x) / (2 * m + 1)


def write_headers(outdir):
    """boys_table.h (grid parameters) and boys_table_data.h (the values)."""
    mpmath.mp.dps = 30
    params = ['/* Generated by intception_b200/emit/boys_table.py. */',
              '#pragma once',
              '#define IB_BOYS_H_INV %d' % BOYS_H_INV,
              '#define IB_BOYS_TMAX %.1f' % BOYS_TMAX,
              '#define IB_BOYS_NPTS %d' % BOYS_NPTS,
              '#define IB_BOYS_NCOL %d' % BOYS_NCOL]
    _write(os.path.join(outdir, 'boys_table.h'), params)
    lines = ['/* Generated by intception_b200/emit/boys_table.py with mpmath %s. */' % mpmath.__version__,
             '#pragma once',
             '#include "boys_table.h"',
             'static const double ib_boys_host_table[IB_BOYS_NPTS * IB_BOYS_NCOL] = {']
    for i in range(BOYS_NPTS):
        x = mpmath.mpf(i) / BOYS_H_INV
        # downward recursion in mpmath from the top column is exact enough and fast
        top = boys(BOYS_NCOL - 1, x)
        ex = mpmath.e ** (-x)
        col = [None] * BOYS_NCOL
        col[-1] = top
        for m in range(BOYS_NCOL - 2, -1, -1):
            col[m] = (2 * x * col[m + 1] + ex) / (2 * m + 1)
        lines.append('  ' + ', '.join(mpmath.nstr(v, 19, min_fixed=0, max_fixed=0) for v in col) + ',')
    lines.append('};')
    _write(os.path.join(outdir, 'boys_table_data.h'), lines)


def _write(path, lines):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    text = '\n'.join(lines) + '\n'
    if os.path.exists(path):
        with open(path) as fh:
            if fh.read() == text:
                return
    tmp = path + '.tmp'
    with open(tmp, 'w') as fh:
        fh.write(text)
    os.replace(tmp, path)


if __name__ == '__main__':
    write_headers(sys.argv[1])
