"""Regenerate Boys-function tables F_m(x) with mpmath (test infrastructure).

The reference stores two tables as JSON (``boys.py:27-69``; data files
``boys_data/boys_data_smallx.json`` and ``boys_data_mediumx.json``):
  * small x: x_i = 0.1*i, i = 0..150, F_0..F_32 at each point,
  * medium x: x_i = 15 + 0.1*i, i = 0..200, F_0..F_6 at each point.
The values are the mathematical function F_m(x) = int_0^1 t^{2m} exp(-x t^2) dt,
so this script recomputes them independently at 40 significant digits and
writes a C header with the two arrays under the names the oracle uses.

F_m(x) = 1F1(m+1/2; m+3/2; -x) / (2m+1)   (Kummer form, valid for all x >= 0).

Usage:  python oracle/gen_boys_tables.py oracle/_gen/boys_tables.h
"""
import os
import sys

import mpmath

mpmath.mp.dps = 40


def boys(m, x):
    x = mpmath.mpf(x)
    if x == 0:
        return mpmath.mpf(1) / (2 * m + 1)
    return mpmath.hyp1f1(m + mpmath.mpf(1) / 2, m + mpmath.mpf(3) / 2, -x) / (2 * m + 1)


def table(x0, npts, step_tenths, nvals):
    rows = []
    for i in range(npts):
        x = mpmath.mpf(x0) + mpmath.mpf(i * step_tenths) / 10
        rows.append([boys(m, x) for m in range(nvals)])
    return rows


def fmt(v):
    return mpmath.nstr(v, 20, min_fixed=0, max_fixed=0, strip_zeros=False)


def write_header(path):
    small = table(0, 151, 1, 33)
    medium = table(15, 201, 1, 7)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, 'w') as fh:
        fh.write('/* Generated by oracle/gen_boys_tables.py (mpmath %s, 40 digits). */\n'
                 % mpmath.__version__)
        fh.write('static const double oracle_boys_smallx[151][33] = {\n')
        for row in small:
            fh.write('  {' + ', '.join(fmt(v) for v in row) + '},\n')
        fh.write('};\n')
        fh.write('static const double oracle_boys_mediumx[201][7] = {\n')
        for row in medium:
            fh.write('  {' + ', '.join(fmt(v) for v in row) + '},\n')
        fh.write('};\n')


if __name__ == '__main__':
    write_header(sys.argv[1] if len(sys.argv) > 1 else
                 os.path.join(os.path.dirname(os.path.abspath(__file__)), '_gen', 'boys_tables.h'))
