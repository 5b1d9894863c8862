"""Intception input script for the four-index electron-repulsion integral (ERI).

Test infrastructure: this script is fed to the reference generator by
``oracle/gen_ref.py`` to emit the C99 oracle.  The reference repository ships no
ERI input script (its only example builds 2-index overlap and nuclear attraction,
``examples/example_input.py:58-110``), so this one is authored here with the same
DSL: Obara-Saika VRRs on a, c and d with the auxiliary Boys index m, then the one
Head-Gordon-Pople HRR the DSL allows (a -> b, ``dsl_extensions.py:903-950``).

Usage (the reference package must be importable, see gen_ref.py):
    ERI_CONTRACTED=1 ERI_SPHERICAL=0 ERI_OUTDIR=dir python eri_input.py
"""
import os
from math import pi
from intception import *

ga = dsl_cartesian_gaussian('a', constant=True)
gb = dsl_cartesian_gaussian('b', constant=True)
gc = dsl_cartesian_gaussian('c', constant=True)
gd = dsl_cartesian_gaussian('d', constant=True)
xa, xb, xc, xd = ga.exp(), gb.exp(), gc.exp(), gd.exp()
A, B, C, D = ga.cen(), gb.cen(), gc.cen(), gd.cen()
m = dsl_integer_index(name='m')

two_pi52 = dsl_value(name='two_pi52', value=2.0 * pi ** 2.5, vartype='double')

# bra pair
zeta = dsl_scalar('zeta', xa + xb)
o_o_zeta = dsl_scalar('o_o_zeta', 1.0 / zeta)
o_o_2zeta = dsl_scalar('o_o_2zeta', 0.5 * o_o_zeta)
xi_ab = dsl_scalar('xi_ab', xa * xb * o_o_zeta)
AB = dsl_position('AB', A - B)
RAB2 = dsl_scalar('RAB2', AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2])
P = dsl_position('P', (xa * A + xb * B) * o_o_zeta)
PA = dsl_position('PA', P - A)
# ket pair
eta = dsl_scalar('eta', xc + xd)
o_o_eta = dsl_scalar('o_o_eta', 1.0 / eta)
o_o_2eta = dsl_scalar('o_o_2eta', 0.5 * o_o_eta)
xi_cd = dsl_scalar('xi_cd', xc * xd * o_o_eta)
CD = dsl_position('CD', C - D)
RCD2 = dsl_scalar('RCD2', CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2])
Q = dsl_position('Q', (xc * C + xd * D) * o_o_eta)
QC = dsl_position('QC', Q - C)
QD = dsl_position('QD', Q - D)
# quartet
o_o_zpe = dsl_scalar('o_o_zpe', 1.0 / (zeta + eta))
o_o_2zpe = dsl_scalar('o_o_2zpe', 0.5 * o_o_zpe)
rho = dsl_scalar('rho', zeta * eta * o_o_zpe)
rho_o_zeta = dsl_scalar('rho_o_zeta', rho * o_o_zeta)
rho_o_eta = dsl_scalar('rho_o_eta', rho * o_o_eta)
W = dsl_position('W', (zeta * P + eta * Q) * o_o_zpe)
WP = dsl_position('WP', W - P)
WQ = dsl_position('WQ', W - Q)
PQ = dsl_position('PQ', P - Q)
RPQ2 = dsl_scalar('RPQ2', PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2])

eri = dsl_integral(ga, gb, gc, gd, m, name='eri')
eri.set_base(two_pi52 * o_o_zeta * o_o_eta * sqrt(o_o_zpe)
             * exp(-xi_ab * RAB2 - xi_cd * RCD2) * boys_f(m, rho * RPQ2))
# [a+1i,0|c,d]: b is zero throughout the VRR stage
eri.add_vrr('vrra', ga,
            PA * eri.int(ga - 1, gb, gc, gd, m) + WP * eri.int(ga - 1, gb, gc, gd, m + 1)
            + o_o_2zeta * (ga - 1) * (eri.int(ga - 2, gb, gc, gd, m)
                                      - rho_o_zeta * eri.int(ga - 2, gb, gc, gd, m + 1)))
eri.add_vrr('vrrc', gc,
            QC * eri.int(ga, gb, gc - 1, gd, m) + WQ * eri.int(ga, gb, gc - 1, gd, m + 1)
            + o_o_2eta * (gc - 1) * (eri.int(ga, gb, gc - 2, gd, m)
                                     - rho_o_eta * eri.int(ga, gb, gc - 2, gd, m + 1))
            + o_o_2zpe * ga * eri.int(ga - 1, gb, gc - 1, gd, m + 1))
eri.add_vrr('vrrd', gd,
            QD * eri.int(ga, gb, gc, gd - 1, m) + WQ * eri.int(ga, gb, gc, gd - 1, m + 1)
            + o_o_2eta * (gd - 1) * (eri.int(ga, gb, gc, gd - 2, m)
                                     - rho_o_eta * eri.int(ga, gb, gc, gd - 2, m + 1))
            + o_o_2eta * gc * (eri.int(ga, gb, gc - 1, gd - 1, m)
                               - rho_o_eta * eri.int(ga, gb, gc - 1, gd - 1, m + 1))
            + o_o_2zpe * ga * eri.int(ga - 1, gb, gc, gd - 1, m + 1))
eri.add_hrr('hrrb', ga, gb)

contracted = os.environ.get('ERI_CONTRACTED', '1') == '1'
spherical = os.environ.get('ERI_SPHERICAL', '0') == '1'
outdir = os.environ.get('ERI_OUTDIR', './output')
lmax = int(os.environ.get('ERI_LMAX', '6'))
opt = generator_options(output_directory=outdir, contracted=contracted,
                        spherical_transformed=spherical, global_user_lmax=lmax,
                        silent=True)
gen = generator(eri, opt=opt)
gen.out()
