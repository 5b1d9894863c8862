"""Contractions that mix tight and diffuse exponents on both shells of a pair.

The mixed_contraction_sph fixture holds quartets of the l <= 4, K <= 8
workload (exponents 0.02..1e5) for which no shell order keeps every
primitive pair's horizontal recurrence well conditioned, with exact values
(the C restatement evaluated in binary128).  The unrolled class kernels
estimate their HRR rounding error after contraction and hand such quartets to
the generic kernel, which builds each primitive pair on the shell that
conditions it; the generic kernel does the same for the classes it serves.
"""
import numpy as np
import pytest

from conftest import load_batch, tolerance
from intception_b200 import eri

pytestmark = pytest.mark.gpu


def _batch_run(b):
    eng = eri.EriEngine(b)
    out = eng.compute().cpu().numpy()
    assert eng.device_status() == eri.IB_OK
    return out


def test_mixed_contractions_match_exact_values():
    b, _, exact = load_batch('mixed_contraction_sph')
    out = _batch_run(b)
    assert eri.last_hrr_redo() > 0  # quartets of unrolled classes were handed over
    assert np.abs(out - exact).max() <= tolerance(exact)


def test_without_the_hrr_check_the_class_kernels_lose_digits():
    """The check is what keeps these quartets exact: switched off, the class
    kernels' single shell order cancels digits in the HRRs."""
    b, _, exact = load_batch('mixed_contraction_sph')
    eri.set_hrr_tol(0.0)
    try:
        out = _batch_run(b)
        assert eri.last_hrr_redo() == 0
    finally:
        eri.set_hrr_tol(1e-13)
    assert np.abs(out - exact).max() > tolerance(exact)


def test_dropin_mixed_contractions_match_exact_values():
    """The drop-in entry on the same quartets: one call per quartet, the
    class kernel (or the generic kernel) and its redo inside the call."""
    b, T, exact = load_batch('mixed_contraction_sph')
    for q in range(b.nq):
        s = b.quartets[q]
        ls = [int(b.shell_l[x]) for x in s]
        n = [2 * l + 1 for l in ls]
        skip = [1, n[0], n[0] * n[1], n[0] * n[1] * n[2]]
        shells = []
        for i, x in enumerate(s):
            p0, k = int(b.shell_ptr[x]), int(b.shell_k[x])
            shells.append(dict(x=b.prim_exp[p0:p0 + k], cen=b.shell_xyz[x], l=ls[i], n=n[i], iskip=skip[i],
                               nprim=k, ncont=1, iskip_cont=0, coef=b.prim_coef[p0:p0 + k], T=T[ls[i]]))
        out = np.zeros(int(np.prod(n)))
        eri.cont_sph_main(shells, out)
        ref = exact[b.out_off[q]:b.out_off[q] + out.size]
        assert np.abs(out - ref).max() <= tolerance(exact), q
