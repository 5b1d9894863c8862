"""The allocation-free batch entry point (intception_b200_eri_batch_noalloc).

It serves callers that cannot call cudaMalloc -- for example a host framework
whose own pool allocator owns the device memory -- by keeping its scratch and
descriptors in fixed-size file-scope device arrays.  Checked through the C ABI
against intception_b200_eri_batch on two calls in a row, so that state left in
the shared arrays by the first call cannot leak into the second, with the
entry's own device status word read after every call.  This file is collected
last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import tolerance
from intception_b200 import basis, eri

pytestmark = pytest.mark.gpu


def _noalloc(eng, b, out):
    lib = eri.load()
    st = lib.intception_b200_eri_batch_noalloc(C.byref(eng._basis), eng.quartets.data_ptr(), eng.out_off.data_ptr(),
                                               b.nq, 1 if b.spherical else 0, out.data_ptr(), None)
    assert st == eri.IB_OK
    assert lib.intception_b200_last_status() == eri.IB_OK
    return lib.intception_b200_noalloc_status(None)


def _run_both(b, lmax=None):
    """(batch result, batch device status, allocation-free result, its device
    status); both outputs start as NaN so that unwritten elements show."""
    import torch
    eng = eri.EriEngine(b)
    if lmax is not None:
        eng._basis.lmax = lmax
    ref = torch.full((b.out_size,), float('nan'), dtype=torch.float64, device='cuda')
    eng.compute(out=ref)
    torch.cuda.synchronize()
    st_ref = eng.device_status()
    out = torch.full((b.out_size,), float('nan'), dtype=torch.float64, device='cuda')
    st = _noalloc(eng, b, out)
    torch.cuda.synchronize()
    return ref.cpu().numpy(), st_ref, out.cpu().numpy(), st


def test_noalloc_matches_batch_on_two_calls():
    b1 = basis.independent_quartet_batch(41, 300, [0, 1, 2, 3], [1, 2, 3], 0.1, 40.0, 4.0, True)
    b2 = basis.independent_quartet_batch(42, 200, [0, 1, 2], [1, 2, 4], 0.1, 40.0, 4.0, False)
    for b in (b1, b2):
        ref, st_ref, out, st = _run_both(b)
        assert st_ref == eri.IB_OK and st == eri.IB_OK
        assert np.all(np.isfinite(out))
        assert np.abs(out - ref).max() <= tolerance(ref)


@pytest.mark.parametrize('sph', [False, True])
def test_noalloc_f_shells_diffuse_and_compact(sph):
    """f shells with exponents down to 0.1 next to tight ones, centres 3 bohr
    apart: the setting where the HRRs cancel digits unless the compact shell
    of an equal-l pair comes first."""
    b = basis.independent_quartet_batch(44 + sph, 150, [2, 3], [1, 2, 3], 0.1, 200.0, 3.0, sph)
    ref, st_ref, out, st = _run_both(b)
    assert st_ref == eri.IB_OK and st == eri.IB_OK
    assert np.abs(out - ref).max() <= tolerance(ref)


def test_noalloc_lmax6_one_quartet_slice():
    """lmax 6, where a single quartet's recurrence levels fill the static
    scratch (one slice, one block)."""
    b = basis.independent_quartet_batch(46, 4, [4, 5, 6], [1, 2], 0.3, 5.0, 3.0, True)
    ref, st_ref, out, st = _run_both(b)
    assert st_ref == eri.IB_OK and st == eri.IB_OK
    assert np.abs(out - ref).max() <= tolerance(ref)


def test_noalloc_bad_l_reports_status_like_batch():
    """Quartets with a shell above the basis's declared lmax: both entries set
    IB_ERR_ARG and write the (ss|ss) value into the first element of the block."""
    b = basis.independent_quartet_batch(47, 60, [0, 1, 3], [1, 2], 0.1, 40.0, 4.0, False)
    bad = (b.shell_l[b.quartets] > 1).any(axis=1)
    assert bad.any() and (~bad).any()
    ref, st_ref, out, st = _run_both(b, lmax=1)
    assert st_ref == eri.IB_ERR_ARG and st == eri.IB_ERR_ARG
    assert np.array_equal(np.isnan(out), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.abs(out[ok] - ref[ok]).max() <= tolerance(ref[ok])
    # the next good call clears the word
    b2 = basis.independent_quartet_batch(48, 20, [0, 1], [1, 2], 0.1, 40.0, 4.0, False)
    _, _, _, st2 = _run_both(b2)
    assert st2 == eri.IB_OK


def test_noalloc_rejects_oversize_batch():
    b = basis.independent_quartet_batch(43, 4, [0, 1], [1], 0.1, 40.0, 4.0, False)
    eng = eri.EriEngine(b)
    lib = eri.load()
    st = lib.intception_b200_eri_batch_noalloc(C.byref(eng._basis), eng.quartets.data_ptr(), eng.out_off.data_ptr(),
                                               65537, 0, eng.out_off.data_ptr(), None)
    assert st == eri.IB_ERR_ARG
    assert lib.intception_b200_last_status() == eri.IB_ERR_ARG
    assert b'65536' in lib.intception_b200_last_error()
