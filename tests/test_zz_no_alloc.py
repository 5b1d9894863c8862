"""The allocation-free batch entry point (intception_b200_eri_batch_noalloc).

It serves callers that cannot call cudaMalloc -- for example a host framework
whose own pool allocator owns the device memory -- by keeping its scratch and
descriptors in fixed-size file-scope device arrays.  Checked through the C ABI
against intception_b200_eri_batch on two calls in a row, so that state left in
the shared arrays by the first call cannot leak into the second.  This file is
collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import tolerance
from intception_b200 import basis, eri

pytestmark = pytest.mark.gpu


def _run_both(b):
    import torch
    eng = eri.EriEngine(b)
    ref = eng.compute()
    out = torch.full((b.out_size,), float('nan'), dtype=torch.float64, device='cuda')
    st = eri.load().intception_b200_eri_batch_noalloc(C.byref(eng._basis), eng.quartets.data_ptr(),
                                                       eng.out_off.data_ptr(), b.nq, 1 if b.spherical else 0,
                                                       out.data_ptr(), None)
    assert st == eri.IB_OK
    torch.cuda.synchronize()
    return ref.cpu().numpy(), out.cpu().numpy()


def test_noalloc_matches_batch_on_two_calls():
    b1 = basis.independent_quartet_batch(41, 300, [0, 1, 2, 3], [1, 2, 3], 0.1, 40.0, 4.0, True)
    b2 = basis.independent_quartet_batch(42, 200, [0, 1, 2], [1, 2, 4], 0.1, 40.0, 4.0, False)
    for b in (b1, b2):
        ref, out = _run_both(b)
        assert np.all(np.isfinite(out))
        assert np.abs(out - ref).max() <= tolerance(ref)


def test_noalloc_rejects_oversize_batch():
    b = basis.independent_quartet_batch(43, 4, [0, 1], [1], 0.1, 40.0, 4.0, False)
    eng = eri.EriEngine(b)
    st = eri.load().intception_b200_eri_batch_noalloc(C.byref(eng._basis), eng.quartets.data_ptr(),
                                                       eng.out_off.data_ptr(), 65537, 0, eng.out_off.data_ptr(),
                                                       None)
    assert st == eri.IB_ERR_ARG
