"""Shared test configuration: the gpu marker, the repository on sys.path and
loaders for the golden fixtures (tests/golden/*.npz, made by make_golden.py
from the reference's own emitted C99)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason='no CUDA device')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)


BATCH_FIXTURES = ['pppp_k3_cart', 'c1_pppp_k3_cart_4096', 'mixed_l2_sph_c2', 'mixed_l2_sph_compact',
                  'mixed_l2_cart_compact', 'l4_cart', 'l4_sph', 'l6_cart', 'l6_sph', 'edge_cart', 'edge_sph']


def load_batch(name):
    """(ShellBatch, list of sph matrices, reference output) of a fixture."""
    from intception_b200 import basis
    z = np.load(os.path.join(GOLDEN, name + '.npz'))
    sph = bool(z['spherical'])
    b = basis.ShellBatch(z['shell_l'], z['shell_k'], z['shell_ptr'], z['shell_xyz'], z['prim_exp'],
                         z['prim_coef'], z['quartets'], z['out_off'], sph, int(z['out_size']))
    flat = z['sph']
    T, o = [], 0
    for l in range(7):
        nc, ns = (l + 1) * (l + 2) // 2, 2 * l + 1
        T.append(flat[o:o + nc * ns].reshape((nc, ns), order='F'))
        o += nc * ns
    return b, T, z['out']


def load_dropin_cases():
    z = np.load(os.path.join(GOLDEN, 'dropin_cases.npz'))
    cases = []
    for k in range(int(z['ncases'])):
        shells = []
        for i in range(4):
            l, n, iskip, nprim, ncont, iskip_cont = (int(v) for v in z['case%d_%d_int' % (k, i)])
            nc = (l + 1) * (l + 2) // 2
            shells.append(dict(x=z['case%d_%d_x' % (k, i)], cen=z['case%d_%d_cen' % (k, i)],
                               coef=z['case%d_%d_coef' % (k, i)],
                               T=z['case%d_%d_T' % (k, i)].reshape((nc, 2 * l + 1), order='F'),
                               l=l, n=n, iskip=iskip, nprim=nprim, ncont=ncont, iskip_cont=iskip_cont))
        cases.append((shells, z['case%d_out' % k], bool(z['case%d_sph' % k])))
    return cases


def tolerance(ref):
    """FP64 parity bar: a flat 1e-12 absolute wherever max |I| <= 10 (every ERI
    fixture: the largest, edge_*, reaches 1.63); above 10 the bar becomes
    1e-13 relative to max |I| (1e-12 absolute would ask for 16 digits)."""
    m = float(np.abs(ref).max()) if np.size(ref) else 0.0
    return 1e-12 if m <= 10.0 else 1e-13 * m
