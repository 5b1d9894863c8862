"""Heavy quartets of the generic kernel: one quartet shared by a cluster.

A quartet of 512 or more primitive quartets that the generic kernel evaluates
(its class has no unrolled kernel, or the HRR check put it on the redo list)
is split over the 8 blocks of a thread-block cluster, each taking every 8th
primitive quartet; the partial contracted tables are summed in rank order.
These tests put such quartets beside light ones, check them against exact
values, and check that a batch gives the same bits run after run.
"""
import numpy as np
import pytest

from conftest import load_batch, tolerance
from intception_b200 import basis, eri

pytestmark = pytest.mark.gpu


def _run(b):
    eng = eri.EriEngine(b)
    out = eng.compute().cpu().numpy()
    assert eng.device_status() == eri.IB_OK
    return out


def test_heavy_generic_quartets_match_exact_values():
    # l 3..4: (gf|gf), (gg|gf), (gg|gg) run on the generic kernel, the other
    # classes on their unrolled kernels beside it; K = 5 on every shell of the
    # first 16 quartets (625 primitive quartets each, above the split
    # threshold of 512), K in 1, 2, 5 on the rest.  The exact values are
    # binary128 evaluations of the C restatement
    b, _, exact = load_batch('generic_split_sph')
    out = _run(b)
    assert np.abs(out - exact).max() <= tolerance(exact)


def test_heavy_generic_quartets_are_reproducible():
    # the generic range: (gg|gg) quartets of K 6..8, split over 2-block clusters
    b = basis.independent_quartet_batch(12, 64, [4], [6, 7, 8], 0.05, 1.0e4, 5.0, True)
    assert np.array_equal(_run(b), _run(b))


def test_cluster_grids():
    import torch
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    full = eri.generic_grid(1)
    assert full >= nsm
    for cs in (2, 4):
        g = eri.generic_grid(cs)
        assert 0 < g <= full and g % cs == 0
    assert eri.generic_grid(3) == -1


def test_split_redo_lists_are_reproducible():
    # the redo lists (4-block clusters): quartets of unrolled classes the HRR check hands over
    b, _, _ = load_batch('mixed_contraction_sph')
    first = _run(b)
    redo = eri.last_hrr_redo()
    assert redo > 0
    second = _run(b)
    assert eri.last_hrr_redo() == redo
    assert np.array_equal(first, second)
