"""The probe checksums the generator back end 'cuda' verifies classes against
(intception_b200/fingerprints.json, recorded from the reference's emitted
C99): every supported class has them, and the library's own drop-ins
reproduce them on the GPU."""
import ctypes as C
import json

import pytest


def test_every_library_class_has_fingerprints():
    from intception_b200 import frontend
    with open(frontend.FINGERPRINTS) as fh:
        fp = json.load(fh)
    assert set(fp) == set(frontend.LIBRARY_CLASS)
    assert len(fp['eri_cont_cart']) == len(frontend._ERI_PROBES)
    assert len(fp['nuclear_2idx_prim_cart']) == len(frontend._PAIR_PROBES)


@pytest.mark.gpu
@pytest.mark.parametrize('mode', ['eri_cont_cart', 'eri_cont_sph', 'overlap_2idx_prim_cart',
                                  'nuclear_2idx_prim_cart'])
def test_library_reproduces_fingerprints(mode):
    from intception_b200 import eri, frontend
    with open(frontend.FINGERPRINTS) as fh:
        want = json.load(fh)[mode]
    lib = C.CDLL(eri.LIB_PATH)
    got = frontend.probe_checksums(lib, mode, frontend.LIBRARY_CLASS[mode])
    assert eri.load().intception_b200_last_status() == 0
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-11 * max(1.0, abs(w))
