"""The C-ABI boundary without a GPU: libintception_b200.so loads and exports
every function include/*.h declares (no compute calls)."""
import ctypes
import glob
import os
import subprocess

from conftest import ROOT
from intception_b200 import eri


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, 'include', '*.h')):
        names.update(eri.header_functions(h))
    return sorted(names)


def test_header_declares_the_dropins():
    names = _declared()
    for v in ('cart', 'sph'):
        assert 'intception_integral_eri_abcd_m_cont_%s_main' % v in names
        assert 'intception_integral_eri_abcd_m_cont_%s_work_array_size' % v in names
    assert 'intception_boys' in names
    assert len(names) > 20


def test_library_exports_every_declared_symbol():
    assert os.path.exists(eri.LIB_PATH), 'build the library first (python -m intception_b200.build)'
    lib = ctypes.CDLL(eri.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_exported_symbols_have_c_linkage():
    out = subprocess.run(['nm', '-D', '--defined-only', eri.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for n in _declared():
        assert n in exported, n  # unmangled name: extern "C"


def test_load_binds_every_entry_point():
    lib = eri.load()  # sets argtypes on the entry points the Python layer calls; no device work
    assert lib.intception_b200_set_slice_cap.restype is ctypes.c_int


def test_library_work_array_size_matches_reference_golden():
    """The library's own exported ..._work_array_size (the drop-in callers size
    work_array with it, contracted_general.py:240-502) on the 1875 argument
    sets the reference's emitted C99 answered in tests/golden/work_array_size.npz;
    host-only, no device work."""
    import numpy as np
    from conftest import GOLDEN
    t = np.load(os.path.join(GOLDEN, 'work_array_size.npz'))['table']
    lib = eri.load()
    for v in ('cart', 'sph'):
        f = getattr(lib, 'intception_integral_eri_abcd_m_cont_%s_work_array_size' % v)
        got = np.array([f(*map(int, r[:12])) for r in t])
        assert np.array_equal(got, t[:, 12]), v
        assert eri.work_array_size(*map(int, t[7, :12]), spherical=(v == 'sph')) == t[7, 12]
