"""Record the probe checksums the generator back end 'cuda' verifies classes
against (intception_b200/fingerprints.json).

Test infrastructure recipe: runs the probes of intception_b200.frontend on the
reference's own emitted C99 for each supported class (oracle/_ref, built by
oracle/gen_ref.py from the reference tree) and writes the checksums.

    python oracle/gen_ref.py && python oracle/make_fingerprints.py
"""
import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from intception_b200 import frontend  # noqa: E402


def main():
    ref = os.path.join(HERE, '_ref')
    libs = {'eri_cont_cart': 'libref_eri_cart.so', 'eri_cont_sph': 'libref_eri_sph.so',
            'overlap_2idx_prim_cart': 'libref_2idx.so', 'nuclear_2idx_prim_cart': 'libref_2idx.so'}
    out = {}
    for mode, so in libs.items():
        lib = C.CDLL(os.path.join(ref, so))
        out[mode] = frontend.probe_checksums(lib, mode, frontend.LIBRARY_CLASS[mode])
        print(mode, out[mode])
    with open(frontend.FINGERPRINTS, 'w') as fh:
        json.dump(out, fh, indent=1)
        fh.write('\n')


if __name__ == '__main__':
    main()
