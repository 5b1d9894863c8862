"""Two-index primitive Cartesian classes of the reference's example script
(``examples/example_input.py:83-107``): ``overlap_2idx`` and ``nuclear_2idx``.

* ``overlap_main`` / ``nuclear_main`` take the emitted argument lists of
  ``intception_integral_overlap_2idx_ab_prim_cart_main`` and
  ``intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main``
  (``primitive_general.py:31-97``) and write ``output_array`` in place
  (``output_array[ia*iskipa + ib*iskipb]``).
* ``overlap_work_array_size`` / ``nuclear_work_array_size`` are the emitted
  ``..._work_array_size``.
* ``TwoIndexBatch`` evaluates many pairs on the device in one launch.

Every call goes to libintception_b200.so; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import eri as _eri

OVERLAP, NUCLEAR = 0, 1
_dp = C.POINTER(C.c_double)
_bound = []


def _lib():
    lib = _eri.load()
    if not _bound:
        pair = [C.c_double, _dp, C.c_int, C.c_int, C.c_int] * 2
        lib.intception_integral_overlap_2idx_ab_prim_cart_main.argtypes = pair + [_dp, _dp]
        lib.intception_integral_overlap_2idx_ab_prim_cart_main.restype = None
        lib.intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main.argtypes = pair + [_dp, _dp, _dp]
        lib.intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main.restype = None
        for f in (lib.intception_integral_overlap_2idx_ab_prim_cart_work_array_size,
                  lib.intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size):
            f.argtypes = [C.c_int, C.c_int]
            f.restype = C.c_int
        lib.intception_b200_twoidx_batch.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 11
        lib.intception_b200_twoidx_batch.restype = C.c_int
        lib.intception_b200_twoidx_test_stall.argtypes = [C.c_longlong, C.c_int]
        lib.intception_b200_twoidx_test_stall.restype = C.c_int
        _bound.append(True)
    return lib


def ncart(l):
    return (l + 1) * (l + 2) // 2


def overlap_work_array_size(la, lb):
    return _lib().intception_integral_overlap_2idx_ab_prim_cart_work_array_size(la, lb)


def nuclear_work_array_size(la, lb):
    return _lib().intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size(la, lb)


def _vec3(v):
    a = np.ascontiguousarray(v, dtype=np.float64)
    if a.shape != (3,):
        raise _eri.IntceptionError('centres are 3-vectors')
    return a


def _out(output_array):
    if output_array.dtype != np.float64 or not output_array.flags['C_CONTIGUOUS']:
        raise _eri.IntceptionError('output_array must be a contiguous float64 array')
    return output_array.ctypes.data_as(_dp)


def overlap_main(xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, output_array, work_array=None):
    """Drop-in for intception_integral_overlap_2idx_ab_prim_cart_main."""
    A, B = _vec3(cA), _vec3(cB)
    wa = work_array if work_array is not None else np.zeros(1)
    _lib().intception_integral_overlap_2idx_ab_prim_cart_main(
        float(xa), A.ctypes.data_as(_dp), la, na, iskipa, float(xb), B.ctypes.data_as(_dp), lb, nb, iskipb,
        wa.ctypes.data_as(_dp), _out(output_array))
    _eri._check()


def nuclear_main(xa, cA, la, na, iskipa, xb, cB, lb, nb, iskipb, cC, output_array, work_array=None):
    """Drop-in for intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main."""
    A, B, Cc = _vec3(cA), _vec3(cB), _vec3(cC)
    wa = work_array if work_array is not None else np.zeros(1)
    _lib().intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main(
        float(xa), A.ctypes.data_as(_dp), la, na, iskipa, float(xb), B.ctypes.data_as(_dp), lb, nb, iskipb,
        Cc.ctypes.data_as(_dp), wa.ctypes.data_as(_dp), _out(output_array))
    _eri._check()


def block_offsets(la, lb):
    """Packed per-pair block offsets (a fastest) and the total size."""
    la = np.asarray(la, dtype=np.int64)
    lb = np.asarray(lb, dtype=np.int64)
    sizes = ((la + 1) * (la + 2) // 2) * ((lb + 1) * (lb + 2) // 2)
    off = np.zeros(len(sizes), dtype=np.int64)
    if len(sizes) > 1:
        np.cumsum(sizes[:-1], out=off[1:])
    return off, int(sizes.sum())


class TwoIndexBatch:
    """A pair set resident on the device (torch tensors hold the memory).

    pairs: dict of host arrays xa[n], ca[n,3] (or 3n), la[n], xb[n], cb, lb[n],
    cc (charge positions; needed for nuclear) and optionally off[n] / size
    (block offsets, a fastest; default packed)."""

    def __init__(self, pairs, device='cuda'):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(self.device)  # noqa: E731
        la, lb = np.asarray(pairs['la']), np.asarray(pairs['lb'])
        self.n = len(la)
        off, size = (pairs['off'], int(pairs['size'])) if 'off' in pairs else block_offsets(la, lb)
        self.size = size
        self.lmax = int(max(la.max(), lb.max())) if self.n else 0
        self.xa = t(pairs['xa'], torch.float64)
        self.ca = t(np.asarray(pairs['ca']).reshape(-1), torch.float64)
        self.la = t(la, torch.int32)
        self.xb = t(pairs['xb'], torch.float64)
        self.cb = t(np.asarray(pairs['cb']).reshape(-1), torch.float64)
        self.lb = t(lb, torch.int32)
        cc = pairs.get('cc')
        self.cc = t(np.asarray(cc).reshape(-1), torch.float64) if cc is not None else None
        self.off = t(off, torch.int64)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib()

    def compute(self, kind, out=None, stream=None, lmax=None):
        """Blocks of every pair for kind OVERLAP or NUCLEAR into out (float64,
        device); returns out.  Asynchronous on stream; device_status() reports
        pairs the kernels refused."""
        torch = self.torch
        if out is None:
            out = torch.empty(self.size, dtype=torch.float64, device=self.device)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        cc = self.cc.data_ptr() if self.cc is not None else None
        st = _lib().intception_b200_twoidx_batch(
            int(kind), self.n, self.lmax if lmax is None else int(lmax), self.xa.data_ptr(), self.ca.data_ptr(),
            self.la.data_ptr(), self.xb.data_ptr(), self.cb.data_ptr(), self.lb.data_ptr(), cc, self.off.data_ptr(),
            out.data_ptr(), self.status.data_ptr(), C.c_void_p(s.cuda_stream))
        _eri._check(st)
        return out

    def device_status(self):
        """The device status word (0 = every pair evaluated); synchronises."""
        return int(self.status.item())


def make_pairs(n, lmax=2, seed=1, box=30.0):
    """Synthetic pair set: la, lb uniform in 0..lmax, exponents log-uniform in
    [0.05, 1e4], A uniform in a box, B and the charge C within 2 bohr of A
    (pairs and charges near each other, as in a molecule)."""
    rng = np.random.default_rng(seed)
    la = rng.integers(0, lmax + 1, n).astype(np.int32)
    lb = rng.integers(0, lmax + 1, n).astype(np.int32)
    xa = np.exp(rng.uniform(np.log(0.05), np.log(1e4), n))
    xb = np.exp(rng.uniform(np.log(0.05), np.log(1e4), n))
    ca = rng.uniform(0.0, box, (n, 3))
    cb = ca + rng.uniform(-2.0, 2.0, (n, 3))
    cc = ca + rng.uniform(-2.0, 2.0, (n, 3))
    return dict(xa=xa, ca=ca, la=la, xb=xb, cb=cb, lb=lb, cc=cc)


def algorithmic_cost(kind, la, lb):
    """(FP64 flops, bytes) per pair of the recurrences as the kernels run them:
    nuclear -- VRR entries (3 flops, 7 with the two-back term), HRR entries
    (2), Boys (Taylor, downward recursion) and setup; overlap -- the three 1D
    tables and 3 multiplies per output.  Bytes: the pair's inputs and its
    output block."""
    na, nb = ncart(la), ncart(lb)
    nbytes = 8 * na * nb + 8 * 2 + 8 * 6 + 4 * 2 + 8 + (24 if kind == NUCLEAR else 0)
    if kind == OVERLAP:
        return 3 * 5 * (la + 1) * (lb + 1) + 3 * na * nb + 30, nbytes
    hi, lo = max(la, lb), min(la, lb)
    L = hi + lo
    flops = 40 + 14 + 3 * L + (L + 1)
    for n in range(1, L + 1):
        for k in range(ncart(n)):
            s = 0
            while (s + 1) * (s + 2) // 2 <= k:
                s += 1
            z = k - s * (s + 1) // 2
            e = (n - s, s - z, z)
            ei = next(v for v in e if v > 0)
            flops += (L - n + 1) * (7 if ei >= 2 else 3)
    ncum = lambda l: (l + 1) * (l + 2) * (l + 3) // 6  # noqa: E731
    for j in range(1, lo + 1):
        flops += 2 * (ncum(L - j) - ncum(hi - 1)) * ncart(j)
    return flops, nbytes
