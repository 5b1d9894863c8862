"""Python host layer over libintception_b200.so (ctypes).

Mirrors the reference's interface for the ERI path:

* ``cont_cart_main`` / ``cont_sph_main`` take the argument list of the
  generated ``intception_integral_eri_abcd_m_cont_{cart,sph}_main``
  (``contracted_general.py:42-68``), as numpy arrays, and write
  ``output_array`` in place.  They return None like the C functions; a failed
  call raises ``IntceptionError`` with the library's message.
* ``work_array_size`` is the emitted ``..._work_array_size``.
* ``boys`` is the emitted ``intception_boys``.
* ``EriEngine`` is the batched device path (torch tensors as device memory).

The CUDA library is required: importing works without it, but every call
raises if ``libintception_b200.so`` is missing or no GPU is present.  There is
no CPU fallback.
"""
import ctypes as C
import os
import re

import numpy as np

from . import basis as _basis

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, 'libintception_b200.so')
HEADER = os.path.join(os.path.dirname(PKG), 'include', 'intception_b200.h')

IB_OK, IB_ERR_ARG, IB_ERR_CUDA, IB_ERR_SCRATCH, IB_ERR_NODEVICE, IB_ERR_TIMEOUT = 0, 1, 2, 3, 4, 5
PREC_FP64, PREC_MIXED = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class IntceptionError(RuntimeError):
    pass


class _Basis(C.Structure):
    _fields_ = [('shell_l', C.c_void_p), ('shell_k', C.c_void_p), ('shell_ptr', C.c_void_p),
                ('shell_xyz', C.c_void_p), ('prim_exp', C.c_void_p), ('prim_coef', C.c_void_p),
                ('nshell', C.c_int), ('nprim', C.c_int), ('lmax', C.c_int)]


def header_functions(path=HEADER):
    """Names of every function the public header declares."""
    text = open(path).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    names = re.findall(r'^\s*(?:const\s+)?(?:void|int|char|double)\s*\**\s*(\w+)\s*\(', text, flags=re.M)
    return sorted(set(names))


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise IntceptionError('libintception_b200.so not built: run python -m intception_b200.build')
    lib = C.CDLL(LIB_PATH)
    idx = [C.c_int] * 6
    per_cart = [_dp, _dp] + idx + [_dp]
    per_sph = per_cart + [_dp]
    lib.intception_integral_eri_abcd_m_cont_cart_main.argtypes = per_cart * 4 + [_dp, _dp]
    lib.intception_integral_eri_abcd_m_cont_cart_main.restype = None
    lib.intception_integral_eri_abcd_m_cont_sph_main.argtypes = per_sph * 4 + [_dp, _dp]
    lib.intception_integral_eri_abcd_m_cont_sph_main.restype = None
    for v in ('cart', 'sph'):
        f = getattr(lib, 'intception_integral_eri_abcd_m_cont_%s_work_array_size' % v)
        f.argtypes = [C.c_int] * 12
        f.restype = C.c_int
    lib.intception_boys.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double]
    lib.intception_boys.restype = None
    lib.intception_b200_last_status.restype = C.c_int
    lib.intception_b200_last_error.restype = C.c_char_p
    lib.intception_b200_lmax.restype = C.c_int
    lib.intception_b200_last_launch_count.restype = C.c_int
    lib.intception_b200_sph_matrix.argtypes = [C.c_int, _dp]
    lib.intception_b200_sph_matrix.restype = C.c_int
    lib.intception_b200_boys_batch.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.intception_b200_boys_batch.restype = C.c_int
    lib.intception_b200_synchronize.restype = C.c_int
    lib.intception_b200_batch_status.restype = C.c_int
    lib.intception_b200_last_fp32_rejections.restype = C.c_int
    lib.intception_b200_eri_batch.argtypes = [C.POINTER(_Basis), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                              C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                              C.c_void_p]
    lib.intception_b200_eri_batch.restype = C.c_int
    lib.intception_b200_schwarz.argtypes = [C.POINTER(_Basis), C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                            C.c_void_p]
    lib.intception_b200_schwarz.restype = C.c_int
    lib.intception_b200_quartet_bounds.argtypes = [C.POINTER(_Basis), C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                   C.c_void_p]
    lib.intception_b200_quartet_bounds.restype = C.c_int
    lib.intception_b200_eri_graph_create.argtypes = [C.POINTER(_Basis), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                     C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                                     C.c_void_p, C.POINTER(C.c_void_p)]
    lib.intception_b200_eri_graph_create.restype = C.c_int
    lib.intception_b200_eri_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    lib.intception_b200_eri_graph_launch.restype = C.c_int
    lib.intception_b200_eri_graph_destroy.argtypes = [C.c_void_p]
    lib.intception_b200_eri_graph_destroy.restype = C.c_int
    lib.intception_b200_eri_batch_noalloc.argtypes = [C.POINTER(_Basis), C.c_void_p, C.c_void_p, C.c_int,
                                                      C.c_int, C.c_void_p, C.c_void_p]
    lib.intception_b200_eri_batch_noalloc.restype = C.c_int
    lib.intception_b200_noalloc_status.argtypes = [C.c_void_p]
    lib.intception_b200_noalloc_status.restype = C.c_int
    lib.intception_b200_fma_peak.argtypes = [C.c_int, C.c_int, _dp]
    lib.intception_b200_fma_peak.restype = C.c_int
    lib.intception_b200_set_slice_cap.argtypes = [C.c_int, C.c_int]
    lib.intception_b200_set_slice_cap.restype = C.c_int
    lib.intception_b200_set_prim_tol.argtypes = [C.c_double]
    lib.intception_b200_set_prim_tol.restype = C.c_int
    lib.intception_b200_set_hrr_tol.argtypes = [C.c_double]
    lib.intception_b200_set_hrr_tol.restype = C.c_int
    lib.intception_b200_last_hrr_redo.argtypes = []
    lib.intception_b200_last_hrr_redo.restype = C.c_int
    lib.intception_b200_generic_grid.argtypes = [C.c_int]
    lib.intception_b200_generic_grid.restype = C.c_int
    lib.intception_b200_set_class_minb.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.intception_b200_set_class_minb.restype = C.c_int
    lib.intception_b200_set_class_fp32.argtypes = [C.c_int, C.c_int]
    lib.intception_b200_set_class_fp32.restype = C.c_int
    _lib = lib
    return lib


def _check(status=None):
    lib = load()
    st = lib.intception_b200_last_status() if status is None else status
    if st != IB_OK:
        raise IntceptionError('intception_b200 status %d: %s' % (st, lib.intception_b200_last_error().decode()))


def lmax():
    return load().intception_b200_lmax()


def fma_peak(fp64=True, iters=4096):
    """Measured FMA throughput of the current device (FLOP/s)."""
    v = C.c_double(0.0)
    _check(load().intception_b200_fma_peak(1 if fp64 else 0, iters, C.byref(v)))
    return v.value


def class_id(la, lb, lc, ld):
    """Canonical class id of (la lb|lc ld): la >= lb, lc >= ld, bra pair >= ket
    pair (the id the batch kernels are registered under)."""
    if la < lb:
        la, lb = lb, la
    if lc < ld:
        lc, ld = ld, lc
    pb, pk = la * (la + 1) // 2 + lb, lc * (lc + 1) // 2 + ld
    if pb < pk:
        pb, pk = pk, pb
    return pb * (pb + 1) // 2 + pk


def set_slice_cap(cap, cls=None):
    """At most cap lane groups (power of two, 0 = no cap) share one quartet
    in the class kernels: every class, or the canonical class (la,lb,lc,ld)."""
    cid = -1 if cls is None else class_id(*cls)
    _check(load().intception_b200_set_slice_cap(cid, int(cap)))


def set_prim_tol(tol):
    """Primitive screening in the batch path (EriEngine.compute, graphs):
    primitive quartets whose Coulomb-norm bound Q_ab Q_cd is below tol are
    skipped, so an element moves by at most Ka Kb Kc Kd * tol; 0 (default)
    skips only exact-zero prefactors.  The drop-ins never screen."""
    _check(load().intception_b200_set_prim_tol(float(tol)))


def set_hrr_tol(tol):
    """Tolerance of the class kernels' HRR rounding-error estimate (output
    units; default 1e-13, 0 = no check): quartets over it are recomputed by
    the generic kernel with every primitive pair built on the shell that
    conditions its HRR."""
    _check(load().intception_b200_set_hrr_tol(float(tol)))


def last_hrr_redo():
    """Quartets of the last batch the generic kernel recomputed for the HRR
    check (waits for the device)."""
    return load().intception_b200_last_hrr_redo()


def generic_grid(cluster_size):
    """Blocks of the generic kernel's launch with heavy quartets split over
    clusters of cluster_size blocks (1: no clusters) on the current device."""
    return load().intception_b200_generic_grid(int(cluster_size))


def set_class_minb(cls, variant, minb):
    """Register budget of canonical class cls = (la,lb,lc,ld) for variant
    0..3 (FP64 cart, FP64 sph, FP32 cart, FP32 sph): the kernel compiled for
    minb in (1, 3, 4, 5) resident blocks per SM; 0 restores the default."""
    _check(load().intception_b200_set_class_minb(class_id(*cls), int(variant), int(minb)))


def set_class_fp32(on, cls=None):
    """Whether the FP32 tier runs the FP32 kernel of class cls (every class
    when None): True, False, or None for the built-in default."""
    cid = -1 if cls is None else class_id(*cls)
    _check(load().intception_b200_set_class_fp32(cid, -1 if on is None else int(bool(on))))


def sph_matrix(l):
    """The library's ncart x (2l+1) matrix (T[icart + isph*ncart])."""
    nc = (l + 1) * (l + 2) // 2
    T = np.zeros(nc * (2 * l + 1))
    _check(load().intception_b200_sph_matrix(l, T.ctypes.data_as(_dp)))
    return T.reshape((nc, 2 * l + 1), order='F')


def work_array_size(la, lb, lc, ld, na_prim, nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont,
                    spherical=False):
    f = getattr(load(), 'intception_integral_eri_abcd_m_cont_%s_work_array_size' % ('sph' if spherical else 'cart'))
    return f(la, lb, lc, ld, na_prim, nb_prim, nc_prim, nd_prim, na_cont, nb_cont, nc_cont, nd_cont)


def _main(variant, shells, work_array, output_array):
    lib = load()
    fn = getattr(lib, 'intception_integral_eri_abcd_m_cont_%s_main' % variant)
    args, keep = [], []
    for s in shells:
        x = np.ascontiguousarray(s['x'], dtype=np.float64)
        cen = np.ascontiguousarray(s['cen'], dtype=np.float64)
        coef = np.ascontiguousarray(s['coef'], dtype=np.float64)
        keep += [x, cen, coef]
        args += [x.ctypes.data_as(_dp), cen.ctypes.data_as(_dp), s['l'], s['n'], s['iskip'], s['nprim'],
                 s['ncont'], s['iskip_cont'], coef.ctypes.data_as(_dp)]
        if variant == 'sph':
            T = np.ascontiguousarray(np.asarray(s['T'], dtype=np.float64).ravel(order='F'))
            keep.append(T)
            args.append(T.ctypes.data_as(_dp))
    if output_array.dtype != np.float64 or not output_array.flags['C_CONTIGUOUS']:
        raise IntceptionError('output_array must be a contiguous float64 array')
    wa = work_array if work_array is not None else np.zeros(1)
    fn(*args, wa.ctypes.data_as(_dp), output_array.ctypes.data_as(_dp))
    _check()


def cont_cart_main(shells, output_array, work_array=None):
    """Drop-in for intception_integral_eri_abcd_m_cont_cart_main.  shells is
    four dicts (a, b, c, d) with keys x, cen, l, n, iskip, nprim, ncont,
    iskip_cont, coef (the emitted per-index arguments, wrappers.py:41-143)."""
    _main('cart', shells, work_array, output_array)


def cont_sph_main(shells, output_array, work_array=None):
    """Drop-in for intception_integral_eri_abcd_m_cont_sph_main (dicts also
    carry T = sph_trans_array_?, ncart x nsph)."""
    _main('sph', shells, work_array, output_array)


def boys(nmax, x, nmin=0, ifskip=1):
    """Drop-in for intception_boys: F_m(x), m = nmin..nmax (array of nmax+1)."""
    f = np.zeros((nmax + 1) * ifskip)
    load().intception_boys(f.ctypes.data_as(_dp), ifskip, nmin, nmax, float(x))
    _check()
    return f[::ifskip]


class EriEngine:
    """Batched contracted ERIs on the current CUDA device.

    The shell table is uploaded once (torch tensors hold the device memory);
    ``compute`` evaluates a quartet list into a flat output vector laid out
    per quartet with a fastest (``basis.ShellBatch`` conventions).
    """

    def __init__(self, batch, device='cuda'):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        b = batch
        self.spherical = bool(b.spherical)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(self.device)  # noqa: E731
        self.shell_l = t(b.shell_l, torch.int32)
        self.shell_k = t(b.shell_k, torch.int32)
        self.shell_ptr = t(b.shell_ptr, torch.int32)
        self.shell_xyz = t(b.shell_xyz, torch.float64)
        self.prim_exp = t(b.prim_exp, torch.float64)
        self.prim_coef = t(b.prim_coef, torch.float64)
        self.lmax = int(b.shell_l.max()) if len(b.shell_l) else 0
        self._basis = _Basis(self.shell_l.data_ptr(), self.shell_k.data_ptr(), self.shell_ptr.data_ptr(),
                             self.shell_xyz.data_ptr(), self.prim_exp.data_ptr(), self.prim_coef.data_ptr(),
                             len(b.shell_l), len(b.prim_exp), self.lmax)
        self.quartets = t(b.quartets.reshape(-1), torch.int32)
        self.out_off = t(b.out_off, torch.int64)
        self.nq = b.nq
        self.out_size = b.out_size
        load()

    def compute(self, out=None, precision=PREC_FP64, bounds=None, skip_below=0.0, fp32_below=0.0, mixed_tol=5e-11,
                stream=None, quartets=None, out_off=None, nq=None):
        """Evaluate the quartet list (or the given one) into out.  bounds: per
        quartet |(ab|cd)| upper bounds (torch float64, device); quartets below
        skip_below are written as zeros; with PREC_MIXED those below
        fp32_below use the FP32 VRR, and any whose FP32 error bound exceeds
        mixed_tol is recomputed in FP64."""
        torch = self.torch
        if out is None:
            out = torch.empty(self.out_size, dtype=torch.float64, device=self.device)
        q = self.quartets if quartets is None else quartets
        o = self.out_off if out_off is None else out_off
        n = self.nq if nq is None else nq
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = load().intception_b200_eri_batch(
            C.byref(self._basis), q.data_ptr(), o.data_ptr(), n, 1 if self.spherical else 0, precision,
            bounds.data_ptr() if bounds is not None else None, float(skip_below), float(fp32_below), float(mixed_tol),
            out.data_ptr(), C.c_void_p(s.cuda_stream))
        _check(st)
        return out

    def graph(self, out, precision=PREC_FP64, bounds=None, skip_below=0.0, fp32_below=0.0, mixed_tol=5e-11):
        """CUDA graph replaying compute(out=out, ...) with one launch; returns
        an EriGraph (call .launch(stream), .close())."""
        h = C.c_void_p()
        _check(load().intception_b200_eri_graph_create(
            C.byref(self._basis), self.quartets.data_ptr(), self.out_off.data_ptr(), self.nq,
            1 if self.spherical else 0, precision, bounds.data_ptr() if bounds is not None else None,
            float(skip_below), float(fp32_below), float(mixed_tol), out.data_ptr(), C.byref(h)))
        return EriGraph(h, self)

    def schwarz(self, pairs, stream=None):
        """sqrt(max |(ij|ij)|) for shell pairs (torch int32 [n, 2], device)."""
        torch = self.torch
        pairs = pairs.contiguous()
        q = torch.empty(pairs.shape[0], dtype=torch.float64, device=self.device)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _check(load().intception_b200_schwarz(C.byref(self._basis), pairs.data_ptr(), pairs.shape[0],
                                              1 if self.spherical else 0, q.data_ptr(), C.c_void_p(s.cuda_stream)))
        return q

    def quartet_bounds(self, stream=None):
        """Schwarz bound of every quartet of the batch: q_ab * q_cd."""
        torch = self.torch
        qv = self.quartets.view(-1, 4)
        pairs = torch.cat([qv[:, 0:2], qv[:, 2:4]]).contiguous()
        q = self.schwarz(pairs, stream)
        return (q[:self.nq] * q[self.nq:]).contiguous()

    def analytic_bounds(self, out=None, stream=None, quartets=None, nq=None):
        """Per-quartet analytic screening bounds (intception_b200_quartet_bounds):
        no ERI evaluated, one pass over the primitive pairs."""
        torch = self.torch
        q = self.quartets if quartets is None else quartets
        n = self.nq if nq is None else nq
        if out is None:
            out = torch.empty(n, dtype=torch.float64, device=self.device)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _check(load().intception_b200_quartet_bounds(C.byref(self._basis), q.data_ptr(), n,
                                                     1 if self.spherical else 0, out.data_ptr(),
                                                     C.c_void_p(s.cuda_stream)))
        return out

    @staticmethod
    def last_launch_count():
        return load().intception_b200_last_launch_count()

    @staticmethod
    def fp32_rejected():
        return load().intception_b200_last_fp32_rejections()

    @staticmethod
    def device_status():
        return load().intception_b200_batch_status()


class HostPipeline:
    """Batches held in pinned host memory, streamed through the current GPU with
    the copies overlapped: while batch i is evaluated, the inputs of batch i+1
    go up and the blocks of batch i-1 come down (``depth`` device buffer sets,
    one stream per direction, events between them; the evaluations themselves
    run one after another on one stream, as they share the library's work
    buffers).  ``submit`` returns once the batch is queued; the host output of a
    batch is valid after ``synchronize`` (or ``wait``) covers it.

    A batch is a dict of pinned host tensors: shell_l, shell_k, shell_ptr
    (int32), shell_xyz, prim_exp, prim_coef (float64), quartets (int32, 4 per
    quartet), out_off (int64), and with screening bounds (float64), laid out as
    ``basis.ShellBatch``.
    """

    INPUTS = ('shell_l', 'shell_k', 'shell_ptr', 'shell_xyz', 'prim_exp', 'prim_coef', 'quartets', 'out_off',
              'bounds')

    def __init__(self, spherical, depth=2, device='cuda'):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.spherical = bool(spherical)
        self.depth = int(depth)
        self.s_in = torch.cuda.Stream(self.device)
        self.s_run = torch.cuda.Stream(self.device)
        self.s_out = torch.cuda.Stream(self.device)
        self.slots = [{'buf': {}, 'ev': {}, 'used': set()} for _ in range(self.depth)]
        self.k = 0
        load()

    def _buffer(self, slot, name, like, n):
        b = slot['buf'].get(name)
        if b is None or b.numel() < n:
            b = self.torch.empty(max(n, 1), dtype=like.dtype, device=self.device)
            slot['buf'][name] = b
        return b

    def _event(self, slot, name):
        ev = slot['ev'].get(name)
        if ev is None:
            ev = slot['ev'][name] = self.torch.cuda.Event()
        return ev

    def _wait(self, stream, slot, name):
        if name in slot['used']:
            stream.wait_event(slot['ev'][name])

    def submit(self, h, out_host, precision=PREC_FP64, skip_below=0.0, fp32_below=0.0, mixed_tol=5e-11, lmax=None):
        """Queue one batch; out_host (pinned float64) receives its blocks.  As
        for the out argument of intception_b200_eri_batch, out_host must hold
        every block of the batch: out_off[q] + na nb nc nd <= out_host.numel()
        for every quartet q (the device buffer is sized from it and the
        kernels write each block at its offset).  lmax: the largest shell l
        (computed from shell_l when None).  Screening (skip_below > 0) and
        PREC_MIXED use h['bounds'] when given, else the analytic bounds
        (intception_b200_quartet_bounds) computed on the device with the batch."""
        torch = self.torch
        slot = self.slots[self.k % self.depth]
        self.k += 1
        nq = h['quartets'].numel() // 4
        nout = out_host.numel()
        if lmax is None:
            lmax = int(h['shell_l'].max()) if h['shell_l'].numel() else 0
        names = [n for n in self.INPUTS if h.get(n) is not None]
        # inputs up, once the slot's previous evaluation has read its inputs
        self._wait(self.s_in, slot, 'run')
        d = {}
        with torch.cuda.stream(self.s_in):
            for n in names:
                src = h[n].reshape(-1)
                d[n] = self._buffer(slot, n, src, src.numel())
                d[n][:src.numel()].copy_(src, non_blocking=True)
        self._event(slot, 'in').record(self.s_in)
        slot['used'].add('in')
        out = self._buffer(slot, 'out', out_host, nout)
        # evaluation, once the inputs are up and the slot's previous blocks are down
        self.s_run.wait_event(slot['ev']['in'])
        self._wait(self.s_run, slot, 'down')
        bas = _Basis(d['shell_l'].data_ptr(), d['shell_k'].data_ptr(), d['shell_ptr'].data_ptr(),
                     d['shell_xyz'].data_ptr(), d['prim_exp'].data_ptr(), d['prim_coef'].data_ptr(),
                     h['shell_l'].numel(), h['prim_exp'].numel(), lmax)
        if 'bounds' not in d and (skip_below > 0.0 or precision == PREC_MIXED):
            d['bounds'] = self._buffer(slot, 'bounds_dev', h['shell_xyz'], nq)
            _check(load().intception_b200_quartet_bounds(C.byref(bas), d['quartets'].data_ptr(), nq,
                                                         1 if self.spherical else 0, d['bounds'].data_ptr(),
                                                         C.c_void_p(self.s_run.cuda_stream)))
        st = load().intception_b200_eri_batch(
            C.byref(bas), d['quartets'].data_ptr(), d['out_off'].data_ptr(), nq, 1 if self.spherical else 0,
            precision, d['bounds'].data_ptr() if 'bounds' in d else None, float(skip_below), float(fp32_below),
            float(mixed_tol), out.data_ptr(), C.c_void_p(self.s_run.cuda_stream))
        _check(st)
        self._event(slot, 'run').record(self.s_run)
        slot['used'].add('run')
        # blocks down
        self.s_out.wait_event(slot['ev']['run'])
        with torch.cuda.stream(self.s_out):
            out_host.reshape(-1)[:nout].copy_(out[:nout], non_blocking=True)
        self._event(slot, 'down').record(self.s_out)
        slot['used'].add('down')

    def wait_event(self):
        """A CUDA event recorded after every queued copy-out (for timing)."""
        ev = self.torch.cuda.Event(enable_timing=True)
        ev.record(self.s_out)
        return ev

    def synchronize(self):
        self.s_out.synchronize()
        self.s_run.synchronize()
        self.s_in.synchronize()


class EriGraph:
    """A captured batch (intception_b200_eri_graph_*)."""

    def __init__(self, handle, engine):
        self.h = handle
        self.engine = engine  # keeps the device inputs alive

    def launch(self, stream=None):
        torch = self.engine.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.engine.device)
        _check(load().intception_b200_eri_graph_launch(self.h, C.c_void_p(s.cuda_stream)))

    def close(self):
        if self.h:
            load().intception_b200_eri_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_reference_layout(batch):
    """List of (offset, dims) per quartet, the layout ``compute`` writes."""
    return [(int(batch.out_off[q]), batch.block_dims(q)) for q in range(batch.nq)]


__all__ = ['IntceptionError', 'load', 'lmax', 'sph_matrix', 'work_array_size', 'cont_cart_main', 'cont_sph_main',
           'boys', 'EriEngine', 'header_functions', '_basis', 'class_id', 'set_slice_cap', 'set_class_minb', 'set_class_fp32', 'HostPipeline']
