"""J/K energies of a density and their nuclear gradient, on the GPU.

    E_J = 1/2 sum_ijkl P_ij P_kl (ij|kl)        E_K = -1/4 sum_ijkl P_ik P_jl (ij|kl)

over real normalised basis functions, with a fixed symmetric density P given
in the spherical basis (m = -l..l, the library's matrices) and transformed to
the Cartesian one (P_cart = T P T^T), so the digestion runs on Cartesian ERI
blocks.  Unique shell quartets (8-fold symmetry) are screened with Schwarz
factors (q_ab q_cd >= screen), evaluated by the batch path in chunks and
digested by ``intception_b200_jk_energy``.

The gradient is the adjoint of the same evaluation: for each of the first
three centres of every quartet the ERI kernels evaluate auxiliary blocks with
that index raised (coefficients 2 alpha c, l+1) and lowered (l-1), and
``intception_b200_jk_force`` maps their elements back onto the components they
differentiate, accumulating atom forces; the fourth centre follows from
translational invariance.  Nothing from the forward pass is stored: backward
recomputes every integral it needs.

Several GPUs (one process each, torch.distributed initialised): every rank
enumerates the same screened quartet chunks and digests every world-th quartet
of each chunk (rank, rank + world, ...: neighbouring quartets cost about the
same, so the shares balance); the partial E_J, E_K and the partial force array
are then summed by one all_reduce each.  No quartet block crosses a GPU.
"""
import ctypes as C

import numpy as np

from . import basis as B
from . import eri


def _lib():
    lib = eri.load()
    if not getattr(lib, '_jk_ready', False):
        lib.intception_b200_jk_energy.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.intception_b200_jk_energy.restype = C.c_int
        lib.intception_b200_jk_force.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]
        lib.intception_b200_jk_force.restype = C.c_int
        lib.intception_b200_jk_force_all.argtypes = [C.c_void_p, C.c_int, C.c_void_p * 6, C.c_void_p * 6,
                                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                     C.c_int, C.c_void_p, C.c_void_p]
        lib.intception_b200_jk_force_all.restype = C.c_int
        lib._jk_ready = True
    return lib


class JKSystem:
    """Atoms, shells and a density; energy(xyz) and gradient(xyz) on the GPU.

    atom_xyz [natom,3] (bohr); shell_atom/shell_l/shell_k [nshell];
    prim_exp/prim_coef [nprim] (normalised coefficients, shells contiguous);
    P_sph [nbf,nbf] symmetric, spherical functions in shell order.
    """

    def __init__(self, atom_xyz, shell_atom, shell_l, shell_k, prim_exp, prim_coef, P_sph, device='cuda',
                 screen=1e-15, chunk=1 << 21, rank=None, world=None, group=None, reduce=True):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.screen = float(screen)
        self.chunk = int(chunk)
        # quartet shard of this process: rank r of world digests quartets r, r + world, ... of every chunk
        dist_on = torch.distributed.is_available() and torch.distributed.is_initialized()
        self.rank = int(rank if rank is not None else (torch.distributed.get_rank(group) if dist_on else 0))
        self.world = int(world if world is not None else (torch.distributed.get_world_size(group) if dist_on else 1))
        self.group = group
        self.reduce = bool(reduce) and self.world > 1  # False: return this rank's partial sums
        # split of the device time between the ERI batches and the digestion
        # kernels (CUDA events around each; read with kernel_split())
        self.profile = False
        self._marks = []
        # gradient digestion: False = one pass over the six auxiliary batches of
        # a chunk (their blocks held together); True = one launch per batch
        self.per_batch_digestion = False
        l = np.asarray(shell_l, np.int32)
        k = np.asarray(shell_k, np.int32)
        e = np.asarray(prim_exp, np.float64)
        c = np.asarray(prim_coef, np.float64)
        ns, npr = len(l), len(e)
        ptr = np.zeros(ns, np.int32)
        ptr[1:] = np.cumsum(k)[:-1]
        self.ns = ns
        self.natom = int(np.asarray(atom_xyz).shape[0])
        self.shell_atom_np = np.asarray(shell_atom, np.int32)
        nc = (l + 1) * (l + 2) // 2
        self.fofs_np = np.concatenate([[0], np.cumsum(nc)[:-1]]).astype(np.int32)
        self.nbf_cart = int(nc.sum())
        nsph = 2 * l + 1
        sofs = np.concatenate([[0], np.cumsum(nsph)[:-1]])
        T = np.zeros((self.nbf_cart, int(nsph.sum())))
        for s in range(ns):
            T[self.fofs_np[s]:self.fofs_np[s] + nc[s], sofs[s]:sofs[s] + nsph[s]] = B.sph_matrix(int(l[s]))
        P_cart = T @ np.asarray(P_sph, np.float64) @ T.T
        # shells 0..ns-1 original, ns..2ns-1 raised (l+1, 2 alpha c), 2ns..3ns-1 lowered (l-1)
        e_all = np.concatenate([e, e, e])
        expand = np.repeat(np.arange(ns), k)
        c_low = np.where(l[expand] >= 1, c, 0.0)
        c_all = np.concatenate([c, 2.0 * e * c, c_low])
        l_all = np.concatenate([l, l + 1, np.maximum(l - 1, 0)]).astype(np.int32)
        k_all = np.concatenate([k, k, k]).astype(np.int32)
        ptr_all = np.concatenate([ptr, ptr + npr, ptr + 2 * npr]).astype(np.int32)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.dev)  # noqa: E731
        self.shell_l = t(l_all, torch.int32)
        self.shell_k = t(k_all, torch.int32)
        self.shell_ptr = t(ptr_all, torch.int32)
        self.prim_exp = t(e_all, torch.float64)
        self.prim_coef = t(c_all, torch.float64)
        self.shell_atom = t(np.concatenate([self.shell_atom_np] * 3), torch.int32)
        self.fofs = t(self.fofs_np, torch.int32)
        self.P = t(P_cart, torch.float64)
        self.shell_xyz = torch.zeros((3 * ns, 3), dtype=torch.float64, device=self.dev)
        self.lmax = int(l.max())
        self.ncart_dev = t(((l_all + 1) * (l_all + 2) // 2).astype(np.int64), torch.int64)
        a, b = np.tril_indices(ns)
        self.pairs = t(np.stack([a, b], axis=1).astype(np.int32), torch.int32)
        self.set_geometry(atom_xyz)

    # ------------------------------------------------------------------ plumbing
    def set_geometry(self, xyz):
        torch = self.torch
        x = torch.as_tensor(xyz, dtype=torch.float64, device=self.dev).reshape(self.natom, 3)
        self.shell_xyz.copy_(x[self.shell_atom.long()])

    def _basis(self, lmax):
        return eri._Basis(self.shell_l.data_ptr(), self.shell_k.data_ptr(), self.shell_ptr.data_ptr(),
                          self.shell_xyz.data_ptr(), self.prim_exp.data_ptr(), self.prim_coef.data_ptr(),
                          3 * self.ns, self.prim_exp.numel(), lmax)

    def _eri(self, quartets, lmax):
        """Cartesian FP64 blocks of quartets [n,4] (device int32): (blocks, offsets)."""
        torch = self.torch
        n = quartets.shape[0]
        sizes = self.ncart_dev[quartets.long()].prod(dim=1)
        off = torch.zeros(n, dtype=torch.int64, device=self.dev)
        if n > 1:
            off[1:] = torch.cumsum(sizes, 0)[:-1]
        total = int(sizes.sum().item()) if n else 0
        out = torch.empty(max(total, 1), dtype=torch.float64, device=self.dev)
        b = self._basis(lmax)
        st = eri.load().intception_b200_eri_batch(C.byref(b), quartets.data_ptr(), off.data_ptr(), n, 0,
                                                  eri.PREC_FP64, None, 0.0, 0.0, 0.0, out.data_ptr(),
                                                  C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream))
        eri._check(st)
        return out, off

    def schwarz(self):
        torch = self.torch
        q = torch.empty(self.pairs.shape[0], dtype=torch.float64, device=self.dev)
        b = self._basis(self.lmax)
        eri._check(eri.load().intception_b200_schwarz(C.byref(b), self.pairs.data_ptr(), self.pairs.shape[0], 0,
                                                      q.data_ptr(),
                                                      C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)))
        return q

    def quartet_chunks(self):
        """Unique screened quartets (a>=b, c>=d, pair index ij >= kl in Schwarz
        order) in chunks of at most self.chunk, as device int32 [n,4]."""
        torch = self.torch
        q = self.schwarz()
        order = torch.argsort(q, descending=True)
        qs = q[order]
        pr = self.pairs[order]
        npair = qs.numel()
        # row i pairs with rows j <= i whose q_j >= screen / q_i (a prefix, q sorted)
        lim = self.screen / torch.clamp(qs, min=1e-300)
        cnt = torch.searchsorted(-qs, -lim, right=True)  # number of j with q_j >= lim
        m = torch.minimum(cnt, torch.arange(1, npair + 1, device=self.dev))
        m = torch.where(qs * qs[0] >= self.screen, m, torch.zeros_like(m))
        cm = torch.cumsum(m, 0)
        i0 = 0
        while i0 < npair:
            base = int(cm[i0 - 1].item()) if i0 else 0
            i1 = int(torch.searchsorted(cm, torch.tensor(base + self.chunk, device=self.dev), right=True).item())
            i1 = max(i1, i0 + 1)
            i1 = min(i1, npair)
            rows = torch.arange(i0, i1, device=self.dev)
            lens = m[i0:i1]
            if int(lens.sum().item()):
                ii = torch.repeat_interleave(rows, lens)
                start = torch.cumsum(lens, 0) - lens
                jj = torch.arange(int(lens.sum().item()), device=self.dev) - torch.repeat_interleave(start, lens)
                yield torch.cat([pr[ii], pr[jj]], dim=1).to(torch.int32).contiguous()
            i0 = i1

    # ------------------------------------------------------------------ shards
    def shard(self, qt):
        """This rank's quartets of a chunk: rows rank, rank + world, ..."""
        return qt if self.world == 1 else qt[self.rank::self.world].contiguous()

    def _sum_over_ranks(self, t):
        """One all_reduce (sum) of a partial result over the ranks."""
        if self.reduce:
            self.torch.distributed.all_reduce(t, op=self.torch.distributed.ReduceOp.SUM, group=self.group)
        return t

    # ------------------------------------------------------------------ energy
    def energy(self, xyz=None):
        """(E_J, E_K) at the geometry xyz [natom,3] (this rank's partial sums
        when the system was made with reduce=False)."""
        torch = self.torch
        if xyz is not None:
            self.set_geometry(xyz)
        e = torch.zeros(2, dtype=torch.float64, device=self.dev)
        for qt in self.quartet_chunks():
            qt = self.shard(qt)
            if qt.shape[0]:
                self._energy_chunk(qt, e)
        ej, ek = self._sum_over_ranks(e).tolist()
        return ej, ek

    def _mark(self):
        """A CUDA event on the current stream when profiling, else None."""
        if not self.profile:
            return None
        ev = self.torch.cuda.Event(enable_timing=True)
        ev.record()
        return ev

    def kernel_split(self):
        """(ms in ERI batches, ms in digestion kernels) since the last call,
        summed over the events recorded while self.profile was set."""
        self.torch.cuda.synchronize()
        t_eri = sum(a.elapsed_time(b) for a, b, _ in self._marks)
        t_dig = sum(b.elapsed_time(c) for _, b, c in self._marks)
        self._marks = []
        return t_eri, t_dig

    def _energy_chunk(self, qt, e):
        """Adds the J/K energies of the unique quartets qt [n,4] to e[0:2]."""
        m0 = self._mark()
        blocks, off = self._eri(qt, self.lmax)
        m1 = self._mark()
        eri._check(_lib().intception_b200_jk_energy(
            qt.data_ptr(), off.data_ptr(), qt.shape[0], self.shell_l.data_ptr(), self.fofs.data_ptr(),
            self.P.data_ptr(), self.nbf_cart, blocks.data_ptr(), e.data_ptr(),
            C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)))
        if m0 is not None:
            self._marks.append((m0, m1, self._mark()))

    def gradient(self, xyz=None):
        """dE/dR [natom,3] of E = E_J + E_K at xyz (FP64)."""
        torch = self.torch
        if xyz is not None:
            self.set_geometry(xyz)
        force = torch.zeros(self.natom * 3, dtype=torch.float64, device=self.dev)
        for qt in self.quartet_chunks():
            qt = self.shard(qt)
            if qt.shape[0]:
                self._force_chunk(qt, force)
        return self._sum_over_ranks(force).view(self.natom, 3)

    def _force_chunk(self, qt, force):
        """Adds the adjoint gradient of the unique quartets qt [n,4] to force:
        the six auxiliary batches (each centre raised and lowered), then one
        digestion pass over them (intception_b200_jk_force_all)."""
        torch = self.torch
        lib = _lib()
        stream = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        lorig = self.shell_l[:self.ns]
        n = qt.shape[0]
        if not self.per_batch_digestion:
            m0 = self._mark()
            offs, blks = [], []
            for pos in range(3):
                for sign in (1, -1):
                    if sign > 0:
                        sel = None
                        aux = qt.clone()
                    else:
                        sel = torch.nonzero(lorig[qt[:, pos].long()] >= 1).flatten()
                        aux = qt[sel].clone()
                    aux[:, pos] += self.ns if sign > 0 else 2 * self.ns
                    blocks, off = self._eri(aux.contiguous(), self.lmax + 1)
                    if sel is not None:
                        full = torch.full((n,), -1, dtype=torch.int64, device=self.dev)
                        full[sel] = off
                        off = full
                    offs.append(off)
                    blks.append(blocks)
            m1 = self._mark()
            eri._check(lib.intception_b200_jk_force_all(
                qt.data_ptr(), n, (C.c_void_p * 6)(*[o.data_ptr() for o in offs]),
                (C.c_void_p * 6)(*[b.data_ptr() for b in blks]), self.shell_l.data_ptr(), self.fofs.data_ptr(),
                self.shell_atom.data_ptr(), self.P.data_ptr(), self.nbf_cart, self.natom, force.data_ptr(),
                stream))
            if m0 is not None:
                self._marks.append((m0, m1, self._mark()))
            return
        # one digestion launch per auxiliary batch (intception_b200_jk_force)
        for pos in range(3):
            for sign in (1, -1):
                if sign > 0:
                    sel = torch.arange(n, device=self.dev, dtype=torch.int32)
                else:
                    sel = torch.nonzero(lorig[qt[:, pos].long()] >= 1).flatten().to(torch.int32)
                if sel.numel() == 0:
                    continue
                aux = qt[sel.long()].clone()
                aux[:, pos] += self.ns if sign > 0 else 2 * self.ns
                m0 = self._mark()
                blocks, off = self._eri(aux.contiguous(), self.lmax + 1)
                m1 = self._mark()
                eri._check(lib.intception_b200_jk_force(
                    qt.data_ptr(), sel.data_ptr(), off.data_ptr(), sel.numel(), pos, sign,
                    self.shell_l.data_ptr(), self.fofs.data_ptr(), self.shell_atom.data_ptr(),
                    self.P.data_ptr(), self.nbf_cart, self.natom, blocks.data_ptr(), force.data_ptr(), stream))
                if m0 is not None:
                    self._marks.append((m0, m1, self._mark()))


def _energy_function():
    import torch

    class JKEnergy(torch.autograd.Function):
        """E(xyz) = E_J + E_K; backward recomputes the derivative integrals
        (nothing from the forward pass is stored but the geometry)."""

        @staticmethod
        def forward(ctx, xyz, system):
            ctx.system = system
            ctx.save_for_backward(xyz)
            ej, ek = system.energy(xyz.detach())
            return xyz.new_tensor(ej + ek)

        @staticmethod
        def backward(ctx, grad):
            (xyz,) = ctx.saved_tensors
            g = ctx.system.gradient(xyz.detach()).to(device=xyz.device, dtype=xyz.dtype)
            return grad.to(xyz.device) * g, None

    return JKEnergy


def jk_energy(xyz, system):
    """Differentiable J/K energy (torch autograd)."""
    return _energy_function().apply(xyz, system)


def lattice_system(natom=60, seed=3, spacing=2.6, jitter=0.3, shells=((0, 6), (0, 3), (1, 3), (2, 1)),
                   alpha=(0.1, 1e3), nocc=10, device='cuda', screen=1e-15, **shard):
    """Jittered cubic lattice: the first natom sites (row-major) of the smallest
    cube holding them, spacing 2.6 bohr, uniform +-0.3 bohr jitter; per atom the
    given (l, K) shells with exponents log-uniform in alpha and coefficients
    uniform [0.1, 1] then normalised; P = C C^T with C ~ normal(0, 0.1),
    nbf x nocc.  shard: rank, world, group, reduce of JKSystem."""
    rng = np.random.default_rng(seed)
    n = int(np.ceil(natom ** (1.0 / 3.0) - 1e-9))
    sites = np.array([(i, j, k) for i in range(n) for j in range(n) for k in range(n)][:natom], np.float64)
    xyz = sites * spacing + rng.uniform(-jitter, jitter, (natom, 3))
    ls = np.array([l for _ in range(natom) for (l, _) in shells], np.int32)
    ks = np.array([kk for _ in range(natom) for (_, kk) in shells], np.int32)
    atom = np.repeat(np.arange(natom), len(shells)).astype(np.int32)
    _, _, _, _, e, c = B.make_shells(rng, ls, ks, alpha[0], alpha[1], 1.0, centres=np.zeros((len(ls), 3)))
    nbf = int((2 * ls + 1).sum())
    Cm = rng.normal(0.0, 0.1, (nbf, nocc))
    P = Cm @ Cm.T
    return JKSystem(xyz, atom, ls, ks, e, c, P, device=device, screen=screen, **shard), xyz


def main(argv=None):
    """Energy and adjoint gradient of the jittered-lattice system, with a
    central-difference check of a few gradient components; prints one JSON."""
    import argparse
    import json
    import time
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument('--atoms', type=int, default=60)
    ap.add_argument('--seed', type=int, default=3)
    ap.add_argument('--screen', type=float, default=1e-15)
    ap.add_argument('--fd-components', type=int, default=3)
    ap.add_argument('--h', type=float, default=1e-4)
    ap.add_argument('--fd4', action='store_true', help='also the four-point central stencil (same h)')
    a = ap.parse_args(argv)
    sys_, xyz = lattice_system(natom=a.atoms, seed=a.seed, screen=a.screen)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    (ej, ek), te = timed(lambda: sys_.energy(xyz))
    nquart = sum(int(q.shape[0]) for q in sys_.quartet_chunks())
    g, tg = timed(lambda: sys_.gradient(xyz).cpu().numpy())
    # the same two passes again with CUDA events around every ERI batch and digestion launch
    sys_.profile = True
    sys_.energy(xyz)
    split_e = sys_.kernel_split()
    sys_.gradient(xyz)
    split_g = sys_.kernel_split()
    sys_.profile = False
    rng = np.random.default_rng(a.seed + 100)
    checks = []
    def shifted(at, d, k):
        x = xyz.copy()
        x[at, d] += k * a.h
        return sum(sys_.energy(x))

    for _ in range(a.fd_components):
        at, d = int(rng.integers(a.atoms)), int(rng.integers(3))
        ep, em = shifted(at, d, 1), shifted(at, d, -1)
        fd = (ep - em) / (2 * a.h)
        chk = {'atom': at, 'xyz': d, 'adjoint': float(g[at, d]), 'central_fd': fd, 'abs_diff': abs(float(g[at, d]) - fd)}
        if a.fd4:
            # the same step h on the four-point central stencil: its O(h^2)
            # truncation term cancels, which tells FD error from adjoint error
            e2p, e2m = shifted(at, d, 2), shifted(at, d, -2)
            fd4 = (8.0 * (ep - em) - (e2p - e2m)) / (12.0 * a.h)
            chk.update(central_fd4=fd4, abs_diff4=abs(float(g[at, d]) - fd4))
        checks.append(chk)
    out = {'atoms': a.atoms, 'nbf_sph': int(sum(2 * int(l) + 1 for l in sys_.shell_l[:sys_.ns].tolist())),
           'shells': sys_.ns, 'unique_quartets_after_screening': nquart, 'screen': a.screen,
           'E_J': ej, 'E_K': ek, 'energy_s': te, 'gradient_s': tg,
           'energy_split_ms': {'eri': split_e[0], 'digestion': split_e[1],
                               'digestion_share': split_e[1] / max(split_e[0] + split_e[1], 1e-9)},
           'gradient_split_ms': {'eri': split_g[0], 'digestion': split_g[1],
                                 'digestion_share': split_g[1] / max(split_g[0] + split_g[1], 1e-9)},
           'max_abs_fd_diff': max(c['abs_diff'] for c in checks) if checks else None,
           'max_abs_fd4_diff': max(c['abs_diff4'] for c in checks) if checks and a.fd4 else None,
           'translational_residual': float(np.abs(g.sum(axis=0)).max()), 'fd_checks': checks}
    print(json.dumps(out))


if __name__ == '__main__':
    main()
