"""CUDA emitter: one fully unrolled sm_100a kernel per canonical ERI class.

This is the B200 counterpart of the reference's C99 emission layer
(``generator/callables/main_source_algorithms/contracted_general.py`` and the
recipes in ``generator/callables/``): where the reference prints loops over a
work array, this emitter resolves the recurrences at generation time into a
straight-line dataflow graph per class, so every VRR/HRR intermediate is a
named scalar the CUDA register allocator can keep on chip.

Schedule per contracted quartet (Head-Gordon-Pople with two HRRs):
  for each primitive quartet (bra pair x ket pair):
      [00|00]^(m) = pref * F_m(T),  m = 0..L                  (Boys, FP64)
      bra VRR:  [e+1i,0|00]^(m)                                 (Obara-Saika)
      ket VRR:  [e0|f+1i,0]^(m)  with the electron-transfer term
      acc[e][f] += [e0|f0]^(0)   e in [la, la+lb], f in [lc, lc+ld]
  bra HRR (a, b+1i) = (a+1i, b) + AB_i (a, b)          (reference form,
                                                        dsl_extensions.py:903-950)
  ket HRR (c, d+1i) = (c+1i, d) + CD_i (c, d)
  optional Cartesian->spherical transform with the library's matrices
  strided store of the (ab|cd) block.

The VRR recurrences are the ones the ERI input script gives the reference
(oracle/eri_input.py): the bra term of vrra and the ket term of vrrc, applied
to the HGP target set instead of the reference's VRR-on-d schedule.

Canonical classes have la >= lb, lc >= ld and pair(la,lb) >= pair(lc,ld); the
host permutes shells and output strides so every quartet maps onto one.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from intception_b200.basis import sph_matrix  # noqa: E402

LMAX_EMIT = 2  # classes with every l <= LMAX_EMIT get an unrolled kernel
# classes kept on the one-thread-per-quartet kernel (everything else whose
# smaller side fits a warp uses the lane-group kernel of group_emitter.py)
THREAD_CLASSES = set()

DIRS = 'xyz'
NPAIR_TOTAL = 7 * 8 // 2                       # shell pairs with l <= 6 (IB_NPAIR)
# pair ids: la >= lb canonical (0..27), and (2,3) -- a d shell built on before
# its f partner -- as pair 28 (IB_NPAIR_EXT): the one reversed pair with class
# kernels, for pairs whose horizontal recurrence is ill-conditioned the
# canonical way round (the runtime routes other reversed pairs to the generic
# kernel)
REV_PAIRS = {(2, 3): NPAIR_TOTAL}
NPAIR_EXT = NPAIR_TOTAL + len(REV_PAIRS)
NCLASS_TOTAL = NPAIR_EXT * (NPAIR_EXT + 1) // 2  # class ids (IB_NCLASS)


def comps(l):
    out = []
    for mx in range(l, -1, -1):
        for my in range(l - mx, -1, -1):
            out.append((mx, my, l - mx - my))
    return out


def comps_range(lo, hi):
    out = []
    for l in range(lo, hi + 1):
        out += comps(l)
    return out


def pair_index(la, lb):
    if la >= lb:
        return la * (la + 1) // 2 + lb
    return REV_PAIRS[(la, lb)]


def class_id(la, lb, lc, ld):
    pb, pk = pair_index(la, lb), pair_index(lc, ld)
    return pb * (pb + 1) // 2 + pk


def canonical_classes(lmax):
    out = []
    pairs = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    pairs.sort(key=lambda p: pair_index(*p))
    for pb in pairs:
        for pk in pairs:
            if pair_index(*pk) <= pair_index(*pb):
                out.append(pb + pk)
    out.sort(key=lambda c: class_id(*c))
    return out


def sub(e, i, k=1):
    t = list(e)
    t[i] -= k
    return tuple(t)


def add(e, i, k=1):
    t = list(e)
    t[i] += k
    return tuple(t)


ZERO = (0, 0, 0)


class Emitter:
    def __init__(self, la, lb, lc, ld):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.L = la + lb + lc + ld
        self.E = comps_range(la, la + lb)
        self.F = comps_range(lc, lc + ld)
        self.tag = '%d%d%d%d' % (la, lb, lc, ld)
        self.lines = []
        self.nodes = {}
        self.nvar = 0
        self.mult = {}  # (base, k) -> var
        self.flops = 0

    # ------------------------------------------------------------------ VRR
    def _mult(self, base, k):
        if k == 1:
            return base
        key = (base, k)
        if key not in self.mult:
            self.mult[key] = '%s_%d' % (base, k)
        return self.mult[key]

    def _new(self, expr, flops):
        name = 'v%d' % self.nvar
        self.nvar += 1
        self.lines.append('      const R %s = %s;' % (name, expr))
        self.flops += flops
        return name

    def _choose_ket_dir(self, e, f):
        best = None
        for i in range(3):
            if f[i] == 0:
                continue
            fm = sub(f, i)
            nterms = 2 + (1 if fm[i] > 0 else 0) * 2 + (1 if e[i] > 0 else 0)
            deps = [(e, fm, 0), (e, fm, 1)]
            if fm[i] > 0:
                deps += [(e, sub(fm, i), 0), (e, sub(fm, i), 1)]
            if e[i] > 0:
                deps.append((sub(e, i), fm, 1))
            have = sum(1 for d in deps if (d[0], d[1]) in self._seen_ef)
            key = (nterms, -have, i)
            if best is None or key < best[0]:
                best = (key, i)
        return best[1]

    def _choose_bra_dir(self, e):
        best = None
        for i in range(3):
            if e[i] == 0:
                continue
            em = sub(e, i)
            nterms = 2 + (2 if em[i] > 0 else 0)
            have = (1 if (em, ZERO) in self._seen_ef else 0)
            key = (nterms, -have, i)
            if best is None or key < best[0]:
                best = (key, i)
        return best[1]

    def node(self, e, f, m):
        key = (e, f, m)
        if key in self.nodes:
            return self.nodes[key]
        if f == ZERO:
            if e == ZERO:
                name = 's%d' % m
                self.nodes[key] = name
                return name
            i = self._choose_bra_dir(e)
            em = sub(e, i)
            d = DIRS[i]
            a0 = self.node(em, ZERO, m)
            a1 = self.node(em, ZERO, m + 1)
            expr = 'PA%s * %s + WP%s * %s' % (d, a0, d, a1)
            fl = 3
            if em[i] > 0:
                e2 = sub(em, i)
                b0 = self.node(e2, ZERO, m)
                b1 = self.node(e2, ZERO, m + 1)
                expr += ' + %s * (%s - roz * %s)' % (self._mult('o2z', em[i]), b0, b1)
                fl += 4
        else:
            i = self._choose_ket_dir(e, f)
            fm = sub(f, i)
            d = DIRS[i]
            a0 = self.node(e, fm, m)
            a1 = self.node(e, fm, m + 1)
            expr = 'QC%s * %s + WQ%s * %s' % (d, a0, d, a1)
            fl = 3
            if fm[i] > 0:
                f2 = sub(fm, i)
                b0 = self.node(e, f2, m)
                b1 = self.node(e, f2, m + 1)
                expr += ' + %s * (%s - roe * %s)' % (self._mult('o2e', fm[i]), b0, b1)
                fl += 4
            if e[i] > 0:
                c1 = self.node(sub(e, i), fm, m + 1)
                expr += ' + %s * %s' % (self._mult('o2zpe', e[i]), c1)
                fl += 2
        name = self._new(expr, fl)
        self.nodes[key] = name
        self._seen_ef.add((e, f))
        return name

    def emit_vrr(self):
        self._seen_ef = set()
        nf = len(self.F)
        acc_lines = []
        # walk targets ket-level by ket-level so intermediates die early
        for jf, f in enumerate(self.F):
            for ie, e in enumerate(self.E):
                v = self.node(e, f, 0)
                acc_lines.append((len(self.lines), '      acc[%d] += (double)%s;' % (ie * nf + jf, v)))
                self.flops += 1
        # interleave accumulation right after each target is produced
        out = []
        pos = 0
        for at, line in acc_lines:
            out += self.lines[pos:at]
            out.append(line)
            pos = at
        out += self.lines[pos:]
        mult_defs = ['      const R %s = (R)%d * %s;' % (name, k, base)
                     for (base, k), name in sorted(self.mult.items())]
        return mult_defs + out

    # ------------------------------------------------------------------ HRR
    def emit_hrr(self):
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        A, B, Cc, D = comps(la), comps(lb), comps(lc), comps(ld)
        E_index = {e: i for i, e in enumerate(self.E)}
        F_index = {f: i for i, f in enumerate(self.F)}
        nf = len(self.F)
        lines = []
        cnt = [0]

        def hrr_graph(targets_a, targets_b, leaf, rvec, prefix):
            memo = {}

            def get(a, b):
                if b == ZERO:
                    return leaf(a)
                if (a, b) in memo:
                    return memo[(a, b)]
                i = 0 if b[0] > 0 else (1 if b[1] > 0 else 2)  # x, then y, then z
                x1 = get(add(a, i), sub(b, i))
                x2 = get(a, sub(b, i))
                name = '%s%d' % (prefix, cnt[0])
                cnt[0] += 1
                lines.append('    const double %s = %s + %s%s * %s;' % (name, x1, rvec, DIRS[i], x2))
                self.hrr_flops += 2
                memo[(a, b)] = name
                return name

            return {(a, b): get(a, b) for a in targets_a for b in targets_b}

        self.hrr_flops = 0
        nab = len(A) * len(B)
        lines.append('    double hb[%d];' % (nab * nf))
        for jf, f in enumerate(self.F):
            res = hrr_graph(A, B, lambda a, jf=jf: 'acc[%d]' % (E_index[a] * nf + jf), 'AB', 'h%d_' % jf)
            for ia, a in enumerate(A):
                for ib, b in enumerate(B):
                    lines.append('    hb[%d] = %s;' % ((ia * len(B) + ib) * nf + jf, res[(a, b)]))
        ncd = len(Cc) * len(D)
        lines.append('    double r[%d];' % (nab * ncd))
        for ab in range(nab):
            res = hrr_graph(Cc, D, lambda c, ab=ab: 'hb[%d]' % (ab * nf + F_index[c]), 'CD', 'k%d_' % ab)
            for ic, c in enumerate(Cc):
                for id_, d in enumerate(D):
                    lines.append('    r[%d] = %s;' % (ab * ncd + ic * len(D) + id_, res[(c, d)]))
        return lines

    # ------------------------------------------------------ sph + store
    def emit_store(self, sph):
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        dims = [len(comps(l)) for l in (la, lb, lc, ld)]
        lines = []
        cur = 'r'
        self.sph_flops = 0
        if sph:
            shape = list(dims)
            for axis in (3, 2, 1, 0):
                l = (la, lb, lc, ld)[axis]
                T = sph_matrix(l)
                nsph = 2 * l + 1
                newshape = list(shape)
                newshape[axis] = nsph
                name = 'sp%d' % axis
                total = newshape[0] * newshape[1] * newshape[2] * newshape[3]
                lines.append('    double %s[%d];' % (name, total))

                def flat(idx, shp):
                    return ((idx[0] * shp[1] + idx[1]) * shp[2] + idx[2]) * shp[3] + idx[3]

                import itertools
                for idx in itertools.product(*[range(n) for n in newshape]):
                    s = idx[axis]
                    terms = []
                    for c in range(shape[axis]):
                        coef = T[c, s]
                        if abs(coef) < 1e-15:
                            continue
                        src = list(idx)
                        src[axis] = c
                        if abs(coef - 1.0) < 1e-15:
                            terms.append('%s[%d]' % (cur, flat(src, shape)))
                        else:
                            terms.append('%.17g * %s[%d]' % (coef, cur, flat(src, shape)))
                        self.sph_flops += 2
                    lines.append('    %s[%d] = %s;' % (name, flat(idx, newshape), ' + '.join(terms) or '0.0'))
                cur = name
                shape = newshape
            dims = shape
        import itertools
        for idx in itertools.product(*[range(n) for n in dims]):
            flat = ((idx[0] * dims[1] + idx[1]) * dims[2] + idx[2]) * dims[3] + idx[3]
            offs = ' + '.join('%d * st%d' % (v, k) for k, v in enumerate(idx) if v)
            lines.append('    o[%s] = %s[%d];' % (offs or '0', cur, flat))
        return lines

    # ------------------------------------------------------------ kernel
    def kernel(self):
        L = self.L
        vrr = self.emit_vrr()
        hrr = self.emit_hrr()
        st_cart = self.emit_store(False)
        st_sph = self.emit_store(True)
        sph_flops = self.sph_flops
        nacc = len(self.E) * len(self.F)
        t = self.tag
        cid = class_id(self.la, self.lb, self.lc, self.ld)
        src = []
        src.append('// ---- class (%d%d|%d%d): %d VRR nodes, %d VRR flops/primitive quartet, %d HRR flops'
                   % (self.la, self.lb, self.lc, self.ld, self.nvar, self.flops, self.hrr_flops))
        src.append('template <typename R, bool SPH>')
        src.append('__global__ void __launch_bounds__(IB_BLOCK) ib_eri_%s(const IbLaunch a) {' % t)
        src.append('  const int beg = a.ranges[2 * %d], end = a.ranges[2 * %d + 1];' % (cid, cid))
        src.append('  if (beg + (int)(blockIdx.x * blockDim.x) >= end) return;  // block-uniform')
        src.append('  for (int p = beg + blockIdx.x * blockDim.x + threadIdx.x; p < end; p += gridDim.x * blockDim.x) {')
        src.append('    IbQuartet g;')
        src.append('    ib_load_quartet(a, p, g);')
        src.append('    double acc[%d];' % nacc)
        src.append('#pragma unroll')
        src.append('    for (int k = 0; k < %d; ++k) acc[k] = 0.0;' % nacc)
        src.append('    for (int ia = 0; ia < g.k[0]; ++ia)')
        src.append('    for (int ib = 0; ib < g.k[1]; ++ib) {')
        src.append('      IbBraPair bp;')
        src.append('      ib_bra_pair<sizeof(R) == 4>(a, g, ia, ib, bp);')
        src.append('      if (bp.K == 0.0) continue;')
        src.append('      for (int ic = 0; ic < g.k[2]; ++ic)')
        src.append('      for (int id = 0; id < g.k[3]; ++id) {')
        src.append('      IbPrimQuartet<R> pq;')
        src.append('      double F[%d];' % (L + 1))
        src.append('      if (!ib_prim_quartet<R, %d>(a, g, bp, ic, id, a.boys_tab, F, pq)) continue;' % L)
        for m in range(L + 1):
            src.append('      const R s%d = (R)F[%d];' % (m, m))
        src.append('      const R PAx = pq.PA[0], PAy = pq.PA[1], PAz = pq.PA[2];')
        src.append('      const R WPx = pq.WP[0], WPy = pq.WP[1], WPz = pq.WP[2];')
        src.append('      const R QCx = pq.QC[0], QCy = pq.QC[1], QCz = pq.QC[2];')
        src.append('      const R WQx = pq.WQ[0], WQy = pq.WQ[1], WQz = pq.WQ[2];')
        src.append('      const R o2z = pq.o2z, roz = pq.roz, o2e = pq.o2e, roe = pq.roe, o2zpe = pq.o2zpe;')
        src.append('      (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz;')
        src.append('      (void)QCx; (void)QCy; (void)QCz; (void)WQx; (void)WQy; (void)WQz;')
        src.append('      (void)o2z; (void)roz; (void)o2e; (void)roe; (void)o2zpe;')
        src += vrr
        src.append('      }')
        src.append('    }')
        src.append('    const double ABx = g.AB[0], ABy = g.AB[1], ABz = g.AB[2];')
        src.append('    const double CDx = g.CD[0], CDy = g.CD[1], CDz = g.CD[2];')
        src.append('    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;')
        src += hrr
        src.append('    double* __restrict__ o = a.out + g.off;')
        src.append('    const int st0 = g.st[0], st1 = g.st[1], st2 = g.st[2], st3 = g.st[3];')
        src.append('    (void)st0; (void)st1; (void)st2; (void)st3;')
        src.append('    if (SPH) {')
        src += ['  ' + s for s in st_sph]
        src.append('    } else {')
        src += ['  ' + s for s in st_cart]
        src.append('    }')
        src.append('  }')
        src.append('}')
        src.append('')
        # host-side launcher and occupancy query for this class
        src.append('static void ib_launch_%s(int variant, int grid, cudaStream_t s, const IbLaunch& a) {' % t)
        src.append('  const size_t smem = 0;')
        src.append('  switch (variant) {')
        src.append('    case 0: ib_eri_%s<double, false><<<grid, IB_BLOCK, smem, s>>>(a); break;' % t)
        src.append('    case 1: ib_eri_%s<double, true><<<grid, IB_BLOCK, smem, s>>>(a); break;' % t)
        src.append('    case 2: ib_eri_%s<float, false><<<grid, IB_BLOCK, smem, s>>>(a); break;' % t)
        src.append('    default: ib_eri_%s<float, true><<<grid, IB_BLOCK, smem, s>>>(a); break;' % t)
        src.append('  }')
        src.append('}')
        src.append('static int ib_occupancy_%s(int variant) {' % t)
        src.append('  int n = 0; const size_t smem = 0;')
        src.append('  switch (variant) {')
        src.append('    case 0: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ib_eri_%s<double, false>, IB_BLOCK, smem); break;' % t)
        src.append('    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ib_eri_%s<double, true>, IB_BLOCK, smem); break;' % t)
        src.append('    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ib_eri_%s<float, false>, IB_BLOCK, smem); break;' % t)
        src.append('    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ib_eri_%s<float, true>, IB_BLOCK, smem); break;' % t)
        src.append('  }')
        src.append('  return n;')
        src.append('}')
        src.append('')
        stats = dict(tag=t, cid=cid, L=L, nodes=self.nvar, vrr_flops=self.flops, hrr_flops=self.hrr_flops,
                     sph_flops=sph_flops, nacc=nacc)
        return '\n'.join(src), stats


DEFAULT_SLICE_CAP = 8


# shared memory a block may use (B200: 227 KB)
SMEM_LIMIT = 227 * 1024


def group_fits(c):
    """Whether class c gets a lane-group kernel: the smaller side fits a
    128-lane group, its base-chain path has at most 6 steps (the lane code
    packs 6), and a block's shared memory stays within SMEM_LIMIT."""
    from .group_emitter import GroupEmitter, orientation
    if orientation(*c) is None or min(c[0] + c[1], c[2] + c[3]) > 6:
        return False
    g = GroupEmitter(*c)
    g.kernel(fp32=False)
    groups = (128 // g.G) if g.wide else 4 * g.QPW
    return groups * g.per_group * 8 <= SMEM_LIMIT


def emitted_classes():
    """Canonical classes with an unrolled kernel: every class with l <= 2
    (FP64 and FP32-VRR variants), and every class with an f or g shell and the
    rest <= g that group_fits (FP64 only; the nuclear-gradient batches of an
    l <= 2 basis reach the one-f classes, an f basis the rest of the f
    classes, l <= 4 bases the g classes).  (gf|gf), (gg|gf), (gg|gg) and
    (gg|ss) stay on the generic kernel."""
    out = [(c, True) for c in canonical_classes(LMAX_EMIT)]
    for c in canonical_classes(4):
        if max(c) >= 3 and group_fits(c):
            out.append((c, False))
    # the reversed (d f| pair against every pair up to f (bra: its pair id is the largest)
    for kp in [(a, b) for a in range(4) for b in range(a + 1)] + [(2, 3)]:
        c = (2, 3) + kp
        if group_fits(c):
            out.append((c, False))
    out.sort(key=lambda x: class_id(*x[0]))
    return out


def emit_all(outdir, lmax=LMAX_EMIT, ngroups=8):
    """Write the class translation units and the dispatch table into outdir.
    Returns the list of per-class statistics."""
    os.makedirs(outdir, exist_ok=True)
    classes = emitted_classes()
    # balance translation units by emitted size (largest classes first)
    from .group_emitter import GroupEmitter, orientation
    bodies = []
    for c, fp32 in classes:
        # the one-thread schedule's counts are the algorithmic work of the class
        tbody, st = Emitter(*c).kernel()
        if orientation(*c) is not None and c not in THREAD_CLASSES:
            body, gst = GroupEmitter(*c).kernel(fp32=fp32)
            st.update(kind='group', G=gst['G'], orient=gst['orient'], lane_flops=gst['lane_flops'])
        else:
            body = tbody
            st['kind'] = 'thread'
        st['fp32'] = fp32
        bodies.append((c, body, st))
    order = sorted(bodies, key=lambda x: -len(x[1]))
    groups = [[] for _ in range(ngroups)]
    sizes = [0] * ngroups
    for item in order:
        k = sizes.index(min(sizes))
        groups[k].append(item)
        sizes[k] += len(item[1])
    written = []
    for g, items in enumerate(groups):
        path = os.path.join(outdir, 'eri_classes_%d.cu' % g)
        parts = ['// Generated by intception_b200/emit/eri_emitter.py -- do not edit.',
                 '#include "ib_eri_device.cuh"', '']
        regs = []
        for c, body, st in items:
            parts.append(body)
            regs.append(st)
        parts.append('void ib_register_group_%d(IbClassEntry* table) {' % g)
        for st in regs:
            parts.append('  table[%d] = IbClassEntry{%d, &ib_launch_%s, &ib_occupancy_%s, %d};'
                         % (st['cid'], st['cid'], st['tag'], st['tag'], 2 if st['fp32'] else 1))
        parts.append('}')
        _write_if_changed(path, '\n'.join(parts) + '\n')
        written.append(path)
    disp = ['// Generated by intception_b200/emit/eri_emitter.py -- do not edit.',
            '#include "ib_eri_device.cuh"']
    for g in range(ngroups):
        disp.append('void ib_register_group_%d(IbClassEntry* table);' % g)
    disp.append('void ib_register_emitted_classes(IbClassEntry* table) {')
    for g in range(ngroups):
        disp.append('  ib_register_group_%d(table);' % g)
    disp.append('}')
    # autotuned defaults (intception_b200/tuning.json, written by
    # python -m intception_b200.autotune on a GPU): per class and variant the
    # register-budget index, per class the slice cap and whether the FP32 tier
    # uses the class's FP32 kernel (where it measured faster than FP64)
    minb = [[0] * 4 for _ in range(NCLASS_TOTAL)]
    # at most 8 lane groups per quartet unless tuned otherwise: measured on the
    # screened l <= 2 step (3.4 % of 1e6 quartets kept, primitive screening at
    # 1e-18), a cap of 8 gave 1.18 ms per step against 1.30 uncapped, 1.36 at 2
    # and 1.64 at 1; a class with many quartets runs one group each anyway
    scap = [DEFAULT_SLICE_CAP] * NCLASS_TOTAL
    fp32on = [1] * NCLASS_TOTAL
    tpath = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'tuning.json')
    if os.path.exists(tpath):
        import json
        with open(tpath) as fh:
            tun = json.load(fh)
        for tag, ent in tun.get('classes', {}).items():
            cid = class_id(*(int(ch) for ch in tag))
            minb[cid] = [int(x) for x in ent.get('minb', [0, 0, 0, 0])]
            scap[cid] = int(ent.get('slice_cap', DEFAULT_SLICE_CAP))
            fp32on[cid] = 1 if ent.get('fp32', True) else 0
    disp.append('extern const int ib_tuned_minb[%d][4] = {%s};'
                % (NCLASS_TOTAL, ', '.join('{%s}' % ', '.join(map(str, r)) for r in minb)))
    disp.append('extern const int ib_tuned_slice_cap[%d] = {%s};' % (NCLASS_TOTAL, ', '.join(map(str, scap))))
    disp.append('extern const int ib_tuned_fp32[%d] = {%s};' % (NCLASS_TOTAL, ', '.join(map(str, fp32on))))
    disp.append('extern const int ib_n_emitted_classes = %d;' % len(classes))
    disp.append('extern const int ib_lmax_emitted = %d;' % lmax)
    _write_if_changed(os.path.join(outdir, 'eri_dispatch.cu'), '\n'.join(disp) + '\n')
    stats = [b[2] for b in bodies]
    with open(os.path.join(outdir, 'class_stats.txt'), 'w') as fh:
        for st in stats:
            fh.write(' '.join('%s=%s' % kv for kv in sorted(st.items())) + '\n')
    return stats


def _write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as fh:
            if fh.read() == text:
                return
    with open(path, 'w') as fh:
        fh.write(text)


if __name__ == '__main__':
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(HERE), 'csrc', '_gen')
    for st in emit_all(out):
        print(st)
