"""Lane-group ERI kernels: G lanes share one contracted quartet.

Each lane of a group owns one Cartesian component s of the "lane side" (the bra
e-range or the ket f-range, whichever has fewer components) and computes, per
primitive quartet, the whole recurrence for the other ("chain") side for that
component in registers:

  base chain   [s|0]^(m): the lane's own component built from [0|0]^(m) along a
               path that takes all z steps, then y, then x, so the two-back
               term of the Obara-Saika recurrence is always the lane's previous
               chain element (no communication);
  chain side   [s|c+1i]^(m) = X_i [s|c]^(m) + W_i [s|c]^(m+1)
                              + c_i/2x ([s|c-1i]^(m) - r [s|c-1i]^(m+1))
                              + s_i/2(zeta+eta) [s-1i|c]^(m+1)
               where the last (electron-transfer) term is the same register of
               the lane that owns s-1i, fetched with __shfl_sync.  The direction
               i depends only on c, so the instruction stream is uniform across
               the group; only s_i and the source lane differ per lane.
  contraction  acc[c] += [s|c]^(0) over the chain-side targets, FP64.

After the primitive loops the group writes its accumulators to shared memory
as [e][f], runs the bra HRR (lanes over f), the spherical transform of a and b,
the ket HRR (lanes over ab), the spherical transform of c and d, and stores.

With the bra as lane side the recurrences are the input script's vrra (base
chain) and vrrc (chain side, transfer term from the bra); with the ket as lane
side they are the mirror images (vrrc as base chain, the bra recurrence with
its transfer term 1/2(zeta+eta) f_i [e|f-1i]^(m+1) as chain side).
"""
import itertools

from .eri_emitter import comps, comps_range, class_id, sub, add, ZERO, DIRS

try:
    from intception_b200.basis import sph_matrix
except ImportError:  # pragma: no cover
    from ..basis import sph_matrix


def ncum(l):
    return 0 if l < 0 else (l + 1) * (l + 2) * (l + 3) // 6


def ncart(l):
    return (l + 1) * (l + 2) // 2


def cidx(c):
    l = sum(c)
    return ncum(l - 1) + c[2] + (c[1] + c[2]) * (c[1] + c[2] + 1) // 2


def orientation(la, lb, lc, ld):
    """'bra' if the lanes own bra components, 'ket' otherwise; None when
    neither side fits a 128-lane (four-warp, whole-block) group."""
    ne, nf = ncum(la + lb), ncum(lc + ld)
    if min(ne, nf) > 128:
        return None
    return 'bra' if ne <= nf else 'ket'


# Chain emission order, per class: 'level' (level by level, each level's
# shuffles batched: more independent work between dependent instructions, more
# live registers) or 'dfs' (dependency order with shuffles inline).  Chosen by
# the autotuner (intception_b200/tuning.json "order"); INTCEPTION_B200_CHAIN_ORDER
# forces one order for every class (the autotuner's tuning builds).
def _chain_orders():
    import json
    import os
    out = {}
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'tuning.json')
    if os.path.exists(path):
        with open(path) as fh:
            for tag, ent in json.load(fh).get('classes', {}).items():
                if ent.get('order') in ('level', 'dfs'):
                    out[tag] = ent['order']
    return out


CHAIN_ORDER = _chain_orders()


def chain_order(tag):
    import os
    forced = os.environ.get('INTCEPTION_B200_CHAIN_ORDER')
    if forced in ('level', 'dfs'):
        return forced
    return CHAIN_ORDER.get(tag, 'dfs')


def group_size(n):
    g = 1
    while g < n:
        g *= 2
    return g


# pack ten-lane groups three to a warp (False: pad them to 16 lanes, two per warp)
PACK_TEN = True

# lane sides of 21..63 components whose levels below the top fit in fewer than
# 32 lanes (the S_hi = 4 sides: 20 low + 15 top components): every warp of the
# group holds all the low levels plus its share of the top level, so the
# transfer operands stay inside the warp (shuffles, no per-level barrier); the
# low levels are evaluated once per warp.  Off (False: one copy, transfer
# operands through shared memory with a named barrier per level): measured on
# B200, (dd|dd) alone 11.6 ms with it against 10.2 ms without (1e5 quartets,
# K 1..6), the l <= 2 FP64 step 16.0 against 15.7 ms -- the duplicated chains
# cost more than the barriers they remove.
DUP_LOW = False

# register budgets offered to the autotuner: __launch_bounds__(IB_BLOCK, MINB)
# asks for MINB resident blocks per SM (1: no register cap); must match
# IB_MINB_VALUES in ib_eri_device.cuh
MINB_VALUES = (1, 3, 4, 5)


class GroupEmitter:
    def __init__(self, la, lb, lc, ld, tuned=None):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.L = la + lb + lc + ld
        # every register budget is instantiated for the l <= 2 classes
        self.tuned = (max(la, lb, lc, ld) <= 3 and la >= lb) if tuned is None else tuned
        self.E, self.F = la + lb, lc + ld
        self.orient = orientation(la, lb, lc, ld)
        assert self.orient is not None
        if self.orient == 'bra':
            self.S_lo, self.S_hi, self.C_lo, self.C_hi = la, self.E, lc, self.F
        else:
            self.S_lo, self.S_hi, self.C_lo, self.C_hi = lc, self.F, la, self.E
        self.NL = ncum(self.S_hi)
        self.G = group_size(self.NL)
        # ten lane-side components: three 10-lane groups per warp (lanes 30
        # and 31 idle) instead of two padded 16-lane groups; shuffles then
        # address absolute lanes and slices come in threes (one warp)
        self.packed = PACK_TEN and self.NL == 10
        if self.packed:
            self.G = 10
        # duplicated low levels (DUP_LOW): warp q of the group holds every
        # component below the top level in lanes 0..nlow-1 and top-level
        # components q*per .. q*per+per-1 in the others
        self.dup = DUP_LOW and self.NL > 32 and ncum(self.S_hi - 1) < 32
        if self.dup:
            self.nlow = ncum(self.S_hi - 1)
            self.per = 32 - self.nlow
            self.ntop = ncart(self.S_hi)
            self.G = 32 * (-(-self.ntop // self.per))
        # G = 64 or 128: two or four warps per quartet; without dup, transfer
        # operands go through shared memory, one named barrier per recurrence level
        self.wide = self.G > 32
        self.smem_xfer = self.wide and not self.dup
        self.QPW = max(1, 32 // self.G)
        self.tag = '%d%d%d%d' % (la, lb, lc, ld)
        self.cid = class_id(la, lb, lc, ld)
        self.lines = []
        self.nodes = {}
        self.nvar = 0
        self.flops = 0
        self.mult = {}
        self.shuffles = {}

    # -------------------------------------------------------------- lane table
    def lane_comp(self, j):
        """(component, index of the lane that serves as lane 0 for its transfer
        sources) of group lane j."""
        if self.dup:
            w, jw = divmod(j, 32)
            if jw < self.nlow:
                return comps_range(0, self.S_hi - 1)[jw], jw
            t = min(w * self.per + jw - self.nlow, self.ntop - 1)  # padding lanes mirror the last one
            return comps(self.S_hi)[t], jw
        jj = min(j, self.NL - 1)  # padding lanes mirror the last component
        return comps_range(0, self.S_hi)[jj], jj

    def lane_table(self):
        rows = []
        for j in range(self.G):
            c, jj = self.lane_comp(j)
            dirs, nbs = [], []
            for d in (2, 1, 0):
                for k in range(c[d]):
                    dirs.append(d)
                    nbs.append(k)
            src = []
            for d in range(3):
                src.append(cidx(sub(c, d)) if c[d] > 0 else jj)
            rows.append((c, dirs, nbs, src))
        return rows

    # -------------------------------------------------------------- chain DAG
    def _new(self, expr, fl):
        name = 'v%d' % self.nvar
        self.nvar += 1
        self.lines.append('        const R %s = %s;' % (name, expr))
        self.flops += fl
        return name

    def _m(self, base, k):
        if k == 1:
            return base
        key = (base, k)
        if key not in self.mult:
            self.mult[key] = '%s_%d' % (base, k)
        return self.mult[key]

    def node(self, c, m):
        key = (c, m)
        if key in self.nodes:
            return self.nodes[key]
        if c == ZERO:
            name = 'b%d' % m
            self.nodes[key] = name
            return name
        i = 0 if c[0] > 0 else (1 if c[1] > 0 else 2)
        cm = sub(c, i)
        d = DIRS[i]
        a0 = self.node(cm, m)
        a1 = self.node(cm, m + 1)
        expr = 'CX%s * %s + CW%s * %s' % (d, a0, d, a1)
        fl = 3
        if cm[i] > 0:
            c2 = sub(cm, i)
            b0 = self.node(c2, m)
            b1 = self.node(c2, m + 1)
            expr += ' + %s * (%s - cro * %s)' % (self._m('co2', cm[i]), b0, b1)
            fl += 4
        if self.S_hi > 0:
            # transfer term from the lane owning s - 1i
            if self.smem_xfer:
                lvl = sum(cm)
                slot = self.slot_index(cm, m + 1)
                expr += ' + tf%s * xb%d[%d * %d + src%s]' % (d, lvl % 2, slot, self.G, 'xyz'.index(d))
            else:
                expr += ' + tf%s * %s' % (d, self._shfl(a1, i, sum(cm)))
            fl += 2
        name = self._new(expr, fl)
        self.nodes[key] = name
        return name

    def _shfl(self, name, i, level):
        """Temporary holding the value `name` of the lane owning s - 1i; the
        shuffles of a level are issued together before its nodes."""
        key = (name, i)
        if key not in self.shuffles:
            self.shuffles[key] = ('x%d' % len(self.shuffles), level)
        return self.shuffles[key][0]

    def _shfl_call(self, name, i):
        """Read register `name` of the lane owning s - 1i (src0..2 hold group-
        relative lanes for power-of-two groups, absolute lanes when packed)."""
        if self.packed:
            return '__shfl_sync(gmask, %s, src%d)' % (name, i)
        if self.dup:
            return '__shfl_sync(0xffffffffu, %s, src%d, 32)' % (name, i)
        return '__shfl_sync(gmask, %s, src%d, %d)' % (name, i, self.G)

    def slot_index(self, c, m):
        """Position of chain node (c, m), m >= 1, in its level's transfer buffer."""
        k = sum(c)
        order = [(cc, mm) for cc in comps(k) for mm in range(1, self.C_hi - k + 1)]
        return order.index((c, m))

    def builder_lanes(self):
        """Declarations of the list-building lanes: the first min(SG, 32) lanes
        of the quartet, their warp mask and first lane."""
        out = ['        const int nbld = min(SG, 32);']
        if self.wide:
            out += ['        const unsigned bmask = 0xffffffffu;', '        const int bbase = 0;']
        else:
            out += ['        const unsigned bmask = SG >= 32 ? 0xffffffffu : sgmask;',
                    '        const int bbase = SG >= 32 ? 0 : lane - r;']
        return out

    def lcls(self):
        """The class's angular momenta as template arguments (canonical order)."""
        return '%d, %d, %d, %d' % (self.la, self.lb, self.lc, self.ld)

    def n_slots(self):
        return max(len(comps(k)) * (self.C_hi - k) for k in range(self.C_hi + 1))

    def emit_chain_wide(self):
        """Level-ordered chain for two-warp groups: compute level k, publish its
        m >= 1 values to shared memory, barrier, continue."""
        targets = comps_range(self.C_lo, self.C_hi)
        for c in targets:
            self.node(c, 0)
        byname = {}
        for (c, m), name in self.nodes.items():
            byname[name] = (c, m)
        level_lines = {}
        # self.lines were appended in DFS order; regroup by level
        for ln in self.lines:
            name = ln.split('const R ')[1].split(' =')[0]
            c, m = byname[name]
            level_lines.setdefault(sum(c), []).append(ln)
        out = ['        ib_group_bar(gid);']
        if ZERO in targets:
            out.append('        acc[%d] += (double)b0;' % targets.index(ZERO))
        # level 0: base values
        for mm in range(1, self.C_hi + 1):
            if ((0, 0, 0), mm) in self.nodes:
                out.append('        xb0[%d * %d + j] = b%d;' % (self.slot_index(ZERO, mm), self.G, mm))
        out.append('        ib_group_bar(gid);')
        t_index = {c: t for t, c in enumerate(targets)}
        for k in range(1, self.C_hi + 1):
            out += level_lines.get(k, [])
            for c in comps(k):
                if (c, 0) in self.nodes and c in t_index:
                    out.append('        acc[%d] += (double)%s;' % (t_index[c], self.nodes[(c, 0)]))
                    self.flops += 1
            if k < self.C_hi:
                for c in comps(k):
                    for mm in range(1, self.C_hi - k + 1):
                        if (c, mm) in self.nodes:
                            out.append('        xb%d[%d * %d + j] = %s;' % (k % 2, self.slot_index(c, mm), self.G,
                                                                         self.nodes[(c, mm)]))
                out.append('        ib_group_bar(gid);')
        defs = ['        const R %s = (R)%d * %s;' % (name, k, base) for (base, k), name in sorted(self.mult.items())]
        return defs + out, len(targets)

    def emit_chain_dfs(self):
        """Chain side in dependency (DFS) order from each target; shuffles sit
        inline next to their use and ptxas schedules them."""
        targets = comps_range(self.C_lo, self.C_hi)
        out = []
        t_index = {c: t for t, c in enumerate(targets)}
        if ZERO in t_index:
            out.append('        acc[%d] += (double)b0;' % t_index[ZERO])
        acc = []
        for t, c in enumerate(targets):
            if c == ZERO:
                continue
            n0 = len(self.lines)
            v = self.node(c, 0)
            acc.append((len(self.lines), '        acc[%d] += (double)%s;' % (t, v)))
            self.flops += 1
        shuf = {var: (src_name, i) for (src_name, i), (var, lvl) in self.shuffles.items()}
        pos = 0
        body = []
        for at, line in acc:
            body += self.lines[pos:at]
            body.append(line)
            pos = at
        body += self.lines[pos:]
        # inline the shuffle temporaries where they are used
        import re
        for ln in body:
            for var in re.findall(r'\bx\d+\b', ln):
                src_name, i = shuf[var]
                ln = re.sub(r'\b%s\b' % var, self._shfl_call(src_name, i), ln)
            out.append(ln)
        defs = ['        const R %s = (R)%d * %s;' % (name, k, base) for (base, k), name in sorted(self.mult.items())]
        return defs + out, len(targets)

    def emit_chain(self):
        """Chain side level by level: the level's transfer operands are fetched
        with back-to-back shuffles first (their latency overlaps), then its
        nodes, then the accumulation of the level's targets."""
        if self.smem_xfer:
            return self.emit_chain_wide()
        if chain_order(self.tag) == 'dfs':
            return self.emit_chain_dfs()
        targets = comps_range(self.C_lo, self.C_hi)
        for c in targets:
            self.node(c, 0)
        byname = {name: key for key, name in self.nodes.items()}
        level_lines = {}
        for ln in self.lines:
            name = ln.split('const R ')[1].split(' =')[0]
            c, m = byname[name]
            level_lines.setdefault(sum(c), []).append(ln)
        shuf_by_level = {}
        for (src_name, i), (var, lvl) in self.shuffles.items():
            shuf_by_level.setdefault(lvl + 1, []).append(
                '        const R %s = %s;' % (var, self._shfl_call(src_name, i)))
        t_index = {c: t for t, c in enumerate(targets)}
        out = []
        if ZERO in t_index:
            out.append('        acc[%d] += (double)b0;' % t_index[ZERO])
        for k in range(1, self.C_hi + 1):
            out += shuf_by_level.get(k, [])
            out += level_lines.get(k, [])
            for c in comps(k):
                if c in t_index:
                    out.append('        acc[%d] += (double)%s;' % (t_index[c], self.nodes[(c, 0)]))
                    self.flops += 1
        defs = ['        const R %s = (R)%d * %s;' % (name, k, base) for (base, k), name in sorted(self.mult.items())]
        return defs + out, len(targets)

    # -------------------------------------------------------------- HRR pieces
    @staticmethod
    def _hrr(targets_a, targets_b, leaf, rvec, prefix, lines, counter):
        memo = {}

        def get(a, b):
            if b == ZERO:
                return leaf(a)
            if (a, b) in memo:
                return memo[(a, b)]
            i = 0 if b[0] > 0 else (1 if b[1] > 0 else 2)
            x1 = get(add(a, i), sub(b, i))
            x2 = get(a, sub(b, i))
            name = '%s%d' % (prefix, counter[0])
            counter[0] += 1
            lines.append('      const double %s = %s + %s%s * %s;' % (name, x1, rvec, DIRS[i], x2))
            memo[(a, b)] = name
            return name

        return {(a, b): get(a, b) for a in targets_a for b in targets_b}

    @staticmethod
    def _sph2(vals, l1, l2, prefix, lines):
        """vals[(i1, i2)] Cartesian names -> spherical names over both indices."""
        T1, T2 = sph_matrix(l1), sph_matrix(l2)
        n1, n2 = ncart(l1), ncart(l2)
        mid = {}
        for s1 in range(2 * l1 + 1):
            for i2 in range(n2):
                terms = []
                for i1 in range(n1):
                    cf = T1[i1, s1]
                    if abs(cf) > 1e-15:
                        terms.append(vals[(i1, i2)] if abs(cf - 1) < 1e-15 else '%.17g * %s' % (cf, vals[(i1, i2)]))
                name = '%sm%d_%d' % (prefix, s1, i2)
                lines.append('      const double %s = %s;' % (name, ' + '.join(terms) if terms else '0.0'))
                mid[(s1, i2)] = name
        out = {}
        for s1 in range(2 * l1 + 1):
            for s2 in range(2 * l2 + 1):
                terms = []
                for i2 in range(n2):
                    cf = T2[i2, s2]
                    if abs(cf) > 1e-15:
                        terms.append(mid[(s1, i2)] if abs(cf - 1) < 1e-15 else '%.17g * %s' % (cf, mid[(s1, i2)]))
                name = '%ss%d_%d' % (prefix, s1, s2)
                lines.append('      const double %s = %s;' % (name, ' + '.join(terms) if terms else '0.0'))
                out[(s1, s2)] = name
        return out

    def emit_epilogue(self, sph):
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        A, B, Cc, D = comps(la), comps(lb), comps(lc), comps(ld)
        Elist = comps_range(la, self.E)
        Flist = comps_range(lc, self.F)
        NE, NF = len(Elist), len(Flist)
        NFP = NF if NF % 2 else NF + 1  # odd row stride: conflict-free column and row access
        e_index = {e: i for i, e in enumerate(Elist)}
        f_index = {f: i for i, f in enumerate(Flist)}
        na = (2 * la + 1) if sph else len(A)
        nb = (2 * lb + 1) if sph else len(B)
        nc = (2 * lc + 1) if sph else len(Cc)
        nd = (2 * ld + 1) if sph else len(D)
        L = []
        # bra HRR, lanes over f
        L.append('    for (int t = r; t < %d; t += SG) {' % NF)
        for e in range(NE):
            L.append('      const double q%d = sb0[%d * %d + t];' % (e, e, NFP))
        cnt = [0]
        body = []
        res = self._hrr(A, B, lambda a: 'q%d' % e_index[a], 'AB', 'h', body, cnt)
        L += body
        if sph:
            vals = {(A.index(a), B.index(b)): res[(a, b)] for a in A for b in B}
            body = []
            sres = self._sph2(vals, la, lb, 'sa', body)
            L += body
            outs = [sres[(i, k)] for i in range(na) for k in range(nb)]
        else:
            outs = [res[(a, b)] for a in A for b in B]
        for u, name in enumerate(outs):
            L.append('      sb0[%d * %d + t] = %s;' % (u, NFP, name))
        L.append('    }')
        L.append('    ib_sg_sync(SG, sg, sgmask);')
        # ket HRR, lanes over ab
        NAB = na * nb
        L.append('    for (int u = r; u < %d; u += SG) {' % NAB)
        for f in range(NF):
            L.append('      const double w%d = sb0[u * %d + %d];' % (f, NFP, f))
        body = []
        cnt = [0]
        res = self._hrr(Cc, D, lambda c: 'w%d' % f_index[c], 'CD', 'k', body, cnt)
        L += body
        if sph:
            vals = {(Cc.index(c), D.index(d)): res[(c, d)] for c in Cc for d in D}
            body = []
            sres = self._sph2(vals, lc, ld, 'sc', body)
            L += body
            cd = {(i, k): sres[(i, k)] for i in range(nc) for k in range(nd)}
        else:
            cd = {(Cc.index(c), D.index(d)): res[(c, d)] for c in Cc for d in D}
        L.append('      double* __restrict__ ou = o + (long long)(u / %d) * g.st[0] + (long long)(u %% %d) * g.st[1];'
                 % (nb, nb))
        for (i, k), name in cd.items():
            off = ' + '.join(x for x in (('%d * g.st[2]' % i) if i else '', ('%d * g.st[3]' % k) if k else '') if x)
            L.append('      ou[%s] = %s;' % (off or '0', name))
        L.append('    }')
        return L, max(NE, len(A) * len(B)) * NFP

    def err_expr(self):
        """FP32 error bound of the primitive quartet held in pq/F (see ib_fp32_err)."""
        if self.orient == 'bra':
            S, C = self.E, self.F
            aS = 'ib_amax3(pq.PA[0], pq.PA[1], pq.PA[2]) + ib_amax3(pq.WP[0], pq.WP[1], pq.WP[2])'
            bS = '%d.0 * (1.0 + (double)pq.roz) * (double)pq.o2z' % S
            aC = 'ib_amax3(pq.QC[0], pq.QC[1], pq.QC[2]) + ib_amax3(pq.WQ[0], pq.WQ[1], pq.WQ[2])'
            bC = '%d.0 * (1.0 + (double)pq.roe) * (double)pq.o2e' % C
        else:
            S, C = self.F, self.E
            aS = 'ib_amax3(pq.QC[0], pq.QC[1], pq.QC[2]) + ib_amax3(pq.WQ[0], pq.WQ[1], pq.WQ[2])'
            bS = '%d.0 * (1.0 + (double)pq.roe) * (double)pq.o2e' % S
            aC = 'ib_amax3(pq.PA[0], pq.PA[1], pq.PA[2]) + ib_amax3(pq.WP[0], pq.WP[1], pq.WP[2])'
            bC = '%d.0 * (1.0 + (double)pq.roz) * (double)pq.o2z' % C
        tC = '%d.0 * (double)pq.o2zpe' % S
        return 'ib_fp32_err(F[0], %s, %s, %d, %s, %s, %s, %d, IB_F32_SETUP_ROUNDINGS)' % (aS, bS, S, aC, bC, tC, C)

    def amp_expr(self):
        """Growth of an accumulator error through the HRRs and transforms."""
        from intception_b200.basis import sph_matrix
        import numpy as np
        sph = 1.0
        for l in (self.la, self.lb, self.lc, self.ld):
            sph *= float(np.abs(sph_matrix(l)).sum(axis=0).max())
        parts = []
        for _ in range(self.lb):
            parts.append('(1.0 + ib_amax3(g.AB[0], g.AB[1], g.AB[2]))')
        for _ in range(self.ld):
            parts.append('(1.0 + ib_amax3(g.CD[0], g.CD[1], g.CD[2]))')
        return ' * '.join(parts + ['(SPH ? %.17g : 1.0)' % sph])

    def hrr_check(self, NE, NF, NFP):
        """HRR rounding-error check on the contracted table sb0 ([e][f], rows
        of levels la..la+lb, columns lc..lc+ld, pitch NFP): the element at
        levels (la+k, lc+j) enters the outputs with coefficients of at most
        C(lb,k) |AB|^(lb-k) C(ld,j) |CD|^(ld-j); the largest |element| x
        weight, times IB_HRR_ERR_COEF, estimates the error."""
        def weights(l0, l1, r):
            # level boundaries of the rows (cumulative counts) and the weight of each level
            bounds, n = [], 0
            for k in range(l1 + 1):
                n += (l0 + k + 1) * (l0 + k + 2) // 2
                bounds.append(n)
            w = []
            for k in range(l1 + 1):
                c = 1
                for t in range(k):
                    c = c * (l1 - t) // (t + 1)
                w.append(' * '.join(['%d.0' % c] + [r] * (l1 - k)))
            return bounds, w

        def select(var, bounds, w):
            e = w[-1]
            for k in range(len(w) - 2, -1, -1):
                e = '(%s < %d ? %s : %s)' % (var, bounds[k], w[k], e)
            return e
        bb, wb = weights(self.la, self.lb, 'rab')
        bd, wd = weights(self.lc, self.ld, 'rcd')
        out = ['    if (a.hrr_tol > 0.0) {',
               '      const double rab = sqrt(g.AB[0] * g.AB[0] + g.AB[1] * g.AB[1] + g.AB[2] * g.AB[2]);',
               '      const double rcd = sqrt(g.CD[0] * g.CD[0] + g.CD[1] * g.CD[1] + g.CD[2] * g.CD[2]);',
               '      (void)rab; (void)rcd;',
               '      double hm = 0.0;',
               '      for (int x = r; x < %d; x += SG) {' % (NE * NF),
               '        const int row = x / %d, col = x - row * %d;' % (NF, NF),
               '        hm = fmax(hm, fabs(sb0[row * %d + col]) * %s * %s);' % (NFP, select('row', bb, wb),
                                                                          select('col', bd, wd)),
               '      }',
               '      if (hm * IB_HRR_ERR_COEF > a.hrr_tol) ib_redo_push(a, p);',
               '    }']
        return out

    # -------------------------------------------------------------- kernel
    def kernel(self, fp32=True):
        """CUDA source of the class kernel and its launcher; fp32=False
        instantiates the FP64 variants only (FP32 requests run in FP64)."""
        chain, NT = self.emit_chain()
        epi_cart, sm_cart = self.emit_epilogue(False)
        epi_sph, sm_sph = self.emit_epilogue(True)
        smem_group = max(sm_cart, sm_sph)
        t = self.tag
        bra = self.orient == 'bra'
        Elist = comps_range(self.la, self.E)
        Flist = comps_range(self.lc, self.F)
        NE, NF = len(Elist), len(Flist)
        NFP = NF if NF % 2 else NF + 1
        s_lo_idx = ncum(self.S_lo - 1)
        rows = self.lane_table()
        src = []
        # lane table
        src.append('// ---- class (%d%d|%d%d) lane-group kernel: lanes own %s components, G=%d, %d quartet(s)/warp,'
                   ' %d chain nodes, %d chain flops/primitive quartet/lane'
                   % (self.la, self.lb, self.lc, self.ld, 'bra' if bra else 'ket', self.G, self.QPW, self.nvar,
                      self.flops))
        # per lane: the base-chain steps padded at the front with identity
        # steps to S_hi (5 bits each: direction 0..2 or 3 = identity, then the
        # exponent before the step), and the component with the lanes owning
        # s - 1x, s - 1y, s - 1z (4 + 4 + 4 + 6 + 6 + 6 bits)
        assert self.S_hi <= 6 and self.G <= 128
        src.append('__constant__ IbLaneCode ib_lane_%s[%d] = {' % (t, self.G))
        for (c, dirs, nbs, sr) in rows:
            pad = self.S_hi - len(dirs)
            steps = [(3, 0)] * pad + list(zip(dirs, nbs))
            code = 0
            for k, (d, nb) in enumerate(steps):
                assert nb < 8
                code |= (d | (nb << 2)) << (5 * k)
            assert max(c) < 8 and max(sr) < 128
            misc = c[0] | (c[1] << 3) | (c[2] << 6) | (sr[0] << 9) | (sr[1] << 16) | (sr[2] << 23)
            src.append('  {0x%08xu, 0x%08xu},' % (code, misc))
        src.append('};')
        src.append('template <typename R, bool SPH, int MINB>')
        src.append('__global__ void __launch_bounds__(IB_BLOCK, MINB) ib_eri_%s(const IbLaunch a) {' % t)
        src.append('  extern __shared__ double ib_smem[];')
        # Slices: W lane groups (W a power of two, chosen per launch) share one
        # contracted quartet, each sweeping every W-th chunk of its primitive
        # quartets; the W partial accumulator tables are summed in shared memory
        # before the HRR.  W grows while the class's quartets cannot fill the
        # grid's groups, so a class with few (or very long) quartets still uses
        # the whole device.  W = 1 is the plain one-group-per-quartet kernel.
        gpb = 'IB_BLOCK / %d' % self.G if self.wide else '(IB_BLOCK / 32) * %d' % self.QPW
        src.append('  constexpr int GPB = %s;  // lane groups per block' % gpb)
        src.append('  const int beg = a.ranges[2 * %d], end = a.ranges[2 * %d + 1];' % (self.cid, self.cid))
        if self.packed:
            src.append('  const int W = ib_slices_in_threes(end - beg, GPB, a.max_slices, a.slice_boost);')
        else:
            src.append('  const int W = ib_slices(end - beg, GPB, a.max_slices, a.slice_boost);')
        src.append('  const int SPB = GPB / W;  // quartets in flight per block')
        src.append('  if (beg + (int)blockIdx.x * SPB >= end) return;  // block-uniform')
        if self.wide:
            src.append('  const int gid = threadIdx.x / %d, j = threadIdx.x %% %d;' % (self.G, self.G))
            src.append('  const unsigned gmask = 0xffffffffu;')
            src.append('  const unsigned sgmask = 0xffffffffu;')
            if self.dup:
                src.append('  const int jw = j & 31, wq = j >> 5;  // lane in its warp, warp in the group')
        else:
            src.append('  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;')
            src.append('  const int gq = lane / %d, j = lane %% %d;' % (self.G, self.G))
            if self.packed:
                # lanes past the last group of the warp take no part: slices stay
                # inside a warp (W = 1 or 3), so no barrier needs them
                src.append('  if (gq >= %d) return;' % self.QPW)
            src.append('  const int gid = warp * %d + gq;' % self.QPW)
            src.append('  const unsigned gmask = %s;' % ('0xffffffffu' if self.G == 32 else
                                                       '(((1u << %d) - 1u) << (gq * %d))' % (self.G, self.G)))
            src.append('  const unsigned sgmask = W * %d >= 32 ? 0xffffffffu : '
                       '(((1u << (W * %d)) - 1u) << ((gq / W) * W * %d));' % (self.G, self.G, self.G))
        src.append('  (void)gmask; (void)sgmask;')
        src.append('  const int sg = gid / W, w = gid - sg * W;  // quartet slot in the block, slice in the quartet')
        src.append('  const int SG = W * %d, r = w * %d + j;  // lanes per quartet, this lane among them'
                   % (self.G, self.G))
        nfield = 17 + self.L + 1 + 1  # setup fields, scaled F_0..F_L, and the live flags
        # the transfer buffers (xb) and the primitive setup table (ps, pz) are
        # live only inside the primitive loop, the contracted table only after
        # it (behind the super-group sync that closes the last tile): they
        # share the area at the start of the group's block
        xb_len = 2 * self.n_slots() * self.G if self.smem_xfer else 0
        loop_len = xb_len + (nfield * self.G if self.G > 1 else 0)
        per_group = max(smem_group, loop_len)
        self.list_off = per_group
        # live-pair lists of the quartet's current tile (2 x 64 bytes), the
        # screening exponents of their pairs (2 x 64 bytes), the counts, the grab slot
        per_group += 34
        self.red_off = per_group  # partial sums of a multi-warp or packed group's FP32 bound
        per_group += self.G if self.packed else (self.G // 32 if self.wide else 0)
        per_group += 1  # this slice's FP32 error bound, summed over the slices
        src.append('  double* __restrict__ sb = ib_smem + gid * %d;' % per_group)
        src.append('  double* __restrict__ sb0 = ib_smem + sg * W * %d;  // slice 0'
                   % per_group)
        if self.smem_xfer:
            src.append('  R* __restrict__ xb0 = reinterpret_cast<R*>(sb);')
            src.append('  R* __restrict__ xb1 = xb0 + %d;' % (self.n_slots() * self.G))
            src.append('  (void)xb1;')
        if self.G > 1:
            src.append('  R* __restrict__ ps = reinterpret_cast<R*>(sb + %d);' % xb_len)
            src.append('  int* __restrict__ pz = reinterpret_cast<int*>(sb + %d);' % (xb_len + (17 + self.L + 1) * self.G))
        self.per_group = per_group
        src.append('  unsigned char* __restrict__ lst = reinterpret_cast<unsigned char*>(sb0 + %d);' % self.list_off)
        src.append('  int* __restrict__ lcnt = reinterpret_cast<int*>(sb0 + %d);' % (self.list_off + 32))
        # lane constants read once and pinned in registers: a divergent
        # constant-bank load re-issued inside the primitive loop would be
        # serialised per distinct lane address
        src.append('  const unsigned lsteps = ib_pin(ib_lane_%s[j].steps), lmisc = ib_pin(ib_lane_%s[j].misc);'
                   % (t, t))
        if self.packed:
            src.append('  const int src0 = gq * %d + ((lmisc >> 9) & 127), src1 = gq * %d + ((lmisc >> 16) & 127), '
                       'src2 = gq * %d + ((lmisc >> 23) & 127);' % (self.G, self.G, self.G))
        elif self.dup:  # lanes of this warp
            src.append('  const int src0 = (lmisc >> 9) & 31, src1 = (lmisc >> 16) & 31, src2 = (lmisc >> 23) & 31;')
        else:
            src.append('  const int src0 = (lmisc >> 9) & 127, src1 = (lmisc >> 16) & 127, src2 = (lmisc >> 23) & 127;')
        src.append('  const double lcx = (double)(lmisc & 7), lcy = (double)((lmisc >> 3) & 7), '
                   'lcz = (double)((lmisc >> 6) & 7);')
        src.append('  (void)src0; (void)src1; (void)src2; (void)lsteps; (void)lcx; (void)lcy; (void)lcz;')
        # quartets handed out one at a time (ib_grab) instead of a fixed stride
        lane0 = '0' if self.wide else 'lane - r'
        grab = 'ib_grab(a.counter, beg, r, SG, sg, sgmask, %s, lcnt + 2)' % lane0
        src.append('  for (int p = %s; p < end; p = %s) {' % (grab, grab))
        src.append('    if (sizeof(R) == 8 && a.recheck && !(a.flags[p] & 1)) continue;  // uniform over the quartet\'s lanes')
        src.append('    IbQuartet g;')
        src.append('    ib_load_quartet(a, p, g);')
        src.append('    const int kb_ = g.k[1], kd_ = g.k[3];')
        src.append('    const int kab = g.k[0] * kb_, kcd = g.k[2] * kd_;')
        # primitive screening (a.prim_tol > 0) for quartets of one pair tile a
        # side: the screened lists are built here, before the accumulators
        # are live; larger quartets keep exact-zero culling only
        # classes with a g shell build only the exact-zero lists: on the l <= 4
        # sample workload with primitive screening on, a step of these kernels
        # (with the low levels then duplicated per warp) stopped on an illegal
        # address once; the screened lists stay off for them until that is
        # explained (their exact path ran clean on the same quartets)
        if max(self.la, self.lb, self.lc, self.ld) >= 4:
            src.append('    constexpr bool pre = false;  // g classes: exact-zero lists only')
        else:
            src.append('    const bool pre = a.prim_tol > 0.0 && kab <= 64 && kcd <= 64;  // uniform over the quartet')
        src.append('    if (pre && r < 32) {')
        src += ['  ' + ln for ln in self.builder_lanes()]
        src.append('      const int2 nn = ib_live_pairs_screened<%s, SPH>(a.prim_exp, a.prim_coef, g.ptr[0], g.ptr[1], '
                   'kb_, g.ptr[2], g.ptr[3], kd_, g.RAB2, g.RCD2, 0, kab, 0, kcd, lst, r, nbld, bmask, bbase, '
                   'a.prim_tol);' % self.lcls())
        src.append('      if (r == 0) { lcnt[0] = nn.x; lcnt[1] = nn.y; }')
        src.append('    }')
        src.append('    double acc[%d];' % NT)
        src.append('#pragma unroll')
        src.append('    for (int k = 0; k < %d; ++k) acc[k] = 0.0;' % NT)
        src.append('    double est = 0.0;  // FP32 rounding-error bound accumulated over primitive quartets')
        src.append('    (void)est;')
        L = self.L
        fields = ['PA[0]', 'PA[1]', 'PA[2]', 'WP[0]', 'WP[1]', 'WP[2]', 'QC[0]', 'QC[1]', 'QC[2]',
                  'WQ[0]', 'WQ[1]', 'WQ[2]', 'o2z', 'roz', 'o2e', 'roe', 'o2zpe']
        names = ['PAx', 'PAy', 'PAz', 'WPx', 'WPy', 'WPz', 'QCx', 'QCy', 'QCz', 'WQx', 'WQy', 'WQz',
                 'o2z', 'roz', 'o2e', 'roe', 'o2zpe']
        self.nfield = len(fields) + L + 1
        # Pair tiles of at most 64 x 64 primitive pairs; in each, the first
        # min(SG, 32) lanes of the quartet list the pairs whose prefactor is
        # not zero (ib_live_pairs), and the slices run over live x live
        # primitive quartets only (the others are exactly zero)
        src.append('    // exact small-integer quotients: (x + 0.5) / k is >= 1/128 away from an integer')
        src.append('    const float rkb = 1.0f / (float)kb_, rkd = 1.0f / (float)kd_;')
        # FP32 tier: growth of an accumulator's error through the HRRs and
        # transforms; a quartet whose error bound already exceeds the
        # tolerance stops its FP32 primitive loop (the final check rejects it)
        src.append('    const double famp = sizeof(R) == 4 ? %s : 0.0;' % self.amp_expr())
        src.append('    (void)famp;')
        src.append('    for (int ab0 = 0; ab0 < kab; ab0 += 64)')
        src.append('    for (int cd0 = 0; cd0 < kcd; cd0 += 64) {')
        src.append('      if (r < 32 && !pre) {')
        src += self.builder_lanes()
        src.append('        const int n0 = ib_live_pairs(a, g, 0, ab0, min(64, kab - ab0), lst, r, nbld, bmask, bbase);')
        src.append('        const int n1 = ib_live_pairs(a, g, 1, cd0, min(64, kcd - cd0), lst + 64, r, nbld, bmask, bbase);')
        src.append('        if (r == 0) { lcnt[0] = n0; lcnt[1] = n1; }')
        src.append('      }')
        src.append('      ib_sg_sync(SG, sg, sgmask);')
        src.append('      const int nl1 = lcnt[1], npl = lcnt[0] * nl1;')
        src.append('      const float rn1 = 1.0f / (float)max(nl1, 1);')
        if self.G == 1:
            # one lane per slice: every W-th live primitive quartet, set up in
            # registers; the bra pair is reused while it does not change
            src.append('      int ab_last = -1;')
            src.append('      IbBraPair bp;')
            src.append('      for (int u = w; u < npl; u += W) {')
            src.append('        const int qa = (int)(((float)u + 0.5f) * rn1), qc = u - qa * nl1;')
            src.append('        if (pre && ib_quartet_negligible(lst, qa, qc, a.prim_tol)) continue;')
            src.append('        const int ab = ab0 + lst[qa], cd = cd0 + lst[64 + qc];')
            src.append('        if (ab != ab_last) {')
            src.append('          const int ia = (int)(((float)ab + 0.5f) * rkb), ib = ab - ia * kb_;')
            src.append('          ib_bra_pair<sizeof(R) == 4>(a, g, ia, ib, bp);')
            src.append('          ab_last = ab;')
            src.append('        }')
            src.append('        const int ic = (int)(((float)cd + 0.5f) * rkd), id = cd - ic * kd_;')
            src.append('        IbPrimQuartet<R> pq;')
            src.append('        double F[%d];' % (L + 1))
            src.append('        if (!ib_prim_quartet<R, %d>(a, g, bp, ic, id, a.boys_tab, F, pq)) continue;' % L)
            src.append('        if (sizeof(R) == 4) {')
            src.append('          est += %s;' % self.err_expr())
            src.append('          if (est * famp > a.mixed_tol) break;  // this slice alone already exceeds it')
            src.append('        }')
            for f, nm in zip(fields, names):
                src.append('        const R %s = pq.%s;' % (nm, f))
            for m in range(L + 1):
                src.append('        const R f%d = (R)F[%d];' % (m, m))
        else:
            # lane j sets up live primitive quartet q0 + j of the chunk; the
            # group then sweeps the chunk reading the shared values (broadcast)
            sync = 'ib_group_bar(gid)' if self.smem_xfer else ('__syncwarp()' if self.dup else '__syncwarp(gmask)')
            # dup: every warp of the group sets up the same chunk of 32
            # primitive quartets for itself (its own slots of the table)
            CH = 32 if self.dup else self.G
            jl = 'jw' if self.dup else 'j'
            self.chunk = CH
            src.append('      for (int q0 = w * %d; q0 < npl; q0 += W * %d) {' % (CH, CH))
            src.append('        {')
            src.append('          const int q = q0 + %s;' % jl)
            src.append('          if (q < npl) {')
            src.append('            const int qa = (int)(((float)q + 0.5f) * rn1), qc = q - qa * nl1;')
            src.append('            const int ab = ab0 + lst[qa], cd = cd0 + lst[64 + qc];')
            src.append('            const int ia = (int)(((float)ab + 0.5f) * rkb), ib = ab - ia * kb_;')
            src.append('            const int ic = (int)(((float)cd + 0.5f) * rkd), id = cd - ic * kd_;')
            src.append('            IbBraPair bp;')
            src.append('            IbPrimQuartet<R> pq;')
            src.append('            double F[%d];' % (L + 1))
            src.append('            bool live = !(pre && ib_quartet_negligible(lst, qa, qc, a.prim_tol));')
            src.append('            if (live) {')
            src.append('              ib_bra_pair<sizeof(R) == 4>(a, g, ia, ib, bp);')
            src.append('              live = ib_prim_quartet<R, %d>(a, g, bp, ic, id, a.boys_tab, F, pq);' % L)
            src.append('            }')
            src.append('            if (live) {')
            for k, f in enumerate(fields):
                src.append('              ps[%d * %d + j] = pq.%s;' % (k, self.G, f))
            for m in range(L + 1):
                src.append('              ps[%d * %d + j] = (R)F[%d];' % (len(fields) + m, self.G, m))
            src.append('              if (sizeof(R) == 4) est += %s;' % self.err_expr())
            src.append('            }')
            src.append('            pz[j] = live ? 1 : 0;  // 0: pair prefactors multiply to zero, or screened out')
            # dup: sums of the bound run over this warp's setup lanes only (every
            # warp of the group set up the same primitive quartets)
            src.append('          }')
            src.append('        }')
            src.append('        %s;' % sync)
            # the group's bound so far (its lanes' partial sums): past the
            # tolerance, the rest of this quartet's FP32 work is skipped
            src.append('        if (sizeof(R) == 4) {')
            src.append('          double eg = est;')
            if self.packed:
                src.append('          sb[%d + j] = est;' % self.red_off)
                src.append('          __syncwarp(gmask);')
                src.append('          eg = 0.0;')
                src.append('          for (int v = 0; v < %d; ++v) eg += sb[%d + v];' % (self.G, self.red_off))
                src.append('          __syncwarp(gmask);')
            elif self.dup:
                src.append('          for (int o = 16; o > 0; o >>= 1) eg += __shfl_xor_sync(0xffffffffu, eg, o);')
            elif self.wide:
                src.append('          for (int o = 16; o > 0; o >>= 1) eg += __shfl_xor_sync(0xffffffffu, eg, o);')
                src.append('          if ((j & 31) == 0) sb[%d + (j >> 5)] = eg;' % self.red_off)
                src.append('          ib_group_bar(gid);')
                src.append('          eg = %s;' % ' + '.join('sb[%d]' % (self.red_off + w) for w in range(self.G // 32)))
                src.append('          ib_group_bar(gid);')
            else:
                src.append('          for (int o = %d; o > 0; o >>= 1) eg += __shfl_xor_sync(gmask, eg, o, %d);'
                           % (self.G // 2, self.G))
            src.append('          if (eg * famp > a.mixed_tol) break;  // uniform over the group')
            src.append('        }')
            src.append('        const int nu = min(%d, npl - q0);' % CH)
            ub = 'wq * 32 + u' if self.dup else 'u'
            src.append('        for (int u = 0; u < nu; ++u) {')
            src.append('          if (!pz[%s]) continue;  // group-uniform: exact-zero primitive quartet' % ub)
            for k, nm in enumerate(names):
                src.append('          const R %s = ps[%d * %d + %s];' % (nm, k, self.G, ub))
            for m in range(L + 1):
                src.append('        const R f%d = ps[%d * %d + %s];' % (m, len(fields) + m, self.G, ub))
        if bra:
            src.append('        const R SXx = PAx, SXy = PAy, SXz = PAz, SWx = WPx, SWy = WPy, SWz = WPz;')
            src.append('        const R so2 = o2z, sro = roz;')
            src.append('        const R CXx = QCx, CXy = QCy, CXz = QCz, CWx = WQx, CWy = WQy, CWz = WQz;')
            src.append('        const R co2 = o2e, cro = roe;')
        else:
            src.append('        const R SXx = QCx, SXy = QCy, SXz = QCz, SWx = WQx, SWy = WQy, SWz = WQz;')
            src.append('        const R so2 = o2e, sro = roe;')
            src.append('        const R CXx = PAx, CXy = PAy, CXz = PAz, CWx = WPx, CWy = WPy, CWz = WPz;')
            src.append('        const R co2 = o2z, cro = roz;')
        src.append('        const R tfx = (R)lcx * o2zpe, tfy = (R)lcy * o2zpe, tfz = (R)lcz * o2zpe;')
        src.append('        (void)tfx; (void)tfy; (void)tfz; (void)SXx; (void)SXy; (void)SXz; (void)SWx; (void)SWy;')
        src.append('        (void)SWz; (void)so2; (void)sro; (void)CXx; (void)CXy; (void)CXz; (void)CWx; (void)CWy;')
        src.append('        (void)CWz; (void)co2; (void)cro;')
        for m in range(L + 1):
            src.append('        R c1_%d = f%d, c2_%d = (R)0;' % (m, m, m))
        # base chain, the same S_hi steps on every lane (identity steps first
        # on lanes of a lower level: px = 1, wx = 0, nb = 0 keeps c1); the
        # first real step of a path has nb = 0, so the c2 it sees is unused
        for k in range(1, self.S_hi + 1):
            src.append('        {')
            src.append('          const unsigned st = lsteps >> %d;' % (5 * (k - 1)))
            src.append('          const int d = (int)(st & 3u);')
            src.append('          const R px = d == 0 ? SXx : (d == 1 ? SXy : (d == 2 ? SXz : (R)1));')
            src.append('          const R wx = d == 0 ? SWx : (d == 1 ? SWy : (d == 2 ? SWz : (R)0));')
            src.append('          const R nb = (R)(int)((st >> 2) & 7u) * so2;')
            for m in range(L - k + 1):
                src.append('          const R t%d = px * c1_%d + wx * c1_%d + nb * (c2_%d - sro * c2_%d);'
                           % (m, m, m + 1, m, m + 1))
            for m in range(L - k + 1):
                src.append('          c2_%d = c1_%d; c1_%d = t%d;' % (m, m, m, m))
            src.append('        }')
        for m in range(self.C_hi + 1):
            src.append('        const R b%d = c1_%d;' % (m, m))
        src += chain
        if self.G == 1:
            src.append('      }')
        else:
            src.append('        }')
            src.append('        %s;' % ('ib_group_bar(gid)' if self.smem_xfer else
                                        ('__syncwarp()' if self.dup else '__syncwarp(gmask)')))
            src.append('      }')
        src.append('      ib_sg_sync(SG, sg, sgmask);  // every slice is done with the lists before the next tile')
        src.append('    }')
        # FP32: sum the error bound over the group, reject the quartet if too large
        src.append('    if (sizeof(R) == 4) {')
        if self.packed:  # not a power of two: through shared memory
            src.append('      sb[%d + j] = est;' % self.red_off)
            src.append('      __syncwarp(gmask);')
            src.append('      est = 0.0;')
            src.append('      for (int v = 0; v < %d; ++v) est += sb[%d + v];' % (self.G, self.red_off))
            src.append('      __syncwarp(gmask);')
        elif self.G > 1 and not self.wide:
            src.append('      for (int o = %d; o > 0; o >>= 1) est += __shfl_xor_sync(gmask, est, o, %d);'
                       % (self.G // 2, self.G))
        elif self.dup:  # every warp holds the whole group's sum
            src.append('      for (int o = 16; o > 0; o >>= 1) est += __shfl_xor_sync(0xffffffffu, est, o);')
        elif self.wide:
            src.append('      for (int o = 16; o > 0; o >>= 1) est += __shfl_xor_sync(0xffffffffu, est, o);')
            src.append('      ib_group_bar(gid);')
            src.append('      if ((j & 31) == 0) sb[%d + (j >> 5)] = est;' % self.red_off)
            src.append('      ib_group_bar(gid);')
            src.append('      est = %s;' % ' + '.join('sb[%d]' % (self.red_off + w) for w in range(self.G // 32)))
            src.append('      ib_group_bar(gid);')
        pg = self.per_group
        src.append('      if (W > 1) {  // sum over the slices')
        src.append('        ib_sg_sync(SG, sg, sgmask);')
        src.append('        if (j == 0) sb[%d] = est;' % (pg - 1))
        src.append('        ib_sg_sync(SG, sg, sgmask);')
        src.append('        est = 0.0;')
        src.append('        for (int v = 0; v < W; ++v) est += sb0[v * %d + %d];' % (pg, pg - 1))
        src.append('      }')
        src.append('      if (est * famp > a.mixed_tol) {')
        src.append('        if (r == 0) a.flags[p] = 1;')
        src.append('        continue;  // uniform over the quartet: the FP64 pass recomputes and stores it')
        src.append('      }')
        src.append('    }')
        # accumulators -> shared [e][f]
        if self.dup:
            # the row of this lane's component; the low levels are written by
            # the group's first warp, padding lanes write nothing
            src.append('    {')
            src.append('      const int cx = lmisc & 7, cy = (lmisc >> 3) & 7, cz = (lmisc >> 6) & 7, cl = cx + cy + cz;')
            src.append('      const int crow = cl * (cl + 1) * (cl + 2) / 6 + cz + (cy + cz) * (cy + cz + 1) / 2;')
            src.append('      const bool mine = jw < %d ? wq == 0 : wq * %d + jw - %d < %d;'
                       % (self.nlow, self.per, self.nlow, self.ntop))
            src.append('      if (mine && crow >= %d) {' % s_lo_idx)
            for tt in range(NT):
                if bra:
                    src.append('        sb[(crow - %d) * %d + %d] = acc[%d];' % (s_lo_idx, NFP, tt, tt))
                else:
                    src.append('        sb[%d * %d + (crow - %d)] = acc[%d];' % (tt, NFP, s_lo_idx, tt))
            src.append('      }')
            src.append('    }')
        else:
            if bra:
                src.append('    if (j >= %d && j < %d) {' % (s_lo_idx, self.NL))
                for tt in range(NT):
                    src.append('      sb[(j - %d) * %d + %d] = acc[%d];' % (s_lo_idx, NFP, tt, tt))
            else:
                src.append('    if (j >= %d && j < %d) {' % (s_lo_idx, self.NL))
                for tt in range(NT):
                    src.append('      sb[%d * %d + (j - %d)] = acc[%d];' % (tt, NFP, s_lo_idx, tt))
            src.append('    }')
        src.append('    ib_sg_sync(SG, sg, sgmask);')
        src.append('    if (W > 1) {  // slice 0 table += the other slices tables')
        src.append('      for (int x = r; x < %d; x += SG) {' % (NE * NF))
        src.append('        const int o = (x / %d) * %d + x %% %d;' % (NF, NFP, NF))
        src.append('        double s = sb0[o];')
        src.append('        for (int v = 1; v < W; ++v) s += sb0[v * %d + o];' % self.per_group)
        src.append('        sb0[o] = s;')
        src.append('      }')
        src.append('      ib_sg_sync(SG, sg, sgmask);')
        src.append('    }')
        if self.lb or self.ld:
            # the contracted table is complete: estimate the HRRs' rounding
            # error from its largest element; a quartet over the tolerance is
            # recomputed by the generic kernel, which builds each primitive
            # pair on the shell that conditions its HRR (this kernel's result
            # is written all the same and overwritten then)
            src += self.hrr_check(NE, NF, NFP)
        src.append('    const double ABx = g.AB[0], ABy = g.AB[1], ABz = g.AB[2];')
        src.append('    const double CDx = g.CD[0], CDy = g.CD[1], CDz = g.CD[2];')
        src.append('    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;')
        src.append('    double* __restrict__ o = a.out + g.off;')
        src.append('    if (SPH) {')
        src += ['  ' + s for s in epi_sph]
        src.append('    } else {')
        src += ['  ' + s for s in epi_cart]
        src.append('    }')
        src.append('    ib_sg_sync(SG, sg, sgmask);')
        src.append('  }')
        src.append('}')
        src.append('')
        if self.wide:
            smem_bytes = '(sizeof(double) * (IB_BLOCK / %d) * %d)' % (self.G, per_group)
        else:
            smem_bytes = '(sizeof(double) * (IB_BLOCK / 32) * %d * %d)' % (self.QPW, per_group)
        src.append('static size_t ib_smem_%s() { return %s; }' % (t, smem_bytes))
        # variant = v4 + 4 * mi: v4 = precision x output (FP64/FP32 x Cartesian/
        # spherical), mi indexes the register budget IB_MINB[mi] (minimum
        # resident blocks per SM); classes outside the tuned set instantiate
        # mi = 0 only
        variants = (('double', 'false'), ('double', 'true'), ('float', 'false'), ('float', 'true'))
        if not fp32:
            variants = variants[:2] * 2
        minbs = list(range(len(MINB_VALUES))) if self.tuned else [0]
        cases = []
        for mi in range(len(MINB_VALUES)):
            for v, (R, S) in enumerate(variants):
                use = mi if mi in minbs else 0
                cases.append((v + 4 * mi, 'ib_eri_%s<%s, %s, %d>' % (t, R, S, MINB_VALUES[use])))
        src.append('static void ib_launch_%s(int variant, int grid, cudaStream_t s, const IbLaunch& a) {' % t)
        src.append('  const size_t smem = ib_smem_%s();' % t)
        src.append('  switch (variant) {')
        for v, fn in cases:
            src.append('    case %d: %s<<<grid, IB_BLOCK, smem, s>>>(a); break;' % (v, fn))
        src.append('  }')
        src.append('}')
        src.append('static int ib_occupancy_%s(int variant) {' % t)
        src.append('  int n = 0; const size_t smem = ib_smem_%s();' % t)
        src.append('  switch (variant) {')
        for v, fn in cases:
            src.append('    case %d: cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicSharedMemorySize, '
                       '(int)smem); cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, %s, IB_BLOCK, '
                       'smem); break;' % (v, fn, fn))
        src.append('  }')
        src.append('  return n;')
        src.append('}')
        src.append('')
        # the group barrier counts the group's G threads (named barrier gid + 1)
        src = [ln.replace('ib_group_bar(gid)', 'ib_group_bar(gid, %d)' % self.G) for ln in src]
        stats = dict(tag=t, cid=self.cid, L=L, kind='group', G=self.G, orient=self.orient, nodes=self.nvar,
                     lane_flops=self.flops, nacc=NE * NF)
        return '\n'.join(src), stats
