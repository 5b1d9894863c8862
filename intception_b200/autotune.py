"""Autotuner for the class kernels (run on the GPU the library will serve).

For every canonical class with l <= 2 (``--classes f``: every emitted class
whose largest l is 3, FP64 variants only, merged into the existing file) it
builds a batch of quartets of that class with the headline workload's
distribution (K uniform in 1..6 per shell,
exponents log-uniform [0.05, 1e4], centres in a 30-bohr cube, coefficients
normalised), times the batch with each register budget the library was
compiled with (``__launch_bounds__(IB_BLOCK, minb)``, minb in 1, 3, 4, 5 resident
blocks per SM) for each of the four variants (FP64/FP32 VRR x Cartesian/
spherical), and keeps the fastest.  The FP32 variants are timed with every
quartet in the FP32 tier and every result accepted, so that the FP32 kernel
itself is what is measured.

Output: ``intception_b200/tuning.json`` -- per class the chosen budget index
per variant (``minb``, indexes into (1, 3, 4, 5)), the chain emission order
(``order``) and the measured times.  ``python -m intception_b200.build`` bakes
it into the library (budgets as defaults, ``eri.set_class_minb`` overrides
them at run time; the order selects the emitted code).

The chain order changes the emitted code, so it is tuned across builds: build
and tune once per order (``INTCEPTION_B200_CHAIN_ORDER=dfs`` and ``=level``
set for both the build and the tuning run), then ``--merge`` the two files.

    python -m intception_b200.autotune [--nq 40000] [--reps 5] [--out PATH]
    python -m intception_b200.autotune --merge dfs.json level.json --out PATH
"""
import argparse
import json
import os
import time

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
MINB_VALUES = (1, 3, 4, 5)
VARIANTS = ('fp64_cart', 'fp64_sph', 'fp32_cart', 'fp32_sph')
FP32_GAIN = 0.97  # the FP32 kernel must be at least 3 % faster (rejected quartets are redone in FP64)


def class_batch(cls, nq, seed, spherical):
    """nq quartets of the shell-l pattern cls, each over four fresh shells."""
    from . import basis
    rng = np.random.default_rng(seed)
    ls = np.tile(np.asarray(cls, np.int32), nq)
    ks = rng.integers(1, 7, 4 * nq).astype(np.int32)
    l, k, ptr, xyz, e, c = basis.make_shells(rng, ls, ks, 0.05, 1.0e4, 30.0)
    q = np.arange(4 * nq, dtype=np.int32).reshape(nq, 4)
    off, total = basis.packed_offsets(l, q, spherical)
    return basis.ShellBatch(l, k, ptr, xyz, e, c, q, off, spherical, total)


def time_variant(eng, out, precision, reps, warmup=2):
    import torch
    from . import eri
    kw = {}
    if precision == eri.PREC_MIXED:
        kw = dict(bounds=eng._tune_bounds, skip_below=0.0, fp32_below=2.0, mixed_tol=1e300)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(warmup):
        eng.compute(out=out, precision=precision, **kw)
    ts = []
    for _ in range(reps):
        ev[0].record()
        eng.compute(out=out, precision=precision, **kw)
        ev[1].record()
        torch.cuda.synchronize()
        ts.append(ev[0].elapsed_time(ev[1]))
    assert eng.device_status() == 0
    return float(np.median(ts))


def tune(nq=40000, reps=5, classes=None, log=print):
    import torch
    from . import eri
    from .emit.eri_emitter import canonical_classes
    torch.cuda.set_device(0)
    from .emit.eri_emitter import emitted_classes
    classes = classes or canonical_classes(2)
    has_fp32 = {c for c, f in emitted_classes() if f}
    result = {}
    for cls in classes:
        tag = '%d%d%d%d' % tuple(cls)
        ent = {'minb': [0, 0, 0, 0], 'ms': {}}
        precs = (eri.PREC_FP64, eri.PREC_MIXED) if tuple(cls) in has_fp32 else (eri.PREC_FP64,)
        for sph in (False, True):
            b = class_batch(cls, nq, seed=1000 + eri.class_id(*cls), spherical=sph)
            eng = eri.EriEngine(b)
            eng._tune_bounds = torch.ones(b.nq, dtype=torch.float64, device='cuda')
            out = torch.empty(b.out_size, dtype=torch.float64, device='cuda')
            for prec in precs:
                v4 = (2 if prec == eri.PREC_MIXED else 0) + (1 if sph else 0)
                times = []
                for mi, mb in enumerate(MINB_VALUES):
                    eri.set_class_minb(cls, v4, mb)
                    times.append(time_variant(eng, out, prec, reps))
                best = int(np.argmin(times))
                eri.set_class_minb(cls, v4, MINB_VALUES[best])
                ent['minb'][v4] = best
                ent['ms'][VARIANTS[v4]] = [round(t, 4) for t in times]
            del eng, out
        # the FP32 tier uses this class's FP32 kernel only where it beats FP64
        if len(precs) == 2:
            ent['fp32'] = bool(min(ent['ms']['fp32_sph']) < FP32_GAIN * min(ent['ms']['fp64_sph']) and
                               min(ent['ms']['fp32_cart']) < FP32_GAIN * min(ent['ms']['fp64_cart']))
        else:  # FP64 kernels only: the FP32 slots take the FP64 choice
            ent['minb'][2], ent['minb'][3] = ent['minb'][0], ent['minb'][1]
            ent['fp32'] = False
        result[tag] = ent
        log('%s %s fp32:%s' % (tag, ' '.join('%s:%s' % (VARIANTS[v], MINB_VALUES[ent['minb'][v]]) for v in range(4)),
                               ent['fp32']))
    return result


def merge(paths, out):
    """Combine tuning runs made with different chain orders (one build per
    order, INTCEPTION_B200_CHAIN_ORDER=dfs|level): per class the order whose
    kernels were fastest over the four variants (each at its best budget), and
    that run's budgets."""
    runs = []
    for p in paths:
        with open(p) as fh:
            runs.append(json.load(fh))
    classes = {}
    for tag in runs[0]['classes']:
        best = None
        for r in runs:
            ent = r['classes'][tag]
            cost = sum(min(v) for v in ent['ms'].values())
            if best is None or cost < best[0]:
                best = (cost, r, ent)
        ent = dict(best[2])
        ent['order'] = best[1]['meta']['chain_order']
        ms = ent['ms']
        ent['fp32'] = bool(min(ms['fp32_sph']) < FP32_GAIN * min(ms['fp64_sph']) and
                           min(ms['fp32_cart']) < FP32_GAIN * min(ms['fp64_cart']))
        ent['ms_by_order'] = {r['meta']['chain_order']: round(sum(min(v) for v in r['classes'][tag]['ms'].values()), 4)
                              for r in runs}
        classes[tag] = ent
    meta = dict(runs[0]['meta'])
    meta['chain_order'] = 'per class (merged: %s)' % ', '.join(r['meta']['chain_order'] for r in runs)
    with open(out, 'w') as fh:
        json.dump({'meta': meta, 'classes': classes}, fh, indent=1)
    return classes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--nq', type=int, default=40000)
    ap.add_argument('--reps', type=int, default=5)
    ap.add_argument('--out', default=os.path.join(PKG, 'tuning.json'))
    ap.add_argument('--classes', default='l2', choices=['l2', 'f'],
                    help='l2: every class with l <= 2 (writes --out); f: the emitted classes whose largest l is 3, '
                         'FP64 only, merged into --out')
    ap.add_argument('--merge', nargs='+', default=None,
                    help='combine tuning files of builds with different chain orders into --out (no GPU)')
    a = ap.parse_args()
    if a.merge:
        merge(a.merge, a.out)
        print('wrote', a.out)
        return
    import torch
    t0 = time.time()
    if a.classes == 'f':
        from .emit.eri_emitter import emitted_classes
        # canonical orders only: a (d f| pair is canonicalised to (f d| by the batch
        # entry, so its reversed class kernels (ill-conditioned pairs) keep the default
        fcls = [c for c, _ in emitted_classes() if max(c) == 3 and c[0] >= c[1] and c[2] >= c[3]]
        res = tune(a.nq, a.reps, classes=fcls)
        with open(a.out) as fh:
            cur = json.load(fh)
        for tag, ent in res.items():
            ent.setdefault('order', cur['classes'].get(tag, {}).get('order', 'dfs'))
            cur['classes'][tag] = ent
        cur['meta']['f_classes'] = {'nq_per_class': a.nq, 'reps': a.reps, 'seconds': round(time.time() - t0, 1),
                                    'variants': 'FP64 Cartesian and spherical'}
        with open(a.out, 'w') as fh:
            json.dump(cur, fh, indent=1)
        print('merged', len(res), 'f classes into', a.out)
        return
    res = tune(a.nq, a.reps)
    meta = {'device': torch.cuda.get_device_name(0), 'nq_per_class': a.nq, 'reps': a.reps,
            'minb_values': list(MINB_VALUES), 'variants': list(VARIANTS),
            'workload': 'per class: K uniform 1..6, alpha log-uniform [0.05,1e4], 30-bohr cube, seed 1000+cid',
            'chain_order': os.environ.get('INTCEPTION_B200_CHAIN_ORDER', 'as built'),
            'seconds': round(time.time() - t0, 1)}
    with open(a.out, 'w') as fh:
        json.dump({'meta': meta, 'classes': res}, fh, indent=1)
    print('wrote', a.out)


if __name__ == '__main__':
    main()
