"""Benchmark: contracted ERI quartets/s on one B200 (or N, weak scaling).

Workload (one step = one pass of the ERI path over one batch):
  1e6 shell quartets, l in {0,1,2} per shell (class uniform over the 81
  (la,lb,lc,ld) classes), K uniform in {1..6} per shell, exponents log-uniform
  in [0.05, 1e4], coefficients uniform [0.1, 1] then normalised, centres
  uniform in a 30-bohr cube, spherical output, seed 1 (rank r uses seed 1+r).
  Synthetic data with the shapes of that configuration.

--workload nuclear_2idx | overlap_2idx times the reference example script's
two-index classes instead (4e6 primitive pairs, l <= 2; one launch per step).

Arms:
  default          : this library, FP64 path and mixed-precision path
  --impl reference : the reference's own CPU implementation of the path (the
                     C99 its generator emits, oracle/_ref, OpenMP over the
                     box's cores) on a bounded sample of the same workload.

Prints one JSON line (rank 0).  value = quartets/s of the headline path over
all ranks, device-timed with inputs resident in HBM (inputs + outputs ~1 GB,
larger than L2, so no flush is needed); e2e = the same through the public API
with host buffers and the H2D/D2H copies inside the timed region.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'contracted ERI quartets/s on B200: mixed-prec vs FP64 at <=1e-10 max abs err'
WORKLOAD = ('1e6 quartets, l<=2 per shell (81 classes uniform), K in 1..6, alpha log-uniform [0.05,1e4], '
            '30-bohr cube, spherical, seed 1')
SKIP_BELOW = 1e-12      # Schwarz screening: blocks with a smaller bound are written as zeros
FP32_BELOW = 1e-4       # mixed path: FP32 VRR attempted below this bound ...
MIXED_TOL = 5e-11       # ... and kept only where its rounding-error bound is below this; else FP64
PRIM_TOL = 1e-18        # screened paths: primitive quartets with Q_ab Q_cd below this skipped
FP32_SWEEP = (0.0, 1e-10, 1e-8, 1e-6, 1e-4)  # candidate FP32-tier bounds (0 = tier off), tuned per run
FP32_CHOSEN = [0.0]
ERR_BAR = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--nq', type=int, default=1_000_000)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-mixed', action='store_true')
    ap.add_argument('--cpu-seconds', type=float, default=15.0)
    ap.add_argument('--workload', default='eri', choices=['eri', 'nuclear_2idx', 'overlap_2idx', 'lattice_l3'],
                    help='eri: the headline; *_2idx: the example script\'s two-index classes; lattice_l3: '
                         'a sample of the 200-atom l <= 3 lattice\'s screened quartets')
    ap.add_argument('--npairs', type=int, default=4_000_000)
    ap.add_argument('--nq-lattice', type=int, default=2_000_000)
    ap.add_argument('--only', default=None, choices=['fp64', 'screened', 'screened_prim'],
                    help='profiling: run only this ERI step (W warm-up + K timed) and print its time')
    return ap.parse_args()


def dist_init(n):
    import torch
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm)}


def live_pairs(batch, i, j):
    """Per quartet, primitive pairs of shells (i, j) with c_a c_b exp(-xi R^2) != 0."""
    sa, sb = batch.quartets[:, i], batch.quartets[:, j]
    ka, kb = batch.shell_k[sa], batch.shell_k[sb]
    pa, pb = batch.shell_ptr[sa], batch.shell_ptr[sb]
    r2 = ((batch.shell_xyz[sa] - batch.shell_xyz[sb]) ** 2).sum(axis=1)
    n = np.zeros(batch.nq, dtype=np.int64)
    for u in range(int(ka.max())):
        for v in range(int(kb.max())):
            ok = (u < ka) & (v < kb)
            ea = batch.prim_exp[np.where(ok, pa + u, 0)]
            eb = batch.prim_exp[np.where(ok, pb + v, 0)]
            ca = batch.prim_coef[np.where(ok, pa + u, 0)]
            cb = batch.prim_coef[np.where(ok, pb + v, 0)]
            with np.errstate(under='ignore', over='ignore'):
                kab = ca * cb * np.exp(-ea * eb / (ea + eb) * r2)
            n += (ok & (kab != 0.0)).astype(np.int64)
    return n


def alg_flops(batch):
    """Algorithmic FP64 work of one step: per live primitive quartet the
    canonical VRR count plus 74 + 2L for geometry and Boys; per quartet the HRR
    and the spherical transform counts; from the emitter's per-class table."""
    with open(os.path.join(ROOT, 'intception_b200', 'class_stats.json')) as fh:
        stats = {s['cid']: s for s in json.load(fh)}
    ls = batch.shell_l[batch.quartets].astype(np.int64)
    ks = batch.shell_k[batch.quartets].astype(np.int64)
    # canonical class id, as the device computes it
    la, lb, lc, ld = ls.T.copy()
    sw = la < lb
    la[sw], lb[sw] = lb[sw], la[sw].copy()
    sw = lc < ld
    lc[sw], ld[sw] = ld[sw], lc[sw].copy()
    pb = la * (la + 1) // 2 + lb
    pk = lc * (lc + 1) // 2 + ld
    sw = pb < pk
    pb2 = np.where(sw, pk, pb)
    pk2 = np.where(sw, pb, pk)
    cid = pb2 * (pb2 + 1) // 2 + pk2
    # primitive quartets whose prefactor is not exactly zero (the kernels skip
    # the others bit-exactly, so they are not work an algorithm must do)
    nprim = live_pairs(batch, 0, 1) * live_pairs(batch, 2, 3)
    ncls = max(stats) + 1
    vrr = np.array([stats[c]['vrr_flops'] + 74 + 2 * stats[c]['L'] if c in stats else 0 for c in range(ncls)])
    hrr = np.array([stats[c]['hrr_flops'] + (stats[c]['sph_flops'] if batch.spherical else 0) if c in stats else 0
                    for c in range(ncls)])
    return float((nprim * vrr[cid] + hrr[cid]).sum()), cid


def cpu_reference(batch, seconds, step_index=0):
    """Time the reference's emitted C99 (oracle/_ref) -- or, when it was not
    built, the oracle port -- on all host cores over a bounded sample.
    Returns (quartets/s, kind, cores, sample description)."""
    from intception_b200 import basis
    from oracle import loader
    T = basis.sph_matrices(6)
    cores = os.cpu_count() or 1
    lib = loader.load_ref('sph' if batch.spherical else 'cart')
    kind = 'reference' if lib is not None else 'port'
    rng = np.random.default_rng(99 + step_index)

    def run(n):
        idx = rng.choice(batch.nq, n, replace=False)
        sub = batch.subset(np.sort(idx))
        t0 = time.perf_counter()
        if lib is not None:
            loader.ref_batch(sub, T, nthreads=cores)
        else:
            loader.oracle_batch(sub, T)
        return time.perf_counter() - t0

    n = 2000
    dt = run(n)
    n2 = int(min(batch.nq, max(n, n * seconds / max(dt, 1e-3))))
    dt2 = run(n2)
    used = cores if lib is not None else 1
    return n2 / dt2, kind, used, '%d random quartets of the workload (uniform sample)' % n2


def run_reference_arm(args, rank, world):
    from intception_b200 import basis
    if rank != 0:
        return
    batch = basis.config_mixed_l2(nq=args.nq, seed=1, spherical=True)
    vals = []
    for i in range(args.warmup + args.steps):
        v, kind, cores, sample = cpu_reference(batch, max(2.0, args.cpu_seconds / 3), i)
        if i >= args.warmup:
            vals.append(v)
    v = float(np.median(vals))
    line = {'metric': METRIC, 'value': v, 'unit': 'quartets/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * args.nq / v, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': WORKLOAD, 'nq': args.nq, 'parallelism': 'openmp host cores'},
            'impl': 'reference',
            'cpu_baseline': {'value': v, 'unit': 'quartets/s', 'cores': cores, 'kind': kind, 'sample': sample},
            'e2e': {'value': v, 'unit': 'quartets/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


TWOIDX_METRIC = 'primitive %s pair blocks/s (example_input.py class, l<=2)'
LATTICE_WORKLOAD = ('200-atom jittered cubic lattice (2.6-bohr spacing, +-0.3 bohr jitter), per atom s(K=6) s(K=3) '
                    'p(K=3) d(K=1) f(K=1), alpha log-uniform [0.1,1e3], seed 2; unique quartets with Schwarz bound '
                    '>= 1e-12; a uniform sample of %d of them, spherical')


def lattice_batch(nq, seed=2):
    """The 200-atom l <= 3 lattice: shells, Schwarz factors of every shell pair
    (on the GPU), and a uniform sample of nq of the unique quartets whose bound
    reaches 1e-12.  Returns (batch, number of such quartets)."""
    import torch
    from intception_b200 import basis, eri
    rng, l_, k_, p_, cxyz, e, c = basis.lattice_shells(seed=seed)
    a, b = np.tril_indices(len(l_))
    pairs = np.stack([a, b], axis=1).astype(np.int32)
    one = np.zeros((1, 4), np.int32)
    off1, tot1 = basis.packed_offsets(l_, one, True)
    b0 = basis.ShellBatch(l_, k_, p_, cxyz, e, c, one, off1, True, tot1)
    q = eri.EriEngine(b0).schwarz(torch.from_numpy(pairs).cuda()).cpu().numpy()
    quartets, total = basis.sample_screened_quartets(q, pairs, nq, rng, SKIP_BELOW)
    off, tot = basis.packed_offsets(l_, quartets, True)
    return basis.ShellBatch(l_, k_, p_, cxyz, e, c, quartets, off, True, tot), total


def run_lattice(args, rank, world, local):
    """The lattice sample: FP64 exact, FP64 with primitive screening, and the
    precision tiers (FP32 VRR below bound 1e-4, its error bound checked), one
    JSON line; value = the fastest path within 1e-10 of exact FP64."""
    import torch
    from intception_b200 import eri
    batch, total = lattice_batch(args.nq_lattice)
    eng = eri.EriEngine(batch)
    out = torch.empty(batch.out_size, dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        assert eng.device_status() == 0
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)

    clk = ClockSampler(local).__enter__()
    eri.set_prim_tol(0.0)
    ms64 = timed(lambda: eng.compute(out=out))
    ref = out.clone()
    bounds = eng.quartet_bounds()
    eri.set_prim_tol(PRIM_TOL)
    msp = timed(lambda: eng.compute(out=out, bounds=bounds, skip_below=SKIP_BELOW))
    errp = max_over_ranks(float((out - ref).abs().max().item()), world)
    msm = timed(lambda: eng.compute(out=out, precision=eri.PREC_MIXED, bounds=bounds, skip_below=SKIP_BELOW,
                                    fp32_below=FP32_BELOW, mixed_tol=MIXED_TOL))
    errm = max_over_ranks(float((out - ref).abs().max().item()), world)
    rej = eng.fp32_rejected()
    nfp32 = int((bounds < FP32_BELOW).sum().item())
    launches = eri.EriEngine.last_launch_count()
    eri.set_prim_tol(0.0)
    clk.__exit__(None, None, None)
    cands = [(ms64, 0.0, 'fp64'), (msp, errp, 'fp64 + primitive screening'), (msm, errm, 'precision tiers')]
    ok = [c for c in cands if c[1] <= ERR_BAR] or cands
    ms, err, path = min(ok)
    nq = batch.nq * world
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference(batch, args.cpu_seconds)
        cpu = {'value': v, 'unit': 'quartets/s', 'cores': cores, 'kind': kind, 'sample': sample}
    if rank == 0:
        print(json.dumps({
            'metric': 'contracted ERI quartets/s on B200, 200-atom l<=3 lattice (screened quartets, sample)',
            'value': nq / (ms * 1e-3), 'unit': 'quartets/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64+f32' if path == 'precision tiers' else 'f64', 'data': 'synthetic',
            'config': {'workload': LATTICE_WORKLOAD % batch.nq, 'screened_quartets_total': total,
                       'headline_path': path, 'prim_tol': PRIM_TOL, 'fp32_below': FP32_BELOW,
                       'mixed_tol': MIXED_TOL, 'l2': 'outputs %.0f MB per step, larger than L2; no flush'
                       % (batch.out_size * 8 / 1e6)},
            'max_abs_err_vs_fp64': err,
            'fp64': {'ms_per_step': ms64, 'value': nq / (ms64 * 1e-3), 'note': 'exact, no screening'},
            'fp64_prim': {'ms_per_step': msp, 'max_abs_err_vs_fp64': errp},
            'mixed': {'ms_per_step': msm, 'max_abs_err_vs_fp64': errm, 'fp32_attempted': nfp32,
                      'fp32_rejected': rej},
            'estimated_full_lattice_s': total / (nq / (ms * 1e-3)),
            'cpu_baseline': cpu, 'gpu_launches': launches * args.steps, 'clocks': clk.summary()}), flush=True)


TWOIDX_WORKLOAD = ('%d primitive pairs%s, la and lb uniform in 0..2, alpha log-uniform [0.05,1e4], A in a 30-bohr '
                   'cube, B%s within 2 bohr of A, seed 1')


def twoidx_cpu(kind, pairs, seconds, step_index=0):
    """The reference's emitted C99 of the example classes (oracle/_ref,
    OpenMP) -- or the oracle port when it was not built -- over a bounded
    random sample of the pairs.  Returns (pairs/s, kind, cores, sample)."""
    from intception_b200 import twoidx
    from oracle import loader
    lib = loader.load_ref_2idx()
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(77 + step_index)
    n_all = len(pairs['la'])

    def run(n):
        idx = np.sort(rng.choice(n_all, n, replace=False))
        sub = {k: np.asarray(pairs[k])[idx] for k in ('xa', 'ca', 'la', 'xb', 'cb', 'lb', 'cc')}
        sub['off'], sub['size'] = twoidx.block_offsets(sub['la'], sub['lb'])
        t0 = time.perf_counter()
        loader.twoidx_batch(kind, sub, lib)
        return time.perf_counter() - t0

    n = 20000
    dt = run(n)
    n2 = int(min(n_all, max(n, n * seconds / max(dt, 1e-3))))
    dt2 = run(n2)
    return (n2 / dt2, 'reference' if lib is not None else 'port', cores if lib is not None else 1,
            '%d random pairs of the workload (uniform sample)' % n2)


def run_twoidx(args, rank, world, local):
    """Two-index workload: one step = one launch over every pair."""
    import torch
    from intception_b200 import eri, twoidx
    kind = twoidx.NUCLEAR if args.workload == 'nuclear_2idx' else twoidx.OVERLAP
    name = 'nuclear-attraction' if kind == twoidx.NUCLEAR else 'overlap'
    workload = TWOIDX_WORKLOAD % (args.npairs, ' x one point charge' if kind == twoidx.NUCLEAR else '',
                                  ' and the charge' if kind == twoidx.NUCLEAR else '')
    pairs = twoidx.make_pairs(args.npairs, 2, seed=1 + rank)
    if args.impl == 'reference':
        if rank != 0:
            return
        vals = []
        for i in range(args.warmup + args.steps):
            v, ckind, cores, sample = twoidx_cpu(kind, pairs, max(2.0, args.cpu_seconds / 3), i)
            if i >= args.warmup:
                vals.append(v)
        v = float(np.median(vals))
        line = {'metric': TWOIDX_METRIC % name, 'value': v, 'unit': 'pairs/s', 'n_gpus': args.gpus,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * args.npairs / v,
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic', 'config': {'workload': workload, 'parallelism': 'openmp host cores'},
                'impl': 'reference',
                'cpu_baseline': {'value': v, 'unit': 'pairs/s', 'cores': cores, 'kind': ckind, 'sample': sample},
                'e2e': {'value': v, 'unit': 'pairs/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line), flush=True)
        return
    batch = twoidx.TwoIndexBatch(pairs)
    out = torch.empty(batch.size, dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        assert batch.device_status() == 0
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)

    clk = ClockSampler(local).__enter__()
    ms = timed(lambda: batch.compute(kind, out=out))
    value = args.npairs * world / (ms * 1e-3)
    # roofline: algorithmic bytes and flops of the step, against measured HBM and FP64 peaks
    cost = {(a, b): twoidx.algorithmic_cost(kind, a, b) for a in range(3) for b in range(3)}
    cls = pairs['la'].astype(np.int64) * 3 + pairs['lb']
    counts = np.bincount(cls, minlength=9)
    flops = float(sum(counts[a * 3 + b] * cost[(a, b)][0] for a in range(3) for b in range(3)))
    nbytes = float(sum(counts[a * 3 + b] * cost[(a, b)][1] for a in range(3) for b in range(3)))
    with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
        hbm = json.load(fh)['hbm_gbs'] * 1e9
    peak64 = eri.fma_peak(True) if rank == 0 else 0.0
    t_hbm, t_fp = nbytes / hbm, flops / peak64 if peak64 else 0.0
    bound = 'hbm' if t_hbm >= t_fp else 'fp64'
    achieved = (nbytes if bound == 'hbm' else flops) / (ms * 1e-3)
    peak = hbm if bound == 'hbm' else peak64
    roofline = {'bound': bound, 'achieved': achieved / (1e9 if bound == 'hbm' else 1e12),
                'peak': peak / (1e9 if bound == 'hbm' else 1e12), 'unit': 'GB/s' if bound == 'hbm' else 'TFLOP/s',
                'frac': achieved / peak, 'traffic': None,
                'peak_source': 'hbm: MEASURED_PEAKS.json hbm_gbs; fp64: intception_b200_fma_peak this run',
                'kernel': 'ib2_%s_kernel' % ('nuclear' if kind == twoidx.NUCLEAR else 'overlap'),
                'alg_bytes_per_step': nbytes, 'alg_flops_per_step': flops,
                'fp64_frac': (flops / (ms * 1e-3)) / peak64 if peak64 else None}
    prof = os.path.join(ROOT, 'profiles', 'traffic_%s.json' % args.workload)
    if os.path.exists(prof):
        with open(prof) as fh:
            roofline['traffic'] = json.load(fh).get('bytes_per_step')
    # e2e: host inputs -> device, the launch, the blocks back to host
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_in = [pin(batch.xa.cpu()), pin(batch.ca.cpu()), pin(batch.la.cpu()), pin(batch.xb.cpu()),
            pin(batch.cb.cpu()), pin(batch.lb.cpu()), pin(batch.off.cpu())]
    d_in = [batch.xa, batch.ca, batch.la, batch.xb, batch.cb, batch.lb, batch.off]
    if kind == twoidx.NUCLEAR:
        h_in.append(pin(batch.cc.cpu()))
        d_in.append(batch.cc)
    h_out = torch.empty(batch.size, dtype=torch.float64).pin_memory()

    def e2e_step():
        for h, d in zip(h_in, d_in):
            d.copy_(h, non_blocking=True)
        batch.compute(kind, out=out)
        h_out.copy_(out, non_blocking=True)

    mse = timed(e2e_step)
    e2e = {'value': args.npairs * world / (mse * 1e-3), 'unit': 'pairs/s',
           'h2d_bytes_per_step': sum(t.numel() * t.element_size() for t in h_in),
           'd2h_bytes_per_step': h_out.numel() * 8, 'ms_per_step': mse}
    clk.__exit__(None, None, None)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, ckind, cores, sample = twoidx_cpu(kind, pairs, args.cpu_seconds)
        cpu = {'value': v, 'unit': 'pairs/s', 'cores': cores, 'kind': ckind, 'sample': sample}
    if rank == 0:
        line = {'metric': TWOIDX_METRIC % name, 'value': value, 'unit': 'pairs/s', 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'config': {'workload': workload, 'npairs_per_gpu': args.npairs,
                           'l2': 'inputs+outputs %.0f MB per step, larger than L2; no flush' % (nbytes / 1e6)},
                'roofline': roofline, 'cpu_baseline': cpu, 'e2e': e2e,
                'gpu_launches': args.steps, 'gpu_launches_per_step': 1, 'clocks': clk.summary()}
        print(json.dumps(line), flush=True)


def run_only(args, eng, out):
    """One step kind alone (for profilers): the FP64 step over every quartet,
    or the screened FP64 step (bounds computed first, outside the timing)."""
    import torch
    from intception_b200 import eri
    bounds, skip = None, 0.0
    if args.only in ('screened', 'screened_prim'):
        bounds, skip = eng.quartet_bounds(), SKIP_BELOW
    eri.set_prim_tol(PRIM_TOL if args.only == 'screened_prim' else 0.0)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        eng.compute(out=out, bounds=bounds, skip_below=skip)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        eng.compute(out=out, bounds=bounds, skip_below=skip)
    ev1.record()
    torch.cuda.synchronize()
    assert eng.device_status() == 0
    print(json.dumps({'only': args.only, 'nq': args.nq, 'steps': args.steps, 'warmup': args.warmup,
                      'ms_per_step': ev0.elapsed_time(ev1) / args.steps,
                      'kernels_per_step': eri.EriEngine.last_launch_count()}), flush=True)


def main():
    args = parse()
    if args.impl == 'reference':
        # host cores only: no process group; rank 0 runs the reference, the
        # other ranks of a multi-GPU launch exit at once
        rank, world = int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1'))
        if args.workload == 'lattice_l3':
            if rank == 0:  # the sample is drawn with the GPU's Schwarz factors; its line carries cpu_baseline
                print(json.dumps({'impl': 'reference', 'unavailable': 'lattice_l3 draws its quartet sample with '
                                  'GPU Schwarz factors; the reference C99 is timed in that line\'s cpu_baseline'}))
            return
        if args.workload != 'eri':
            run_twoidx(args, rank, world, 0)
        else:
            run_reference_arm(args, rank, world)
        return
    rank, world, local = dist_init(args.gpus)
    if args.workload == 'lattice_l3':
        run_lattice(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload != 'eri':
        run_twoidx(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from intception_b200 import basis, eri
    batch = basis.config_mixed_l2(nq=args.nq, seed=1 + rank, spherical=True)
    eng = eri.EriEngine(batch)
    stream = torch.cuda.current_stream()
    out = torch.empty(batch.out_size, dtype=torch.float64, device='cuda')
    if args.only:
        run_only(args, eng, out)
        return

    def step(precision=eri.PREC_FP64, bounds=None, skip=0.0):
        eng.compute(out=out, precision=precision, bounds=bounds, skip_below=skip, fp32_below=FP32_BELOW,
                    mixed_tol=MIXED_TOL)

    def timed(fn, clocks=None):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        assert eng.device_status() == 0
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # ---------------- FP64 path, every quartet evaluated, device-resident inputs
    clk = ClockSampler(local).__enter__()  # sampled over every timed region below
    ms64 = timed(step)
    launches = eri.EriEngine.last_launch_count()
    value64 = args.nq * world / (ms64 * 1e-3)
    ref64 = out.clone()

    # ---------------- Schwarz bounds (per shell pair, once per basis), then the screened paths
    mixed = None
    screened = None
    screened_prim = None
    if not args.no_mixed:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bounds = eng.quartet_bounds()
        e1.record(stream)
        torch.cuda.synchronize()
        schwarz_ms = e0.elapsed_time(e1)
        n_kept = int((bounds >= SKIP_BELOW).sum().item())
        ms_s = timed(lambda: step(eri.PREC_FP64, bounds, SKIP_BELOW))
        err_s = max_over_ranks(float((out - ref64).abs().max().item()), world)
        screened = {'value': args.nq * world / (ms_s * 1e-3), 'ms_per_step': ms_s, 'max_abs_err_vs_fp64': err_s,
                    'screened_quartets_per_s': n_kept * world / (ms_s * 1e-3)}
        # primitive screening on top (kept for every path below): a primitive
        # quartet whose Schwarz-type bound Q_ab Q_cd is below PRIM_TOL moves
        # no element by more than PRIM_TOL, so a block by at most K^4 PRIM_TOL
        eri.set_prim_tol(PRIM_TOL)
        ms_p = timed(lambda: step(eri.PREC_FP64, bounds, SKIP_BELOW))
        err_p = max_over_ranks(float((out - ref64).abs().max().item()), world)
        screened_prim = {'value': args.nq * world / (ms_p * 1e-3), 'ms_per_step': ms_p, 'max_abs_err_vs_fp64': err_p,
                         'prim_tol': PRIM_TOL, 'error_bound_per_element': 1296 * PRIM_TOL,
                         'screened_quartets_per_s': n_kept * world / (ms_p * 1e-3)}
        # precision tiers: zeros below SKIP_BELOW, FP32 VRR (with its rounding-error
        # bound, rejected quartets redone in FP64) below fp32_below, FP64 above.
        # fp32_below is tuned here; 0 switches the FP32 tier off.
        sweep = []
        for fb in FP32_SWEEP:
            mode = eri.PREC_MIXED if fb > 0 else eri.PREC_FP64
            msx = timed(lambda: eng.compute(out=out, precision=mode, bounds=bounds, skip_below=SKIP_BELOW,
                                            fp32_below=fb, mixed_tol=MIXED_TOL))
            errx = max_over_ranks(float((out - ref64).abs().max().item()), world)
            nf = int(((bounds >= SKIP_BELOW) & (bounds < fb)).sum().item()) if fb > 0 else 0
            rej = eng.fp32_rejected() if fb > 0 else 0
            sweep.append({'fp32_below': fb, 'ms_per_step': msx, 'max_abs_err_vs_fp64': errx,
                          'fp32_attempted': nf, 'fp32_rejected': rej})
        ok = [r for r in sweep if r['max_abs_err_vs_fp64'] <= ERR_BAR] or sweep
        best = min(ok, key=lambda r: r['ms_per_step'])
        fb = best['fp32_below']
        msmx = best['ms_per_step']
        err = best['max_abs_err_vs_fp64']
        mixed = {'value': args.nq * world / (msmx * 1e-3), 'ms_per_step': msmx, 'max_abs_err_vs_fp64': err,
                 'screened_quartets_per_s': n_kept * world / (msmx * 1e-3),
                 'kept_fraction': n_kept / args.nq, 'skip_below': SKIP_BELOW, 'prim_tol': PRIM_TOL, 'fp32_below': fb,
                 'mixed_tol': MIXED_TOL, 'fp32_tier_active': fb > 0, 'fp32_sweep': sweep,
                 'schwarz_ms': schwarz_ms, 'schwarz_note': 'per-pair Schwarz factors, computed once per basis '
                 'on the GPU (intception_b200_schwarz), outside the timed step; this workload has no pair reuse'}
        FP32_CHOSEN[0] = fb

    headline_mixed = mixed is not None and mixed['max_abs_err_vs_fp64'] <= ERR_BAR
    # the headline configuration replayed from a CUDA graph (sort, items, class
    # kernels and their side-stream fork/join captured once)
    if headline_mixed:
        fb = FP32_CHOSEN[0]
        graph = eng.graph(out, precision=eri.PREC_MIXED if fb > 0 else eri.PREC_FP64, bounds=bounds,
                          skip_below=SKIP_BELOW, fp32_below=fb, mixed_tol=MIXED_TOL)
    else:
        graph = eng.graph(out)
    ms_graph = timed(graph.launch)
    launches = eri.EriEngine.last_launch_count()  # kernels of one replayed step of the headline path
    err_graph = max_over_ranks(float((out - ref64).abs().max().item()), world)
    graph.close()
    if headline_mixed:
        mixed['graph_ms_per_step'] = ms_graph
        mixed['graph_max_abs_err_vs_fp64'] = err_graph
        # the tuned tier path, measured three ways: the sweep's best setting,
        # its graph replay, and (FP32 tier off) the screened FP64 run above
        cands = [mixed['ms_per_step'], ms_graph]
        if FP32_CHOSEN[0] == 0 and screened_prim is not None:
            cands.append(screened_prim['ms_per_step'])
        ms = min(cands)
        value = args.nq * world / (ms * 1e-3)
    else:
        ms = min(ms64, ms_graph)
        value = args.nq * world / (ms * 1e-3)

    # ---------------- roofline of the FP64 step against the measured FP64 FMA peak
    flops, _ = alg_flops(batch)
    peak64 = eri.fma_peak(True) if rank == 0 else 0.0
    achieved = flops / (ms64 * 1e-3)
    roofline = {'bound': 'fp64', 'achieved': achieved / 1e12, 'peak': peak64 / 1e12, 'unit': 'TFLOP/s',
                'frac': achieved / peak64 if peak64 else None, 'traffic': None,
                'peak_source': 'measured FP64 FMA-chain kernel (intception_b200_fma_peak), this run',
                'kernel': 'whole FP64 step (per-class kernels run concurrently)',
                'alg_flops_per_step': flops}
    prof = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(prof):
        with open(prof) as fh:
            roofline['traffic'] = json.load(fh).get('bytes_per_step')

    # ---------------- e2e through the public API with host buffers: every step
    # uploads its inputs from pinned host memory, evaluates, and reads its blocks
    # back; eri.HostPipeline overlaps step i+1's upload and step i-1's read-back
    # with step i's evaluation
    e2e = None
    if rank == 0 or world > 1:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        h = {'shell_l': pin(batch.shell_l), 'shell_k': pin(batch.shell_k), 'shell_ptr': pin(batch.shell_ptr),
             'shell_xyz': pin(batch.shell_xyz), 'prim_exp': pin(batch.prim_exp),
             'prim_coef': pin(batch.prim_coef), 'quartets': pin(batch.quartets.reshape(-1)),
             'out_off': pin(batch.out_off)}
        prec = eri.PREC_MIXED if (headline_mixed and FP32_CHOSEN[0] > 0) else eri.PREC_FP64
        if headline_mixed:  # the per-quartet bounds are an input of the screened path
            h['bounds'] = bounds.cpu().pin_memory()
        h_out = [torch.empty(batch.out_size, dtype=torch.float64).pin_memory() for _ in range(2)]
        h2d = sum(t.numel() * t.element_size() for t in h.values())
        d2h = h_out[0].numel() * 8
        pipe = eri.HostPipeline(batch.spherical, depth=2)
        lmax_b = int(batch.shell_l.max())

        def e2e_step(i):
            pipe.submit(h, h_out[i % 2], precision=prec, skip_below=SKIP_BELOW if headline_mixed else 0.0,
                        fp32_below=FP32_CHOSEN[0], mixed_tol=MIXED_TOL, lmax=lmax_b)

        for i in range(args.warmup):
            e2e_step(i)
        pipe.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        e_start = torch.cuda.Event(enable_timing=True)
        e_start.record(pipe.s_in)  # the pipeline's first work of the timed region is on its upload stream
        for i in range(args.steps):
            e2e_step(args.warmup + i)
        e_end = pipe.wait_event()
        pipe.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        mse = max_over_ranks(e_start.elapsed_time(e_end) / args.steps, world)
        # the last read-back is the reference result of this configuration
        e2e_err = float(np.abs(h_out[(args.warmup + args.steps - 1) % 2].numpy() - ref64.cpu().numpy()).max())
        e2e = {'value': args.nq * world / (mse * 1e-3), 'unit': 'quartets/s', 'h2d_bytes_per_step': h2d,
               'd2h_bytes_per_step': d2h, 'ms_per_step': mse, 'max_abs_err_vs_fp64': e2e_err,
               'api': 'eri.HostPipeline (pinned host inputs -> blocks in pinned host memory, depth 2)'}

    clk.__exit__(None, None, None)
    eri.set_prim_tol(0.0)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference(batch, args.cpu_seconds)
        cpu = {'value': v, 'unit': 'quartets/s', 'cores': cores, 'kind': kind, 'sample': sample}

    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': 'quartets/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None, 'dtype': 'f64+f32' if (headline_mixed and FP32_CHOSEN[0] > 0) else 'f64', 'data': 'synthetic',
                'config': {'workload': WORKLOAD, 'nq_per_gpu': args.nq,
                           'l2': 'inputs+outputs ~1 GB per step, larger than L2; no flush',
                           'headline_path': ('precision tiers: screened zeros below %.0e, FP32 below %g, FP64 above; '
                                             'primitive quartets with bound below %.0e skipped'
                                             % (SKIP_BELOW, FP32_CHOSEN[0], PRIM_TOL)) if headline_mixed else 'fp64'},
                'fp64': {'value': value64, 'ms_per_step': ms64, 'note': 'every quartet evaluated in FP64'},
                'cuda_graph_ms_per_step': ms_graph,
                'fp64_screened': screened,
                'fp64_screened_prim': screened_prim,
                'mixed': mixed,
                'mixed_over_fp64': (mixed['value'] / value64) if mixed else None,
                'mixed_over_fp64_screened': (mixed['value'] / screened['value']) if mixed else None,
                'roofline': roofline, 'cpu_baseline': cpu, 'e2e': e2e,
                'gpu_launches': launches * args.steps,
                'gpu_launches_per_step': launches,
                'clocks': clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
