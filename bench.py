"""Benchmark: contracted ERI quartets/s on one B200 (or N, one batch split).

Workload (one step = one pass of the ERI path over one batch):
  1e6 shell quartets, l in {0,1,2} per shell (class uniform over the 81
  (la,lb,lc,ld) classes), K uniform in {1..6} per shell, exponents log-uniform
  in [0.05, 1e4], coefficients uniform [0.1, 1] then normalised, centres
  uniform in a 30-bohr cube, spherical output, seed 1.  Synthetic data with
  the shapes of that configuration.  With N GPUs the same batch is split into
  N cost-balanced contiguous shards of its class-sorted quartet list
  (intception_b200.shard), one per rank: strong scaling, no collective on the
  data path.

Paths timed per step, every step a complete pass (screening bounds included):
  fp64_exact     every quartet evaluated in FP64 (the drop-ins' semantics)
  fp64_screened  analytic quartet bounds on the device, blocks with bound
                 < 1e-12 written as zeros, primitive quartets with bound
                 < 1e-18 skipped, the rest in FP64
  mixed          the same screening, FP32 VRR for kept quartets with bound
                 below fp32_below (tuned over a sweep, then measured again),
                 its rounding-error bound checked, rejected quartets in FP64
value = the mixed path (the product's batched path); mixed_over_fp64 compares
it with fp64_screened, which does the same screening.

--workload nuclear_2idx | overlap_2idx times the reference example script's
two-index classes instead (4e6 primitive pairs, l <= 2; one launch per step);
--workload lattice_l3 a sample of the 200-atom l <= 3 lattice.

Arms:
  default          : this library
  --impl reference : the reference's own CPU implementation of the path (the
                     C99 its generator emits, oracle/_ref, OpenMP over the
                     box's cores) behind the same screening, on a bounded
                     sample of the same workload.

Prints one JSON line (rank 0).  Device-timed with inputs resident in HBM
(inputs + outputs ~1 GB, larger than L2, so no flush is needed); e2e = the
same through the public API with host buffers and the H2D/D2H copies inside
the timed region.
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
SKIP_BELOW = 1e-12      # screening: blocks whose bound is smaller are written as zeros
FP32_BELOW = 1e-4       # mixed path: FP32 VRR attempted below this bound ...
MIXED_TOL = 5e-11       # ... and kept only where its rounding-error bound is below this; else FP64
PRIM_TOL = 1e-18        # screened paths: primitive quartets with Q_ab Q_cd below this skipped
HRR_TOL = 1e-13         # class kernels: HRR rounding-error estimate above this -> generic kernel (library default)
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
    ap.add_argument('--workload', default='eri',
                    choices=['eri', 'nuclear_2idx', 'overlap_2idx', 'lattice_l3', 'c5'],
                    help='eri: the headline; *_2idx: the example script\'s two-index classes; lattice_l3: '
                         'a sample of the 200-atom l <= 3 lattice\'s screened quartets; c5: a sample of the '
                         'l <= 4, K <= 8 screened-quartet workload')
    ap.add_argument('--npairs', type=int, default=4_000_000)
    ap.add_argument('--nq-lattice', type=int, default=2_000_000)
    ap.add_argument('--nq-c5', type=int, default=50_000)
    ap.add_argument('--only', default=None, choices=['fp64', 'fp64_cart', 'screened', 'screened_prim', 'bounds',
                                                     'class', 'c5classes'],
                    help='profiling: run only this ERI step (W warm-up + K timed) and print its time; fp64_cart '
                         'is the FP64 step with Cartesian output (no spherical transform); class runs one class '
                         '(--cls) alone, FP64 then its FP32 kernel with every quartet in the FP32 tier; c5classes '
                         'times each class of --cls (comma-separated) on the l <= 4 shell distribution')
    ap.add_argument('--cls', default='2222', help='--only class: the class as four digits la lb lc ld')
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


def cpu_reference(batch, seconds, step_index=0, skip_below=SKIP_BELOW):
    """Time the reference's emitted C99 (oracle/_ref) -- or, when it was not
    built, the oracle port -- on all host cores over a bounded random sample of
    the batch, behind the same analytic screening as the GPU's screened paths
    (bounds computed in the timed call; skip_below 0 evaluates every quartet).
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
            if skip_below > 0:
                loader.ref_batch_screened(sub, T, skip_below, nthreads=cores)
            else:
                loader.ref_batch(sub, T, nthreads=cores)
        else:
            loader.oracle_batch(sub, T)
        return time.perf_counter() - t0

    n = 2000 if skip_below == 0 else 20000
    dt = run(n)
    n2 = int(min(batch.nq, max(n, n * seconds / max(dt, 1e-3))))
    dt2 = run(n2)
    used = cores if lib is not None else 1
    what = ('analytic bounds, zeros below %.0e, the rest through the emitted function' % skip_below
            if skip_below > 0 else 'every quartet through the emitted function')
    return n2 / dt2, kind, used, '%d random quartets of the workload (uniform sample); %s' % (n2, what)


def reference_error(batch, outs, nsample=20000, seed=123, exact_worst=0):
    """Max |GPU - reference C99| over a seeded sample of the batch's quartets:
    outs maps a path name to that path's device output for the whole batch.
    The reference evaluates every sampled quartet (no screening), so a
    screened path's figure includes its screening error.  exact_worst > 0:
    the quartets with the largest differences (up to that many, K product
    <= 2000) are also evaluated exactly (the oracle in binary128), and each
    side's error against those values is reported."""
    from intception_b200 import basis
    from oracle import loader
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(batch.nq, min(nsample, batch.nq), replace=False))
    sub = batch.subset(idx)
    ref = loader.ref_batch(sub, basis.sph_matrices(6), nthreads=os.cpu_count() or 1)
    kind = 'reference'
    if ref is None:
        ref, kind = loader.oracle_batch(sub, basis.sph_matrices(6)), 'port'
    sizes = basis.block_sizes(batch.shell_l, batch.quartets[idx], batch.spherical)
    gather = np.concatenate([np.arange(o, o + n) for o, n in zip(batch.out_off[idx], sizes)])
    res = {name: float(np.abs(out[gather] - ref).max()) for name, out in outs.items()}
    # the quartets with the largest differences (first path), for diagnosis
    name0 = next(iter(outs))
    diff = np.abs(outs[name0][gather] - ref)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    perq = np.maximum.reduceat(diff, starts) if len(starts) else np.zeros(0)
    worst = []
    for w in np.argsort(-perq)[:5]:
        qq = batch.quartets[idx[w]]
        exps = [batch.prim_exp[batch.shell_ptr[s_]:batch.shell_ptr[s_] + batch.shell_k[s_]] for s_ in qq]
        ent = {'l': [int(batch.shell_l[s_]) for s_ in qq], 'k': [int(batch.shell_k[s_]) for s_ in qq],
               'exp_range': [[float(e.min()), float(e.max())] for e in exps],
               'err': float(perq[w]), 'max_abs': float(np.abs(ref[starts[w]:starts[w] + sizes[w]]).max())}
        if len(worst) < exact_worst and np.prod(ent['k']) <= 2000 and perq[w] > 1e-13:
            ex = loader.oracle_batch_quad(batch.subset(idx[w:w + 1]), basis.sph_matrices(6))
            ent['gpu_vs_exact'] = float(np.abs(outs[name0][gather][starts[w]:starts[w] + sizes[w]] - ex).max())
            ent['reference_vs_exact'] = float(np.abs(ref[starts[w]:starts[w] + sizes[w]] - ex).max())
        worst.append(ent)
    res['worst_quartets_' + name0] = worst
    res['sample'] = '%d seeded random quartets of this rank\'s batch vs the %s C99, unscreened' % (len(idx), kind)
    res['max_abs_reference'] = float(np.abs(ref).max())
    return res


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
            'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': WORKLOAD, 'nq': args.nq, 'parallelism': 'openmp host cores',
                       'screening': 'the GPU arm\'s: analytic quartet bounds in the step, zero blocks below %.0e'
                       % SKIP_BELOW},
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


C5_WORKLOAD = ('l in 0..4 per shell, K uniform in 1..8, alpha log-uniform [0.02,1e5], centres uniform in a '
               '10-bohr cube, spherical, seed 4; candidates screened with the analytic bounds at 1e-12; a sample of '
               '%d kept quartets standing for the 5e7-quartet batch')


def c5_batch(nq, seed=4):
    """nq quartets of the l <= 4 workload that pass the 1e-12 screen: candidate
    quartets (four fresh shells each) are drawn in rounds and kept by their
    analytic bound, computed on the GPU.  Returns (batch, kept fraction)."""
    import torch
    from intception_b200 import basis, eri
    rng_seed, kept, drawn, parts = seed, [], 0, []
    while sum(len(k) for k in kept) < nq:
        cand = basis.independent_quartet_batch(rng_seed, max(nq, 20000), [0, 1, 2, 3, 4], [1, 2, 3, 4, 5, 6, 7, 8],
                                               0.02, 1.0e5, 10.0, True)
        rng_seed += 1000
        bnd = eri.EriEngine(cand).analytic_bounds().cpu().numpy()
        idx = np.nonzero(bnd >= SKIP_BELOW)[0]
        drawn += cand.nq
        kept.append(idx)
        parts.append(cand)
    # keep the first nq survivors (in draw order) in one shell table
    qs = []
    need = nq
    for cand, idx in zip(parts, kept):
        take = idx[:need]
        need -= len(take)
        qs.append(cand.subset(take))
        if need == 0:
            break
    ls = np.concatenate([b.shell_l for b in qs])
    ks = np.concatenate([b.shell_k for b in qs])
    xyz = np.concatenate([b.shell_xyz for b in qs])
    e = np.concatenate([b.prim_exp for b in qs])
    c = np.concatenate([b.prim_coef for b in qs])
    ptr = np.concatenate([[0], np.cumsum(ks)[:-1]]).astype(np.int32)
    quart, base = [], 0
    for b in qs:
        quart.append(b.quartets + base)
        base += len(b.shell_l)
    quart = np.concatenate(quart).astype(np.int32)
    off, total = basis.packed_offsets(ls, quart, True)
    b = basis.ShellBatch(ls, ks, ptr, xyz, e, c, quart, off, True, total)
    frac = sum(len(k) for k in kept) / drawn
    return b, frac


def run_c5(args, rank, world, local):
    """The l <= 4 workload on a sample of its screened quartets: FP64 (every
    sampled quartet) and the mixed path (analytic bounds in the step, FP32
    tier below 1e-4 where a class has FP32 kernels), its CUDA-graph replay;
    the reference C99 on the host cores beside it."""
    import torch
    from intception_b200 import eri
    batch, frac = c5_batch(args.nq_c5)
    eng = eri.EriEngine(batch)
    out = torch.empty(batch.out_size, dtype=torch.float64, device='cuda')
    if args.only == 'fp64':  # profilers: the FP64 step alone
        run_only(args, eng, out)
        return
    bounds = torch.empty(batch.nq, dtype=torch.float64, device='cuda')
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

    def screened_step(precision):
        eng.analytic_bounds(out=bounds)
        eng.compute(out=out, precision=precision, bounds=bounds, skip_below=SKIP_BELOW, fp32_below=FP32_BELOW,
                    mixed_tol=MIXED_TOL)

    clk = ClockSampler(local).__enter__()
    eri.set_prim_tol(0.0)
    ms64 = timed(lambda: eng.compute(out=out))
    redo64 = eri.last_hrr_redo()
    ref = out.clone()
    host = {'fp64_exact': ref.cpu().numpy()}
    # once, untimed: the class kernels' results without the HRR check (no redo)
    eri.set_hrr_tol(0.0)
    eng.compute(out=out)
    host['fp64_no_hrr_check'] = out.cpu().numpy()
    eri.set_hrr_tol(HRR_TOL)
    eri.set_prim_tol(PRIM_TOL)
    mss = timed(lambda: screened_step(eri.PREC_FP64))
    errs = max_over_ranks(float((out - ref).abs().max().item()), world)
    msm = timed(lambda: screened_step(eri.PREC_MIXED))
    redom = eri.last_hrr_redo()
    errm = max_over_ranks(float((out - ref).abs().max().item()), world)
    host['mixed'] = out.cpu().numpy()
    launches = eri.EriEngine.last_launch_count() + 1
    graph = eng.graph(out, precision=eri.PREC_MIXED, bounds=bounds, skip_below=SKIP_BELOW, fp32_below=FP32_BELOW,
                      mixed_tol=MIXED_TOL)

    def graph_step():
        eng.analytic_bounds(out=bounds)
        graph.launch()

    msg = timed(graph_step)
    errg = max_over_ranks(float((out - ref).abs().max().item()), world)
    graph.close()
    # the headline: the fastest path within 1e-10 of exact FP64, then measured again on its own
    cands = [(ms64, 0.0, 'fp64'), (mss, errs, 'fp64 + screening'), (msm, errm, 'precision tiers')]
    _, _, path = min([c for c in cands if c[1] <= ERR_BAR] or cands)
    if path == 'fp64':
        eri.set_prim_tol(0.0)
    ms_head = timed({'fp64': lambda: eng.compute(out=out), 'fp64 + screening': lambda: screened_step(eri.PREC_FP64),
                     'precision tiers': lambda: screened_step(eri.PREC_MIXED)}[path])
    err_head = max_over_ranks(float((out - ref).abs().max().item()), world)
    eri.set_prim_tol(0.0)
    clk.__exit__(None, None, None)
    # live primitive quartets of the sample (the per-primitive cost against (ff|ff))
    nprim = float((live_pairs(batch, 0, 1) * live_pairs(batch, 2, 3)).sum())
    cpu, ref_err = None, None
    if rank == 0:
        ref_err = reference_error(batch, host, nsample=2000, exact_worst=3)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference(batch, args.cpu_seconds, skip_below=0.0)
        cpu = {'value': v, 'unit': 'quartets/s', 'cores': cores, 'kind': kind, 'sample': sample}
    if rank == 0:
        nq = batch.nq * world
        print(json.dumps({
            'metric': 'contracted ERI quartets/s on B200, l<=4 K<=8 screened quartets (sample of the 5e7 batch)',
            'value': nq / (ms_head * 1e-3), 'unit': 'quartets/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms_head, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64+f32' if path == 'precision tiers' else 'f64', 'data': 'synthetic',
            'config': {'workload': C5_WORKLOAD % batch.nq, 'kept_fraction_of_candidates': frac,
                       'headline_path': path + ' (the fastest path within 1e-10 of exact FP64, measured again)',
                       'prim_tol': PRIM_TOL, 'fp32_below': FP32_BELOW, 'mixed_tol': MIXED_TOL,
                       'l2': 'outputs %.0f MB per step; no flush' % (batch.out_size * 8 / 1e6)},
            'max_abs_err_vs_fp64': err_head, 'max_abs_err_vs_reference': ref_err,
            'fp64': {'ms_per_step': ms64, 'value': nq / (ms64 * 1e-3), 'note': 'every sampled quartet, FP64',
                     'ns_per_live_primitive_quartet': ms64 * 1e6 / nprim, 'hrr_redo': redo64},
            'fp64_screened': {'ms_per_step': mss, 'value': nq / (mss * 1e-3), 'max_abs_err_vs_fp64': errs,
                              'note': 'the mixed path\'s screening, FP64 throughout'},
            'mixed': {'ms_per_step': msm, 'max_abs_err_vs_fp64': errm, 'hrr_redo': redom},
            'cuda_graph': {'ms_per_step': msg, 'max_abs_err_vs_fp64': errg},
            'hrr_tol': HRR_TOL,
            'mixed_over_fp64': mss / msm, 'live_primitive_quartets': nprim,
            'estimated_5e7_quartets_s': 5e7 / (nq / (ms_head * 1e-3)),
            'cpu_baseline': cpu, 'gpu_launches': launches * args.steps, 'clocks': clk.summary()}), flush=True)


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
    host = {'fp64_exact': ref.cpu().numpy()}
    # Schwarz factors are per basis (computed once, reused by every batch of
    # this lattice's quartets); the sample holds only quartets above 1e-12
    bounds = eng.quartet_bounds()
    eri.set_prim_tol(PRIM_TOL)

    def prim_step():
        eng.compute(out=out, bounds=bounds, skip_below=SKIP_BELOW)

    def mixed_step():
        eng.compute(out=out, precision=eri.PREC_MIXED, bounds=bounds, skip_below=SKIP_BELOW, fp32_below=FP32_BELOW,
                    mixed_tol=MIXED_TOL)

    msp = timed(prim_step)
    errp = max_over_ranks(float((out - ref).abs().max().item()), world)
    host['fp64_prim'] = out.cpu().numpy()
    msm = timed(mixed_step)
    errm = max_over_ranks(float((out - ref).abs().max().item()), world)
    host['mixed'] = out.cpu().numpy()
    rej = eng.fp32_rejected()
    redo_m = eri.last_hrr_redo()
    nfp32 = int((bounds < FP32_BELOW).sum().item())
    # the fastest path within 1e-10 of exact FP64, then measured again on its own
    cands = [(ms64, 0.0, 'fp64'), (msp, errp, 'fp64 + primitive screening'), (msm, errm, 'precision tiers')]
    ok = [c for c in cands if c[1] <= ERR_BAR] or cands
    _, _, path = min(ok)
    if path == 'fp64':
        eri.set_prim_tol(0.0)
    fn = {'fp64': lambda: eng.compute(out=out), 'fp64 + primitive screening': prim_step,
          'precision tiers': mixed_step}[path]
    ms = timed(fn)
    err = max_over_ranks(float((out - ref).abs().max().item()), world)
    launches = eri.EriEngine.last_launch_count()
    eri.set_prim_tol(0.0)
    clk.__exit__(None, None, None)
    nq = batch.nq * world
    cpu, ref_err = None, None
    if rank == 0:
        ref_err = reference_error(batch, host, nsample=10000)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference(batch, args.cpu_seconds, skip_below=0.0)
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
                       % (batch.out_size * 8 / 1e6),
                       'bounds': 'Schwarz factors, once per basis (outside the step)'},
            'max_abs_err_vs_fp64': err,
            'max_abs_err_vs_reference': ref_err,
            'fp64': {'ms_per_step': ms64, 'value': nq / (ms64 * 1e-3), 'note': 'exact, no screening'},
            'fp64_prim': {'ms_per_step': msp, 'max_abs_err_vs_fp64': errp},
            'mixed': {'ms_per_step': msm, 'max_abs_err_vs_fp64': errm, 'fp32_attempted': nfp32,
                      'fp32_rejected': rej, 'hrr_redo': redo_m},
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
    roofline['traffic'] = profiled_traffic('traffic_%s.md' % args.workload)
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


def profiled_traffic(name):
    """DRAM bytes per step recorded from an ncu capture in profiles/<name>
    (its line 'bytes per step: N'), or None when there is no such record."""
    import re
    path = os.path.join(ROOT, 'profiles', name)
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        m = re.search(r'^bytes per step: ([0-9.eE+]+)', fh.read(), re.M)
    return float(m.group(1)) if m else None


def run_only(args, eng, out):
    """One step kind alone (for profilers): the FP64 step over every quartet,
    the screened FP64 step (analytic bounds inside the step), or the
    analytic-bound kernel alone (bounds)."""
    import torch
    from intception_b200 import eri
    screened = args.only in ('screened', 'screened_prim', 'bounds')
    bounds = torch.empty(eng.nq, dtype=torch.float64, device='cuda') if screened else None
    eri.set_prim_tol(PRIM_TOL if args.only == 'screened_prim' else 0.0)

    def step():
        if screened:
            eng.analytic_bounds(out=bounds)
        if args.only != 'bounds':  # bounds: the analytic-bound kernel alone
            eng.compute(out=out, bounds=bounds, skip_below=SKIP_BELOW if screened else 0.0)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    assert eng.device_status() == 0
    print(json.dumps({'only': args.only, 'nq': eng.nq, 'steps': args.steps, 'warmup': args.warmup,
                      'ms_per_step': ev0.elapsed_time(ev1) / args.steps,
                      'kernels_per_step': 1 if args.only == 'bounds' else
                      eri.EriEngine.last_launch_count() + (1 if screened else 0)}), flush=True)


def run_c5_classes(args):
    """Per-class cost on the l <= 4 workload's shell distribution (K uniform
    in 1..8, exponents log-uniform in [0.02, 1e5], centres in a 10-bohr
    cube, spherical): each class of --cls (comma-separated la lb lc ld
    digits) alone, --nq quartets, FP64, the HRR check on; ns per live
    primitive quartet (c_a c_b exp(-xi R^2) != 0 on both pairs)."""
    import torch
    from intception_b200 import basis, eri
    from intception_b200.emit.eri_emitter import emitted_classes

    def canon(c):
        p0, p1 = sorted(c[:2], reverse=True), sorted(c[2:], reverse=True)
        key = lambda p: p[0] * (p[0] + 1) // 2 + p[1]  # noqa: E731
        return tuple(p0 + p1) if key(p0) >= key(p1) else tuple(p1 + p0)
    emitted = {c for c, _ in emitted_classes()}
    rows = []
    for tag in args.cls.split(','):
        cls = tuple(int(ch) for ch in tag)
        rng = np.random.default_rng(2000 + int(tag))
        ls = np.tile(np.asarray(cls, np.int32), args.nq)
        ks = rng.integers(1, 9, 4 * args.nq).astype(np.int32)
        l, k, ptr, xyz, e, c = basis.make_shells(rng, ls, ks, 0.02, 1.0e5, 10.0)
        q = np.arange(4 * args.nq, dtype=np.int32).reshape(args.nq, 4)
        off, total = basis.packed_offsets(l, q, True)
        b = basis.ShellBatch(l, k, ptr, xyz, e, c, q, off, True, total)
        eng = eri.EriEngine(b)
        out = torch.empty(b.out_size, dtype=torch.float64, device='cuda')

        def timed():
            for _ in range(args.warmup):
                eng.compute(out=out)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                eng.compute(out=out)
            e1.record()
            torch.cuda.synchronize()
            assert eng.device_status() == 0
            return e0.elapsed_time(e1) / args.steps
        ms = timed()
        redo = eri.last_hrr_redo()
        eri.set_hrr_tol(0.0)  # the class's own kernel alone: no quartet handed to the generic kernel
        ms0 = timed()
        eri.set_hrr_tol(HRR_TOL)
        live = float((live_pairs(b, 0, 1) * live_pairs(b, 2, 3)).sum())
        rows.append({'cls': tag, 'nq': args.nq, 'ms': ms, 'live_primitive_quartets': live,
                     'ns_per_live_primitive_quartet': ms * 1e6 / live, 'hrr_redo': redo,
                     'ms_without_hrr_check': ms0, 'ns_per_live_primitive_quartet_without_hrr_check': ms0 * 1e6 / live,
                     'kernel': 'unrolled' if canon(cls) in emitted else 'generic'})
        print(json.dumps(rows[-1]), flush=True)


def run_one_class(args):
    """One class alone (--cls), --nq quartets with the headline distribution:
    W warm-up + K timed steps of the FP64 kernel, then of the class's FP32
    kernel with every quartet in the FP32 tier and every result kept (what the
    FP32 kernel costs, for profilers)."""
    import torch
    from intception_b200 import eri
    from intception_b200.autotune import class_batch
    cls = tuple(int(ch) for ch in args.cls)
    b = class_batch(cls, args.nq, seed=1000, spherical=True)
    eng = eri.EriEngine(b)
    out = torch.empty(b.out_size, dtype=torch.float64, device='cuda')
    ones = torch.ones(b.nq, dtype=torch.float64, device='cuda')
    eri.set_class_fp32(True, cls)
    res = {'only': 'class', 'cls': args.cls, 'nq': b.nq}
    for name, prec in (('fp64', eri.PREC_FP64), ('fp32', eri.PREC_MIXED)):
        kw = dict(bounds=ones, skip_below=0.0, fp32_below=2.0, mixed_tol=1e300) if prec == eri.PREC_MIXED else {}
        for _ in range(args.warmup):
            eng.compute(out=out, precision=prec, **kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            eng.compute(out=out, precision=prec, **kw)
        e1.record()
        torch.cuda.synchronize()
        assert eng.device_status() == 0
        res[name + '_ms'] = e0.elapsed_time(e1) / args.steps
    eri.set_class_fp32(None, cls)
    print(json.dumps(res), flush=True)


def run_eri(args, rank, world, local):
    """The headline workload: one C2 batch, split over the ranks."""
    import torch
    from intception_b200 import basis, eri, shard
    if args.only == 'class':
        run_one_class(args)
        return
    if args.only == 'c5classes':
        run_c5_classes(args)
        return
    full = basis.config_mixed_l2(nq=args.nq, seed=1, spherical=args.only != 'fp64_cart')
    batch = full if world == 1 else shard.shard_for_rank(full, rank, world)[0]
    eng = eri.EriEngine(batch)
    stream = torch.cuda.current_stream()
    out = torch.empty(batch.out_size, dtype=torch.float64, device='cuda')
    bounds = torch.empty(batch.nq, dtype=torch.float64, device='cuda')
    if args.only:
        run_only(args, eng, out)
        return
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

    def screened_step(precision, fb):
        eng.analytic_bounds(out=bounds)  # part of every screened step
        eng.compute(out=out, precision=precision, bounds=bounds, skip_below=SKIP_BELOW, fp32_below=fb,
                    mixed_tol=MIXED_TOL)

    def err_vs(ref):
        return max_over_ranks(float((out - ref).abs().max().item()), world)

    rate = lambda ms: args.nq / (ms * 1e-3)  # noqa: E731  whole job: the full batch over the slowest rank

    clk = ClockSampler(local).__enter__()  # sampled over every timed region below
    # ---- FP64, every quartet evaluated, no screening of any kind
    eri.set_prim_tol(0.0)
    ms64 = timed(lambda: eng.compute(out=out))
    launches64 = eri.EriEngine.last_launch_count()
    redo64 = eri.last_hrr_redo()
    ref64 = out.clone()
    host_fp64 = out.cpu().numpy() if rank == 0 else None
    # ---- screened FP64: analytic bounds in the step, zeros below SKIP_BELOW, primitive screening
    eri.set_prim_tol(PRIM_TOL)
    ms_s = timed(lambda: screened_step(eri.PREC_FP64, 0.0))
    err_s = err_vs(ref64)
    kept_idx = np.nonzero((bounds >= SKIP_BELOW).cpu().numpy())[0]
    n_kept = len(kept_idx)  # this rank's quartets kept by the screening
    # the screened step without primitive screening: its kept quartets' algorithmic
    # work over its time is the utilisation of the concurrent class kernels
    eri.set_prim_tol(0.0)
    ms_s0 = timed(lambda: screened_step(eri.PREC_FP64, 0.0))
    eri.set_prim_tol(PRIM_TOL)
    # ---- FP32-tier setting: a sweep over fp32_below (0 = tier off), then the
    # chosen setting measured on its own as the headline
    sweep = []
    if not args.no_mixed:
        for fb in FP32_SWEEP[1:]:
            msx = timed(lambda: screened_step(eri.PREC_MIXED, fb))
            sweep.append({'fp32_below': fb, 'ms_per_step': msx, 'max_abs_err_vs_fp64': err_vs(ref64),
                          'fp32_attempted': int(((bounds >= SKIP_BELOW) & (bounds < fb)).sum().item()),
                          'fp32_rejected': eng.fp32_rejected()})
    ok = [r for r in sweep if r['max_abs_err_vs_fp64'] <= ERR_BAR]
    best = min(ok, key=lambda r: r['ms_per_step']) if ok else None
    fb = best['fp32_below'] if best is not None and best['ms_per_step'] < ms_s else 0.0
    FP32_CHOSEN[0] = fb
    prec = eri.PREC_MIXED if fb > 0 else eri.PREC_FP64
    msm = timed(lambda: screened_step(prec, fb))
    launches = eri.EriEngine.last_launch_count() + 1  # + the bounds kernel
    err_m = err_vs(ref64)
    rej = eng.fp32_rejected() if fb > 0 else 0
    redo_m = eri.last_hrr_redo()
    host_mixed = out.cpu().numpy() if rank == 0 else None
    value = rate(msm)
    # ---- the headline configuration replayed from a CUDA graph (bounds kernel
    # outside the graph, on the same stream)
    graph = eng.graph(out, precision=prec, bounds=bounds, skip_below=SKIP_BELOW, fp32_below=fb, mixed_tol=MIXED_TOL)

    def graph_step():
        eng.analytic_bounds(out=bounds)
        graph.launch()

    ms_graph = timed(graph_step)
    err_graph = err_vs(ref64)
    graph.close()

    # ---- roofline of the FP64 step against the measured FP64 FMA peak
    flops, _ = alg_flops(batch)
    flops_kept, _ = alg_flops(batch.subset(kept_idx)) if n_kept else (0.0, None)
    peak64 = eri.fma_peak(True)
    peak32 = eri.fma_peak(False)  # the FP32 tier's pipe: its rate over FP64's bounds what FP32 VRR can gain
    achieved = flops / (ms64 * 1e-3)
    roofline = {'bound': 'fp64', 'achieved': achieved / 1e12, 'peak': peak64 / 1e12, 'unit': 'TFLOP/s',
                'frac': achieved / peak64 if peak64 else None, 'traffic': None,
                'peak_source': 'measured FP64 FMA-chain kernel (intception_b200_fma_peak), this run; '
                               'MEASURED_PEAKS.json has no FP64 figure',
                'kernel': 'whole FP64 step of this rank (per-class kernels run concurrently)',
                'alg_flops_per_step': flops}
    roofline['traffic'] = profiled_traffic('traffic_fp64_l2_sph.md')
    if roofline['traffic']:
        roofline['traffic_source'] = ('dram__bytes_read.sum + dram__bytes_write.sum of the FP64 step\'s '
                                      'kernels, one ncu capture at 2e5 quartets scaled by the quartet count '
                                      '(profiles/traffic_fp64_l2_sph.md)')

    # ---- e2e through the public API with host buffers: every step uploads its
    # inputs from pinned host memory, computes the analytic bounds and the
    # screened blocks on the device, and reads its blocks back;
    # eri.HostPipeline overlaps step i+1's upload and step i-1's read-back with
    # step i's evaluation
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h = {'shell_l': pin(batch.shell_l), 'shell_k': pin(batch.shell_k), 'shell_ptr': pin(batch.shell_ptr),
         'shell_xyz': pin(batch.shell_xyz), 'prim_exp': pin(batch.prim_exp),
         'prim_coef': pin(batch.prim_coef), 'quartets': pin(batch.quartets.reshape(-1)),
         'out_off': pin(batch.out_off)}
    h_out = [torch.empty(batch.out_size, dtype=torch.float64).pin_memory() for _ in range(2)]
    h2d = sum(t.numel() * t.element_size() for t in h.values())
    d2h = h_out[0].numel() * 8
    pipe = eri.HostPipeline(batch.spherical, depth=2)
    lmax_b = int(batch.shell_l.max())

    def e2e_step(i):
        pipe.submit(h, h_out[i % 2], precision=prec, skip_below=SKIP_BELOW, fp32_below=fb, mixed_tol=MIXED_TOL,
                    lmax=lmax_b)

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
    e2e_err = float(np.abs(h_out[(args.warmup + args.steps - 1) % 2].numpy() - ref64.cpu().numpy()).max())
    e2e = {'value': rate(mse), 'unit': 'quartets/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
           'ms_per_step': mse, 'max_abs_err_vs_fp64': max_over_ranks(e2e_err, world),
           'api': 'eri.HostPipeline (pinned host inputs -> analytic bounds and screened blocks on the device -> '
                  'blocks in pinned host memory, depth 2)'}
    clk.__exit__(None, None, None)
    eri.set_prim_tol(0.0)

    # ---- outside the timing: reference error on a sample, CPU baseline
    ref_err, cpu, cpu_all = None, None, None
    if rank == 0:
        ref_err = reference_error(batch, {'fp64_exact': host_fp64, 'headline': host_mixed})
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference(batch, args.cpu_seconds)
        cpu = {'value': v, 'unit': 'quartets/s', 'cores': cores, 'kind': kind, 'sample': sample}
        v0, kind0, cores0, sample0 = cpu_reference(batch, args.cpu_seconds / 2, skip_below=0.0)
        cpu_all = {'value': v0, 'unit': 'quartets/s', 'cores': cores0, 'kind': kind0, 'sample': sample0}

    if rank == 0:
        fp64_s = {'value': rate(ms_s), 'ms_per_step': ms_s, 'max_abs_err_vs_fp64': err_s,
                  'without_primitive_screening': {
                      'ms_per_step': ms_s0, 'kept_alg_flops': flops_kept,
                      'fp64_frac': (flops_kept / (ms_s0 * 1e-3)) / peak64 if peak64 else None,
                      'note': 'algorithmic work of the kept quartets over the step time: the utilisation '
                              'of the concurrent class kernels (bounds, sort and zero fill included)'}}
        line = {'metric': METRIC, 'value': value, 'unit': 'quartets/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': msm, 'higher_is_better': True, 'scaling': 'strong',
                'vs_baseline': None, 'dtype': 'f64+f32' if fb > 0 else 'f64', 'data': 'synthetic',
                'config': {'workload': WORKLOAD, 'nq_total': args.nq, 'nq_this_rank': batch.nq,
                           'split': 'one batch, %d cost-balanced contiguous shards of its class-sorted list' % world,
                           'l2': 'inputs+outputs ~1 GB per step, larger than L2; no flush',
                           'headline_path': ('mixed: analytic bounds in the step, zeros below %.0e, primitive '
                                             'quartets below %.0e skipped, FP32 VRR below bound %g (0: tier off, '
                                             'all FP64), rounding-error bound %.0e'
                                             % (SKIP_BELOW, PRIM_TOL, fb, MIXED_TOL))},
                'max_abs_err_vs_fp64': err_m,
                'max_abs_err_vs_reference': ref_err,
                'fp64_exact': {'value': rate(ms64), 'ms_per_step': ms64, 'kernels_per_step': launches64,
                               'hrr_redo': redo64, 'note': 'every quartet evaluated in FP64, no screening'},
                'fp64_screened': fp64_s,
                'mixed': {'value': value, 'ms_per_step': msm, 'fp32_below': fb, 'fp32_tier_active': fb > 0,
                          'fp32_rejected': rej, 'hrr_redo': redo_m, 'hrr_tol': HRR_TOL, 'mixed_tol': MIXED_TOL,
                          'fp32_sweep': sweep,
                          'note': 'fp32_below chosen by the sweep (fastest within 1e-10), then measured again '
                                  'on its own; the same screening as fp64_screened'},
                'mixed_over_fp64': value / rate(ms_s),
                'fma_peaks_tflops': {'fp64': peak64 / 1e12, 'fp32': peak32 / 1e12, 'fp32_over_fp64': peak32 / peak64,
                                     'source': 'intception_b200_fma_peak, this run (independent FMA chains)'},
                'screening_gain': rate(ms_s) / rate(ms64),
                'kept_fraction': n_kept / batch.nq,
                'cuda_graph': {'ms_per_step': ms_graph, 'max_abs_err_vs_fp64': err_graph},
                'roofline': roofline, 'cpu_baseline': cpu, 'cpu_baseline_unscreened': cpu_all, 'e2e': e2e,
                'gpu_launches': launches * args.steps, 'gpu_launches_per_step': launches,
                'clocks': clk.summary()}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == 'reference':
        # host cores only: no process group; rank 0 runs the reference, the
        # other ranks of a multi-GPU launch exit at once
        rank, world = int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1'))
        if args.workload in ('lattice_l3', 'c5'):
            if rank == 0:  # the sample is drawn with GPU screening bounds; its line carries cpu_baseline
                print(json.dumps({'impl': 'reference', 'unavailable': '%s draws its quartet sample with GPU '
                                  'screening bounds; the reference C99 is timed in that line\'s cpu_baseline'
                                  % args.workload}))
            return
        if args.workload != 'eri':
            run_twoidx(args, rank, world, 0)
        else:
            run_reference_arm(args, rank, world)
        return
    rank, world, local = dist_init(args.gpus)
    try:
        if args.workload == 'lattice_l3':
            run_lattice(args, rank, world, local)
        elif args.workload == 'c5':
            run_c5(args, rank, world, local)
        elif args.workload != 'eri':
            run_twoidx(args, rank, world, local)
        else:
            run_eri(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
