#!/usr/bin/env python
"""Benchmark of the Wyckoff-search trial evaluation (trial structures evaluated/s).

Workload (one "step"): one complete Wyckoff search of the PbSO4-like Pnma
problem -- 4096 replicas x 5000 generations, 75 % single-site / 25 %
collective moves, replica ladders of 8, exchange every 10 generations, the
resolution and penalty ramps of the reference -- run on the device as one
launch.  Every step starts from fresh random coordinates (uploaded before the
timed region) and the L2 cache is flushed before each step.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Rank 0 prints one JSON line.  With N > 1 (torchrun), each rank runs its own
4096-replica search (weak scaling; replicas and ladders are independent, so
there is no collective on the data path) and the time is the maximum over
ranks.  ``--impl reference`` times the CPU implementation (the FP64 oracle
port of the reference's trial evaluation, OpenMP over replicas) on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from powder6_b200.dist import barrier, max_over_ranks  # noqa: E402

PARTICLES = 4096
GENERATIONS = 5000
SWAP_EVERY = 10
MUFU_PER_CLK_PER_SM = 16   # SFU transcendental rate of an sm_100 SM (4 per sub-partition)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--particles', type=int, default=PARTICLES)
    ap.add_argument('--generations', type=int, default=GENERATIONS)
    ap.add_argument('--cos-mode', type=int, default=-1,
                    help='0 SFU cosine, 1 FMA polynomial, 2 factored FP64; -1 (default): 2 where the group allows it')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-sub-workloads', action='store_true',
                    help='default workload: leave out the PT and contraction sub-results')
    ap.add_argument('--workload', default='wyckoff',
                    choices=['wyckoff', 'pt', 'contract', 'batch', 'learned', 'refine', 'cf', 'profile', 'fragment'],
                    help='wyckoff: the plain Wyckoff search (default); pt: the NaCl parallel-tempering fit; '
                         'contract: the fixed-profile contraction Y = I . P (16384 x 3000 x 12000); '
                         'batch: 64 uneven Wyckoff searches in one persistent launch; '
                         'learned: the learned-proposal search (P2_1/c, 17 sites, 8192 replicas); '
                         'refine: least-squares refinement of 512 perturbed PbSO4 structures; '
                         'cf: charge flipping, 128 random starts of the adaptive plan on a 64^3 grid; '
                         'profile: the PbSO4-like search against its powder pattern (fixed cell and profile, '
                         'split-BF16 contraction), with time to target Rwp, chosen vs plain; '
                         'fragment: config 5 as a rigid fragment scored on its pattern (one search per step, '
                         'about 30 s each)')
    ap.add_argument('--method', default='split', choices=['split', 'split3', 'fp32'],
                    help='contract: two-part split-BF16 (default), three-part split-BF16 (six products, '
                         'chi^2 within 4e-6 of FP64, half the rate), or plain FP32 CUDA cores')
    ap.add_argument('--cf-trials', type=int, default=None, help='cf: random starts (default 128)')
    ap.add_argument('--cf-cycles', type=int, default=None, help='cf: cycles per step (default 100)')
    ap.add_argument('--pt-method', default='rietveld', choices=['rietveld', 'wppf'],
                    help='pt: heights from the structure (default) or free and solved by NNLS in every evaluation')
    ap.add_argument('--chains', type=int, default=64)
    ap.add_argument('--sweeps', type=int, default=2000)
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.dev), f'--query-gpu={self.Q}',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
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
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(max(mx)), 'reasons': sorted(reasons),
                'samples': len(sm)}


def algorithmic_cos(P, groups, n_particles):
    """Cosines a search evaluates: per generation, every active reflection times
    the atoms entering |F|^2 (centring translates excluded), for every replica,
    plus one re-measurement of the current state at each resolution step."""
    gm = P.refl.group_meta.reshape(-1, 4)
    n_f = int((P.tables.gen_skip[:P.n_tot] == 0).sum())
    refl_act = np.array([int(gm[g - 1, 0] + gm[g - 1, 1]) for g in groups])
    steps = 1 + int((np.diff(groups) != 0).sum())
    reeval = sum(int(gm[g - 1, 0] + gm[g - 1, 1]) for g in np.unique(groups))
    per_particle = int(refl_act.sum()) + reeval
    factor = 1 if P.centro else 2
    return per_particle * n_f * n_particles * factor, steps


def cpu_baseline(P, groups, pen, n_particles, seconds=10.0):
    from oracle import oracle as O
    r = O.WyckoffCpuRunner(P, n_particles, seed=7)
    gens = np.linspace(0, len(groups) - 1, 1000).astype(int)
    t0 = time.perf_counter()
    trials = 0
    used = 0
    for g in gens:
        trials += r.generation(int(groups[g]), float(pen[g]))
        used += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {'value': trials / dt, 'unit': 'trials/s', 'cores': O.num_threads(), 'kind': 'port',
            'sample': f'{n_particles} replicas x {used} generations spread evenly over the 5000-generation '
                      f'schedule ({trials} trials, {dt:.1f} s, FP64, OpenMP over replicas)'}


TTT_SEEDS = 8


def wyckoff_time_to_target(P, n, sess):
    """Time to target wR2 (outside the timed region).  The target is 1.05 x the
    converged wR2 the FP64 CPU port of the trial evaluation reaches on the
    same problem and schedule (tests/golden/wyckoff_target.json, written by
    tests/golden/make_wyckoff_target.py), so it does not come from the search
    being timed.  The clock runs from the start of run_wyckoff_search (random
    start, generations in chunks of 250 so the best can be read between
    launches) to the first chunk boundary, or the end of the quench, at which
    the best wR2 is within the target; median over TTT_SEEDS seeds."""
    from powder6_b200.swarm_wyckoff import COS_NAMES, run_wyckoff_search
    fx = ROOT / 'tests' / 'golden' / 'wyckoff_target.json'
    if fx.exists():
        ref = json.loads(fx.read_text())
        wr2, source = float(ref['converged_wr2']), 'FP64 CPU port, full schedule (' + fx.name + ')'
    else:
        conv = run_wyckoff_search(P, num_particles=n, generations=GENERATIONS, seed=11, session=sess)
        wr2, source = 1.0 - conv.best_cc, 'this GPU search (no reference-side fixture)'
    target = 1.0 - 1.05 * wr2
    runs = [run_wyckoff_search(P, num_particles=n, generations=GENERATIONS, seed=101 + k, chunk=250, session=sess,
                               target_cc=target) for k in range(TTT_SEEDS)]
    hits = [r.time_to_target for r in runs if r.time_to_target is not None]
    return {'median_s': float(np.median(hits)) if hits else None, 'reached': f'{len(hits)}/{len(runs)}',
            'converged_wr2': wr2, 'target_wr2': 1.05 * wr2, 'target_source': source,
            'final_wr2': [1.0 - r.best_cc for r in runs], 'cpu_check_delta': [r.cpu_check.get('delta') for r in runs],
            'note': f'chunks of 250 generations; plain search ({COS_NAMES[sess.cos_mode]}) + quench; '
                    f'median over {TTT_SEEDS} seeds'}


def run_reference_batch(args, world, rank):
    """The FP64 oracle port of the trial evaluation on a bounded sample of the
    batch (all host threads): the reference runs one search per worker."""
    if rank != 0:
        return
    from oracle import oracle as O
    from powder6_b200.swarm_wyckoff import schedule
    from powder6_b200.workloads import batched_problems
    items = batched_problems(64, seed=1)
    trials, t_used = 0, 0.0
    for _ in range(args.warmup):
        it = items[0]
        O.WyckoffCpuRunner(it.problem, min(it.replicas, 256), seed=3).generation(it.problem.refl.n_groups, 1.0)
    t0 = time.perf_counter()
    k = 0
    while time.perf_counter() - t0 < 2.0 * args.steps and k < len(items):
        it = items[k]
        g, pen = schedule(BATCH_GENERATIONS, it.problem.refl.n_groups)
        r = O.WyckoffCpuRunner(it.problem, it.replicas, seed=3)
        trials += r.generation(int(g[len(g) // 2]), float(pen[len(g) // 2]))
        k += 1
    dt = time.perf_counter() - t0
    v = trials / dt
    sample = f'one mid-schedule generation of each of the first {k} searches ({trials} trials, FP64 oracle port, OpenMP)'
    print(json.dumps({
        'impl': 'reference', 'metric': 'trial structures evaluated/s', 'value': v, 'unit': 'trials/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000 * dt / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': '64 uneven Wyckoff searches (sampled)'},
        'cpu_baseline': {'value': v, 'unit': 'trials/s', 'cores': O.num_threads(), 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'trials/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


def dist_setup(args):
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
    return world, rank, local


def run_reference(args, world, rank):
    if rank != 0:
        return
    from powder6_b200.swarm_wyckoff import schedule
    from powder6_b200.workloads import wyckoff_problem
    from oracle import oracle as O
    P = wyckoff_problem(seed=1)
    groups, pen = schedule(args.generations, P.refl.n_groups)
    r = O.WyckoffCpuRunner(P, args.particles, seed=7)
    gens = np.linspace(0, args.generations - 1, 4 * (args.steps + args.warmup)).astype(int)
    it = iter(gens)
    per_step = 4

    def step():
        n = 0
        for _ in range(per_step):
            g = next(it)
            n += r.generation(int(groups[g]), float(pen[g]))
        return n
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    trials = sum(step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    v = trials / dt
    sample = (f'{args.particles} replicas x {per_step} generations per step, generations spread evenly over the '
              f'{args.generations}-generation schedule; FP64 oracle port, OpenMP over replicas')
    print(json.dumps({
        'impl': 'reference', 'metric': 'trial structures evaluated/s', 'value': v, 'unit': 'trials/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000 * dt / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': f'wyckoff-search Pnma PbSO4-like, {args.particles} replicas x {args.generations} '
                               f'generations (sampled), d_min 1.2 A'},
        'cpu_baseline': {'value': v, 'unit': 'trials/s', 'cores': O.num_threads(), 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'trials/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


PT_WORKLOAD = ('pt-rietveld NaCl Fm-3m a=5.640 (Na 4a, Cl 4b, Biso 1.0), Cu Ka1/Ka2 1.5406/1.5444 ratio 0.5, '
               '2theta 10-120 step 0.02 (5501 points), TCH U,V,W,X,Y = 0.004,-0.002,0.003,0.02,0.01 (FullProf '
               'units, converted), 6-term Chebyshev, Poisson counts peak ~1e4; refined scale, a, Biso, U, V, W, zero '
               'from +/-5 % starts')


def pt_setup(seed, method='rietveld'):
    """The NaCl problem (observations synthesised from the structure), fitted
    with the structure's heights ('rietveld') or free ones ('wppf')."""
    from oracle import oracle as O
    from powder6_b200.pt_gpu import nacl_problem, start_vectors, synthesise
    P = nacl_problem(seed=1)
    truth = synthesise(P, O.PtModel(P).pattern, seed=1)
    P.method = method
    x0 = start_vectors(P, truth, 1, seed=seed)[0]
    return P, truth, x0


def pt_target(P, truth):
    """Target: 1.05 x the Rwp the least-squares finish converges to from the truth (FP64 oracle)."""
    from oracle import oracle as O
    from powder6_b200.pt_gpu import reflection_dmin, rwp
    _, ref = O.PtModel(P, dmin=reflection_dmin(P)).lm(truth, 30)
    target_rwp = 1.05 * rwp(P, ref['chi2'])
    return target_rwp, target_rwp ** 2 * float(np.sum(P.w * P.y ** 2))


def run_reference_pt(args, world, rank):
    """The CPU tempering (temper at 16 chains, the reference's cap) of the FP64 oracle port on one host thread."""
    if rank != 0:
        return
    from oracle import oracle as O
    from powder6_b200.pt_gpu import pt_scales, reflection_dmin
    P, truth, x0 = pt_setup(5, args.pt_method)
    M = O.PtModel(P, dmin=reflection_dmin(P))
    sc = pt_scales(P, x0)
    chains, per_step = 16, 2

    def step(seed):
        _, st = M.temper(x0, sc, chains=chains, sweeps=per_step, seed=seed)
        return st['proposals']
    for i in range(args.warmup):
        step(100 + i)
    t0 = time.perf_counter()
    trials = sum(step(200 + i) for i in range(args.steps))
    dt = time.perf_counter() - t0
    v = trials / dt
    sample = (f'{chains} chains x {per_step} sweeps x {len(x0)} proposals per step (FP64 oracle port of temper, '
              f'one host thread)')
    print(json.dumps({
        'impl': 'reference', 'metric': 'trial structures evaluated/s', 'value': v, 'unit': 'trials/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000 * dt / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': PT_WORKLOAD + ' (sampled)', 'method': args.pt_method},
        'cpu_baseline': {'value': v, 'unit': 'trials/s', 'cores': 1, 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'trials/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


def pt_cpu_baseline(P, x0, seconds=10.0):
    from oracle import oracle as O
    from powder6_b200.pt_gpu import pt_scales, reflection_dmin
    M = O.PtModel(P, dmin=reflection_dmin(P))
    sc = pt_scales(P, x0)
    t0 = time.perf_counter()
    trials, runs = 0, 0
    while time.perf_counter() - t0 < seconds:
        _, st = M.temper(x0, sc, chains=16, sweeps=2, seed=300 + runs)
        trials += st['proposals']
        runs += 1
    dt = time.perf_counter() - t0
    return {'value': trials / dt, 'unit': 'trials/s', 'cores': 1, 'kind': 'port',
            'sample': f'{runs} runs of 16 chains x 2 sweeps x {len(x0)} proposals ({int(trials)} trials, {dt:.1f} s, '
                      f'FP64 oracle port of temper, one host thread)'}


PT_FP64_FLOPS_PER_POINT = 4 * 6 + 6   # Chebyshev background (6 terms: recurrence + accumulate), residual, w r^2


def pt_roofline(fp64_achieved, fp64_peak, flops_eval, nsm, mhz, trials, ms, chains):
    """The sweep kernel's bound is instruction issue and latency, not a pipe:
    warp instructions per evaluation (profiles/pt_sweep_traffic.txt, from an
    ncu capture of one sweep launch) x evaluations/s against 4 warp
    instructions/clk/SM; the FP64 figure is kept beside it."""
    fp64 = {'bound': 'fp64', 'achieved': fp64_achieved, 'peak': fp64_peak, 'unit': 'TFLOP/s',
            'frac': fp64_achieved / fp64_peak, 'traffic': None,
            'note': f'{flops_eval} FP64 flops per evaluation ({PT_FP64_FLOPS_PER_POINT} per pattern point: '
                    f'Chebyshev background, residual, w r^2; the FP32 peak shapes and the per-reflection '
                    f'FP64 stage not counted); peak 64 FP64 FMA/clk/SM x {nsm} SMs x {mhz:.0f} MHz'}
    inst, traffic = None, None
    tf = ROOT / 'profiles' / 'pt_sweep_traffic.txt'
    if tf.exists():
        for ln in tf.read_text().splitlines():
            if ln.startswith('warp_instructions_per_evaluation:'):
                inst = float(ln.split(':', 1)[1])
            if ln.startswith('bytes_per_launch:'):
                traffic = int(ln.split(':', 1)[1])
    if not inst:
        return fp64
    peak = 4 * nsm * mhz * 1e6 / 1e9
    issued = inst * trials / (ms / 1000.0) / 1e9
    return {'bound': 'issue', 'achieved': issued, 'peak': peak, 'unit': 'Gwarp-inst/s', 'frac': issued / peak,
            'traffic': traffic,
            'note': f'{inst:.0f} warp instructions per evaluation (ncu, one sweep launch of the same fit) x '
                    f'evaluations/s; peak = 4 warp instructions/clk/SM x {nsm} SMs x {mhz:.0f} MHz; '
                    f'{chains} chains on two-CTA clusters occupy {2 * chains} SMs, one evaluation in flight each',
            'fp64_equivalent': fp64}


def main_pt(args, world, rank, local, emit=True):
    """One step = one tempering run of the NaCl fit: args.sweeps sweeps of
    args.chains chains from a +/-5 % start.  value: proposals per second of
    the sweeps (CUDA events around one batch of all the sweeps, state
    resident); e2e: proposals per second of refine() through the public API
    (linear start, the same sweeps with the reference's batching and FP64
    re-scores, least-squares finish; host start vector in, result out);
    time_to_target_rwp: wall seconds from the start of refine() to a best
    Rwp <= 1.05 x the converged Rwp, median over the steps."""
    import torch
    from powder6_b200.pt_gpu import PTContext, PTSession, pt_scales, refine
    torch.cuda.set_device(local)
    P, truth, _ = pt_setup(5, args.pt_method)
    target_rwp, target_chi2 = pt_target(P, truth)
    starts = [pt_setup(10 + i + 100 * rank, args.pt_method)[2] for i in range(args.warmup + args.steps)]

    def ctx_for(x0, seed):
        return PTContext(P, x0, {'chains': args.chains, 'sweeps': args.sweeps, 'maxTemp': 100.0, 'seed': seed,
                                 'scales': pt_scales(P, x0)})
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    dev_ms, launches = [], 0
    with PTSession(ctx_for(starts[0], 1), local) as s:
        for i, x0 in enumerate(starts):
            s.initial([x0])
            s.batch(1, True)
            flush.zero_()
            torch.cuda.synchronize()
            l0 = s.launch_count()
            s.launch(args.sweeps)
            s.synchronize(600)
            if i >= args.warmup:
                dev_ms.append(s.last_batch_ms())
                launches += s.launch_count() - l0
    barrier(world)
    trials = args.chains * args.sweeps * len(starts[0])
    total_ms = max_over_ranks(float(sum(dev_ms)), world)
    value = world * trials * args.steps / (total_ms / 1000.0)
    e2e_s, ttt, rwps, ttt_pt = [], [], [], []
    with ClockSampler(local) as clk:
        for i, x0 in enumerate(starts):
            t0 = time.perf_counter()
            r = refine(ctx_for(x0, 7 + i), local, target_chi2=target_chi2)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                e2e_s.append(dt)
                ttt.append(r['time_to_target'])
                rwps.append(r['rwp'])
                # the tempering alone: linear start and sweeps, no least-squares finish
                ttt_pt.append(refine(ctx_for(x0, 7 + i), local, target_chi2=target_chi2,
                                     finish=False)['time_to_target'])
    e2e_total = max_over_ranks(float(sum(e2e_s)), world)
    e2e_value = world * trials * args.steps / e2e_total
    if rank == 0:
        clocks = clk.summary()
        ms = float(np.mean(dev_ms))
        reached = [t for t in ttt if t is not None]
        reached_pt = [t for t in ttt_pt if t is not None]
        import torch
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks['sm_mhz'] or 1965.0
        fp64_peak = 2 * 64 * nsm * mhz * 1e6 / 1e12          # 64 FP64 FMA/clk/SM on sm_100
        flops_eval = PT_FP64_FLOPS_PER_POINT * len(P.tth)
        fp64_achieved = flops_eval * trials / (ms / 1000.0) / 1e12
        line = {
            'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'fp32 profile, fp64 peaks and chi2', 'data': 'synthetic',
            'config': {'workload': PT_WORKLOAD, 'method': args.pt_method, 'chains': args.chains, 'sweeps': args.sweeps,
                       'step': 'one tempering run (all sweeps) for value; one refine() for e2e',
                       'l2': 'flushed before every step (256 MB write)', 'parallelism': f'replicas only x{world}'},
            'time_to_target_rwp': {'median_s': float(np.median(reached)) if reached else None,
                                   'reached': f'{len(reached)}/{len(ttt)}', 'target_rwp': target_rwp,
                                   'final_rwp_median': float(np.median(rwps)),
                                   'tempering_only': {'median_s': float(np.median(reached_pt)) if reached_pt else None,
                                                      'reached': f'{len(reached_pt)}/{len(ttt_pt)}',
                                                      'note': 'linear start + tempering, no least-squares finish'}},
            'roofline': pt_roofline(fp64_achieved, fp64_peak, flops_eval, nsm, mhz, trials, ms, args.chains),
            'e2e': {'value': e2e_value, 'unit': 'trials/s', 'h2d_bytes_per_step': len(starts[0]) * 8,
                    'd2h_bytes_per_step': len(starts[0]) * 8},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        if not args.no_cpu_baseline and world == 1:
            line['cpu_baseline'] = pt_cpu_baseline(P, starts[0])
        if emit:
            print(json.dumps(line), flush=True)
        return line


CT_EVALS_PER_STEP = 64
CT_WORKLOAD = ('fixed-profile contraction Y = I . P: 16384 replicas x 3000 reflections (lognormal sigma 1.5) x 12000 '
               'points (2theta 5-125 step 0.01), pseudo-Voigt columns FWHM U(0.05, 0.3) deg truncated at +/-20 FWHM, '
               'per-replica weighted chi^2 against a Poisson observed pattern')


def ct_cpu_rows(p, seconds):
    """FP64 oracle product on a sample of replica rows, host BLAS threads."""
    from oracle import oracle as O
    rows = 256
    t0 = time.perf_counter()
    done = 0
    while time.perf_counter() - t0 < seconds:
        lo = (done * rows) % (len(p.intensities) - rows)
        O.contract_fp64(p.intensities[lo:lo + rows], p.profile_t, p.yobs, p.w)
        done += rows
    dt = time.perf_counter() - t0
    return done, dt


def run_reference_ct(args, world, rank):
    if rank != 0:
        return
    from powder6_b200.contraction import banded_problem
    p = banded_problem(seed=1)
    for _ in range(args.warmup):
        ct_cpu_rows(p, 0.5)
    trials, dt = ct_cpu_rows(p, 2.0 * args.steps)
    v = trials / dt
    cores = os.cpu_count()
    sample = f'{trials} replicas in blocks of 256 rows (FP64 product over the full profile matrix, host BLAS)'
    print(json.dumps({
        'impl': 'reference', 'metric': 'trial structures evaluated/s', 'value': v, 'unit': 'trials/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000 * dt / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': CT_WORKLOAD + ' (sampled rows)'},
        'cpu_baseline': {'value': v, 'unit': 'trials/s', 'cores': cores, 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'trials/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


def main_ct(args, world, rank, local, emit=True):
    """One step = CT_EVALS_PER_STEP evaluations of all 16384 replicas (split of I
    into bf16 parts, the banded product, FP64 chi^2 per replica), so the
    timed region is long enough to sample the clocks.  value: replicas per
    second from CUDA events, I resident (196 MB, larger than L2); e2e: the
    same through p6_ct_run_host from pinned host memory (I in, chi^2 out)."""
    import torch
    from powder6_b200.contraction import FP32, SPLIT3_BF16, SPLIT_BF16, ContractionSession, banded_problem
    torch.cuda.set_device(local)
    p = banded_problem(seed=1 + rank)
    method = {'split': SPLIT_BF16, 'split3': SPLIT3_BF16}.get(args.method, FP32)
    tensor = method in (SPLIT_BF16, SPLIT3_BF16)
    M, K = p.intensities.shape
    N = p.profile_t.shape[0]
    pinned = torch.empty((M, K), dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = p.intensities
    host = pinned.numpy()
    reps = CT_EVALS_PER_STEP
    with ContractionSession(p, device=local) as s:
        s.set_intensities(host)
        q = s.query()
        for _ in range(args.warmup):
            s.evaluate(method)
            s.synchronize()
        barrier(world)
        l0 = s.query()['launches']
        times = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                t = 0.0
                for _ in range(reps):
                    s.evaluate(method)
                    s.synchronize()
                    t += s.last_ms()
                times.append(t)
        launches = s.query()['launches'] - l0
        total_ms = max_over_ranks(float(sum(times)), world)
        value = world * M * reps * args.steps / (total_ms / 1000.0)
        e2e = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            s.run_host(host, method)
            e2e.append(time.perf_counter() - t0)
        e2e_total = max_over_ranks(float(sum(e2e)), world)
        e2e_value = world * M * args.steps / e2e_total
        # chosen vs plain on this configuration: the time of one evaluation of all
        # replicas with the chosen product against the FP32 CUDA-core products
        cvp = {}
        if world == 1:
            from powder6_b200.contraction import FP32_DENSE, METHOD_NAMES
            s.set_intensities(host)
            for m in (method, FP32_DENSE, FP32):
                s.evaluate(m)
                s.synchronize()
                s.evaluate(m)
                s.synchronize()
                cvp[METHOD_NAMES[m]] = s.last_ms()
            cvp = {'chosen': METHOD_NAMES[method], 'ms_per_evaluation': cvp,
                   'ratio_vs_fp32_dense': cvp[METHOD_NAMES[FP32_DENSE]] / cvp[METHOD_NAMES[method]],
                   'ratio_vs_fp32_banded': cvp[METHOD_NAMES[FP32]] / cvp[METHOD_NAMES[method]],
                   'note': 'one evaluation of all replicas (split, product, chi^2); the plain method is the '
                           'dense FP32 render of every reflection at every point'}
    if rank == 0:
        clocks = clk.summary()
        ms = float(np.mean(times))
        ms_eval = ms / reps
        n_mt = (M + 127) // 128
        if tensor:
            products = 3 if method == SPLIT_BF16 else 6
            flops = products * 2.0 * 128 * 256 * 64 * q['band_kblocks'] * n_mt
            note = f'executed tcgen05 MMA flops ({products} bf16 products per K step over each tile band)'
            peak = measured_peak('bf16_tflops')
        else:
            flops = 2.0 * 128 * 128 * q['band_cols128'] * n_mt
            note = 'executed FP32 FMA flops over each tile band'
            peak = (None, None)
        useful = 2.0 * M * float(np.count_nonzero(p.profile_t))
        achieved = flops / (ms_eval / 1000.0) / 1e12
        line = {
            'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None,
            'dtype': ('bf16x3 split, fp32 accumulate, fp64 chi2' if method == SPLIT_BF16 else
                      'bf16 three-part split (6 products), fp32 accumulate, fp64 chi2' if method == SPLIT3_BF16 else
                      'fp32, fp64 chi2'),
            'data': 'synthetic',
            'config': {'workload': CT_WORKLOAD, 'method': args.method, 'replicas': M, 'reflections': K, 'points': N,
                       'step': f'{reps} evaluations of all {M} replicas', 'ms_per_evaluation': ms_eval,
                       'l2': 'inputs larger than L2 (I is 196 MB)', 'parallelism': f'replicas only x{world}'},
            'roofline': {'bound': 'tensor' if tensor else 'fp32', 'achieved': achieved,
                         'peak': peak[0], 'unit': 'TFLOP/s',
                         'frac': achieved / peak[0] if peak[0] else None, 'traffic': None,
                         'note': f'{note}: {flops:.4g} per launch; useful banded flops {useful:.4g}; '
                                 f'dense-equivalent {2.0 * M * K * N:.4g}; peak {peak[1]}'},
            'e2e': {'value': e2e_value, 'unit': 'trials/s', 'h2d_bytes_per_step': M * K * 4,
                    'd2h_bytes_per_step': M * 8},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        if cvp:
            line['chosen_vs_plain'] = cvp
        if not args.no_cpu_baseline and world == 1:
            trials, dt = ct_cpu_rows(p, 10.0)
            line['cpu_baseline'] = {'value': trials / dt, 'unit': 'trials/s', 'cores': os.cpu_count(),
                                    'kind': 'port',
                                    'sample': f'{trials} replicas in blocks of 256 rows, FP64 product with the full '
                                              f'profile matrix (host BLAS), {dt:.1f} s'}
        if emit:
            print(json.dumps(line), flush=True)
        return line


BATCH_GENERATIONS = 2000


def main_batch(args, world, rank, local):
    """One step = all 64 uneven searches (space groups P-1, P2_1/c, C2/c, Pnma,
    P6_3/m, Fm-3m; 1-24 sites; 256-2048 replicas) through BATCH_GENERATIONS
    generations each, in one persistent launch replayed from a CUDA graph,
    with the launch shape the autotuner picked.  value: replica-generations
    per second (CUDA events); the same searches launched one after another
    are timed beside it ('sequential')."""
    import torch
    from powder6_b200.batch import WyckoffBatch, autotune, reset, setup_searches
    from powder6_b200.swarm_wyckoff import SW_DEFAULTS, schedule
    from powder6_b200.workloads import batched_problems
    torch.cuda.set_device(local)
    items = batched_problems(64, seed=1 + rank)
    setup = setup_searches(items, BATCH_GENERATIONS, seed=1 + rank)
    n = len(setup.sessions)
    swap = int(SW_DEFAULTS['swapEvery'])
    try:
        with WyckoffBatch(setup.sessions) as b:
            tuning = autotune(b, setup)
            for _ in range(args.warmup):
                reset(setup)
                b.run([0] * n, setup.generations, swap, True, use_graph=True)
                b.synchronize()
            barrier(world)
            l0 = b.query()['launches']
            times = []
            with ClockSampler(local) as clk:
                for _ in range(args.steps):
                    reset(setup)
                    torch.cuda.synchronize()
                    b.run([0] * n, setup.generations, swap, True, use_graph=True)
                    b.synchronize()
                    times.append(b.last_ms())
            launches = b.query()['launches'] - l0
            q = b.query()
        # the same searches, one launch each
        reset(setup)
        seq = 0.0
        for s_ in setup.sessions:
            s_.run(0, BATCH_GENERATIONS, swap, True)
            s_.synchronize(600)
            seq += s_.last_kernel_ms()
        # end to end: host states in, one batched run, states out
        e2e = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            reset(setup)
            b2 = WyckoffBatch(setup.sessions)
            b2.set_launch(tuning['ctas_per_sm'], tuning['order'])
            b2.run([0] * n, setup.generations, swap, True, use_graph=False)
            b2.synchronize()
            for s_ in setup.sessions:
                s_.read_state()
            e2e.append(time.perf_counter() - t0)
            b2.close()
        trials = int(sum(s_.num_particles * g for s_, g in zip(setup.sessions, setup.generations)))
        cos_total = 0
        for it, s_ in zip(items, setup.sessions):
            g, _ = schedule(BATCH_GENERATIONS, it.problem.refl.n_groups)
            cos_total += algorithmic_cos(it.problem, g, s_.num_particles)[0]
        h2d = sum(s_.num_particles * (s_.coords_per_particle * 4 + 48) for s_ in setup.sessions)
        d2h = sum(s_.num_particles * (2 * s_.coords_per_particle * 4 + 48) for s_ in setup.sessions)
    finally:
        for s_ in setup.sessions:
            s_.close()
    total_ms = max_over_ranks(float(sum(times)), world)
    value = world * trials * args.steps / (total_ms / 1000.0)
    e2e_total = max_over_ranks(float(sum(e2e)), world)
    if rank == 0:
        clocks = clk.summary()
        ms = float(np.mean(times))
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks['sm_mhz'] or 1965.0
        peak = MUFU_PER_CLK_PER_SM * nsm * mhz * 1e6 / 1e9
        achieved = cos_total / (ms / 1000.0) / 1e9
        refl = [it.problem.refl.n_refl for it in items]
        line = {
            'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'fp32', 'data': 'synthetic',
            'config': {'workload': f'{n} uneven Wyckoff searches in one persistent launch (CUDA graph): space groups '
                                   f'P-1, P2_1/c, C2/c, Pnma, P6_3/m, Fm-3m; 1-24 sites; {min(refl)}-{max(refl)} '
                                   f'reflections; 256-2048 replicas; {BATCH_GENERATIONS} generations each',
                       'replicas_total': int(sum(s_ for s_ in [it.replicas for it in items])),
                       'step': 'every search through all its generations, one launch',
                       'l2': 'per-search tables are re-staged by each CTA; states re-uploaded before each step',
                       'tuning': {k: tuning[k] for k in ('ctas_per_sm', 'order', 'probe_ms')},
                       'smem_bytes': q['smem_bytes'], 'items': q['items'],
                       'sequential_ms': seq, 'batched_speedup': seq / ms,
                       'parallelism': f'replicas only x{world}'},
            'roofline': {'bound': 'sfu', 'achieved': achieved, 'peak': peak, 'unit': 'Gcos/s', 'frac': achieved / peak,
                         'traffic': None,
                         'note': f'{cos_total:.4g} algorithmic cosines per step; peak = {MUFU_PER_CLK_PER_SM} SFU '
                                 f'ops/clk/SM x {nsm} SMs x {mhz:.0f} MHz'},
            'e2e': {'value': world * trials * args.steps / e2e_total, 'unit': 'trials/s', 'h2d_bytes_per_step': h2d,
                    'd2h_bytes_per_step': d2h},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        print(json.dumps(line), flush=True)


LEARNED_GENERATIONS = 1000


REFINE_STRUCTURES = 512
REFINE_WORKLOAD = ('Wyckoff-constrained least-squares refinement (coord_refine) of 512 PbSO4-like Pnma structures '
                   '(true coordinates + U(-0.003, 0.003) on every coordinate, seeded), 87 groups of 112 '
                   'reflections, to convergence (at most 60 iterations)')


def refine_starts(P, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([P.true_coords + rng.uniform(-0.003, 0.003, P.true_coords.shape) for _ in range(n)])


def main_refine(args, world, rank, local):
    """One step = the refinement of REFINE_STRUCTURES perturbed structures to
    convergence in one p6_wy_refine call (FP64 group intensities, analytic
    constrained Jacobians and normal equations on the device, the damping
    control of all structures in lock step on the host).  value: structures
    per second, wall time of the C call (it takes and returns host arrays by
    design: the damping control runs on the host); e2e: the same through the
    Python wrapper (array packing included); cpu_baseline: the FP64
    restatement of the algorithm on one host thread, on a sample."""
    import ctypes as C
    import torch
    from powder6_b200 import _lib
    from powder6_b200.swarm_wyckoff import (P6WyRefineOpts, REFINE_DEFAULTS, WyckoffSession, refine_coordinates)
    from powder6_b200.workloads import wyckoff_problem
    torch.cuda.set_device(local)
    P = wyckoff_problem(seed=1)
    n = REFINE_STRUCTURES
    steps_in = [refine_starts(P, n, 100 + 10 * rank + i) for i in range(args.warmup + args.steps)]
    assign = np.zeros(n, dtype=np.uint32)
    walls, e2e, iters, rs, conv = [], [], [], [], []
    with WyckoffSession(P, 64, device=local) as s:
        ro = P6WyRefineOpts(**REFINE_DEFAULTS)
        l0 = 0
        with ClockSampler(local) as clk:
            for i, x0 in enumerate(steps_in):
                x = np.ascontiguousarray(x0, dtype=np.float64).copy()
                r1 = np.zeros(n)
                it = np.zeros(n, dtype=np.int32)
                cv = np.zeros(n, dtype=np.int32)
                if i == args.warmup:
                    l0 = s.launch_count()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                _lib.check(s.lib.p6_wy_refine(s.h, n, _lib.ptr(assign), _lib.ptr(x), C.cast(C.pointer(ro), C.c_void_p),
                                              None, _lib.ptr(r1), None, _lib.ptr(it), _lib.ptr(cv)))
                dt = time.perf_counter() - t0
                if i >= args.warmup:
                    walls.append(dt)
                    iters.append(float(np.mean(it)))
                    rs.append(float(np.median(r1)))
                    conv.append(int(cv.sum()))
        launches = s.launch_count() - l0
        for i in range(args.steps):
            t0 = time.perf_counter()
            refine_coordinates(s, steps_in[args.warmup + i], assign)
            e2e.append(time.perf_counter() - t0)
    total = max_over_ranks(float(sum(walls)), world)
    value = world * n * args.steps / total
    e2e_value = world * n * args.steps / max_over_ranks(float(sum(e2e)), world)
    if rank == 0:
        clocks = clk.summary()
        line = {
            'metric': 'structures refined/s', 'value': value, 'unit': 'structures/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000.0 * total / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': REFINE_WORKLOAD, 'structures': n, 'mean_accepted_steps': float(np.mean(iters)),
                       'median_final_wr': float(np.median(rs)), 'converged_per_step': conv,
                       'step': f'one p6_wy_refine call on {n} structures',
                       'parallelism': f'structures only x{world}'},
            'e2e': {'value': e2e_value, 'unit': 'structures/s', 'h2d_bytes_per_step': n * P.max_sites * 3 * 8 + n * 4,
                    'd2h_bytes_per_step': n * P.max_sites * 3 * 8 + n * 24},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle as O
            sample = refine_starts(P, 64, 7)
            t0 = time.perf_counter()
            done = 0
            for x0 in sample:
                O.wy_refine(P, 0, x0)
                done += 1
                if time.perf_counter() - t0 > 10.0:
                    break
            dt = time.perf_counter() - t0
            line['cpu_baseline'] = {'value': done / dt, 'unit': 'structures/s', 'cores': 1, 'kind': 'port',
                                    'sample': f'{done} structures refined by the FP64 restatement (numpy, one host '
                                              f'thread), {dt:.1f} s'}
        print(json.dumps(line), flush=True)


def run_reference_refine(args, world, rank):
    """The reference arm of the refinement workload: the FP64 restatement of
    refineCoordinatesAgainstWppf on one host thread; each step refines a
    bounded sample of the workload's structures."""
    if rank != 0:
        return
    from oracle import oracle as O
    from powder6_b200.workloads import wyckoff_problem
    P = wyckoff_problem(seed=1)
    per_step = 4
    times = []
    for i in range(args.warmup + args.steps):
        sample = refine_starts(P, per_step, 100 + i)
        t0 = time.perf_counter()
        for x0 in sample:
            O.wy_refine(P, 0, x0)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    v = per_step * args.steps / sum(times)
    print(json.dumps({
        'impl': 'reference', 'metric': 'structures refined/s', 'value': v, 'unit': 'structures/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000.0 * sum(times) / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': REFINE_WORKLOAD, 'sample': f'{per_step} structures per step'},
        'cpu_baseline': {'value': v, 'unit': 'structures/s', 'cores': 1, 'kind': 'port',
                         'sample': f'{per_step} structures per step, FP64 restatement (numpy), one host thread'},
        'e2e': {'value': v, 'unit': 'structures/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}), flush=True)


CF_GRID = 64
CF_TRIALS = 128
CF_CYCLES = 100
CF_WORKLOAD = (f'charge flipping, synthetic P2_1/c structure (9.1 x 7.3 x 10.4 A, beta 104, d >= 0.8 A), '
               f'{CF_GRID}^3 grid, {CF_TRIALS} random starts of the adaptive plan (3 settings), {CF_CYCLES} cycles')


def cf_setup(rank=0, n_trials=CF_TRIALS):
    from powder6_b200.charge_flipping import (build_reflection_model, cf_plan, classify_weak_orbits, synthetic_job)
    job = synthetic_job(grid=CF_GRID, dmin=0.8, seed=1)
    m = build_reflection_model(job, CF_GRID)
    plan = cf_plan(min(128, max(6, n_trials)))
    trials = []
    for i in range(n_trials):
        t = plan['trials'][i % len(plan['trials'])]
        wk = classify_weak_orbits(m, t['weakFraction'], 'cluster')
        trials.append({'threshold': t['threshold'], 'symLambda': t['symLambda'], 'seed': 1000 * rank + i + 1,
                       'weak': wk['flags'] if wk['weakOrbits'] else None})
    return job, m, trials


def cf_cpu_rate(m, trials, seconds):
    """Cycles per second of the FP64 restatement (numpy FFTs, one thread)."""
    from oracle.oracle_cf import CfState
    from powder6_b200.charge_flipping import model_initial_grid
    done, t0 = 0, time.perf_counter()
    st = None
    while time.perf_counter() - t0 < seconds:
        t = trials[done % len(trials)]
        if st is None or done % 10 == 0:
            st = CfState(m, model_initial_grid(m, CF_GRID, t['seed']), t['threshold'], t['symLambda'], t['seed'],
                         t['weak'])
        st.cycle()
        done += 1
    return done / (time.perf_counter() - t0), done


def main_cf(args, world, rank, local):
    """One step = CF_CYCLES cycles of all CF_TRIALS trials (or --cf-cycles, --cf-trials) (one graph replay
    per cycle: six transform passes and the reciprocal step, every trial in
    each launch).  value: trial-cycles per second from CUDA events on the
    session's stream, grids resident; e2e: the same per step through the
    public API with the starting grids uploaded from pinned host memory
    (set_grid), the run, the best R read back and the best trial's density
    map read back; the grids (128 x 2 MB) exceed L2, so no flush is needed."""
    import torch
    from powder6_b200.charge_flipping import CFSession, model_initial_grid
    torch.cuda.set_device(local)
    n_trials = args.cf_trials or CF_TRIALS
    cycles = args.cf_cycles or CF_CYCLES
    job, m, trials = cf_setup(rank, n_trials)
    # the starting grids in pinned host memory, as an application streaming
    # starts would hold them (the e2e leg uploads them every step)
    pinned = torch.empty((n_trials, 2 * CF_GRID ** 3), dtype=torch.float32).pin_memory()
    for i, t in enumerate(trials):
        pinned[i] = torch.from_numpy(model_initial_grid(m, CF_GRID, t['seed']))
    starts = [pinned[i].numpy() for i in range(n_trials)]
    ms, e2e = [], []
    with CFSession(m, trials, device=local) as s:
        for i, g in enumerate(starts):
            s.set_grid(g, i)
        for _ in range(args.warmup):
            s.run(cycles)
        l0 = s.launch_count()
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                s.run(cycles)
                ms.append(s.last_ms())
        launches = s.launch_count() - l0
        fft_ms, rec_ms = s.time_kernels(3)
        for _ in range(args.steps):
            t0 = time.perf_counter()
            for i, g in enumerate(starts):
                s.set_grid(g, i)
            s.run(cycles)
            best = s.best_r()
            s.read(int(np.argmin(best)), 'map')
            e2e.append(time.perf_counter() - t0)
    total_ms = max_over_ranks(float(sum(ms)), world)
    units = world * n_trials * cycles * args.steps
    value = units / (total_ms / 1000.0)
    e2e_value = units / max_over_ranks(float(sum(e2e)), world)
    if rank == 0:
        cells = CF_GRID ** 3
        pass_bytes = 2 * cells * 8 * n_trials            # read + write every trial's grid once
        achieved = pass_bytes / (fft_ms * 1e-3) / 1e9
        peak, peak_note = measured_peak('hbm_gbs')
        clocks = clk.summary()
        traffic = None
        tf = ROOT / 'profiles' / 'cf_fft_traffic.txt'
        if tf.exists() and n_trials == CF_TRIALS:
            for ln in tf.read_text().splitlines():
                if ln.startswith('bytes_per_pass:'):
                    traffic = int(ln.split(':', 1)[1])
        line = {
            'metric': 'charge-flipping trial-cycles/s', 'value': value, 'unit': 'cycles/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': CF_WORKLOAD if (n_trials, cycles) == (CF_TRIALS, CF_CYCLES) else
                       f'{CF_WORKLOAD} (run with {n_trials} starts, {cycles} cycles)',
                       'grid': CF_GRID, 'trials': n_trials, 'cycles_per_step': cycles,
                       'orbits': m['nOrbits'], 'clusters': m['nClusters'], 'members': m['nMembers'],
                       'l2': f'grids {n_trials * cells * 8 / 1e6:.0f} MB' + (' > L2, no flush' if n_trials * cells * 8 > 126e6
                                                                      else ' (in L2)'),
                       'fft_pass_ms': fft_ms, 'reciprocal_ms': rec_ms,
                       'parallelism': f'trials only x{world}'},
            'e2e': {'value': e2e_value, 'unit': 'cycles/s', 'h2d_bytes_per_step': n_trials * cells * 8,
                    'd2h_bytes_per_step': n_trials * 4 + cells * 4 + n_trials * cycles * 4},
            'roofline': {'kernel': 'cf_fft_kernel<64>', 'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                         'unit': 'GB/s', 'frac': achieved / peak if peak else None, 'peak_source': peak_note,
                         'traffic': traffic, 'unit_of_launch': f'one pass over all {n_trials} trials',
                         'algorithmic_bytes_per_launch': pass_bytes},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        if not args.no_cpu_baseline and world == 1:
            rate, done = cf_cpu_rate(m, trials, 10.0)
            line['cpu_baseline'] = {'value': rate, 'unit': 'cycles/s', 'cores': 1, 'kind': 'port',
                                    'sample': f'{done} cycles of the FP64 restatement (numpy FFTs, one thread) on '
                                              f'the same model, trials in turn'}
        print(json.dumps(line), flush=True)


def run_reference_cf(args, world, rank):
    """The reference arm of the charge-flipping workload: the FP64
    restatement of the cycle (numpy FFTs, one host thread); each step is a
    bounded sample of 10 trial-cycles."""
    if rank != 0:
        return
    from oracle.oracle_cf import CfState
    from powder6_b200.charge_flipping import model_initial_grid
    job, m, trials = cf_setup(0)
    times, per_step = [], 10
    for i in range(args.warmup + args.steps):
        t = trials[i % len(trials)]
        st = CfState(m, model_initial_grid(m, CF_GRID, t['seed']), t['threshold'], t['symLambda'], t['seed'],
                     t['weak'])
        t0 = time.perf_counter()
        for _ in range(per_step):
            st.cycle()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    v = per_step * args.steps / sum(times)
    print(json.dumps({
        'impl': 'reference', 'metric': 'charge-flipping trial-cycles/s', 'value': v, 'unit': 'cycles/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000.0 * sum(times) / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': CF_WORKLOAD, 'sample': f'{per_step} cycles of one trial per step'},
        'cpu_baseline': {'value': v, 'unit': 'cycles/s', 'cores': 1, 'kind': 'port',
                         'sample': f'{per_step} cycles of one trial per step, FP64 restatement (numpy), one thread'},
        'e2e': {'value': v, 'unit': 'cycles/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}), flush=True)


def main_learned(args, world, rank, local):
    """One step = one learned-proposal search (P2_1/c, 17 independent C/N/S
    sites, 575 reflections, 8192 replicas, LEARNED_GENERATIONS generations; 8
    candidates per replica ranked by the network, the best evaluated with the
    exact fitness).  The network is trained beforehand (outside the timed
    region) on 819k moves of the plain search.  value: replica-generations
    per second over the device span of the search loop; time_to_target:
    wall seconds to a best wR2 within 1.05x the wR2 a plain search of the
    same length reaches, for the learned search and for the plain fused
    search from the same starts."""
    import torch
    from powder6_b200.learned import ProposalNet, collect_records, gain_targets, learned_problem, run as lrun
    from powder6_b200.swarm_wyckoff import WyckoffSession, run_wyckoff_search, schedule
    torch.cuda.set_device(local)
    P = learned_problem()
    n, G = 8192, LEARNED_GENERATIONS
    with WyckoffSession(P, n, run_key=77 + rank, incremental=0, device=local) as s:
        X, gains, _ = collect_records(s, P, 200, seed=4 + rank, every=2)
        T, _ = gain_targets(gains)
        net = ProposalNet(64, 256, 1, seed=7, device=local)
        t0 = time.perf_counter()
        losses = net.train(X, T, epochs=8, batch=2048, lr=1e-3)
        train_s = time.perf_counter() - t0
        conv = run_wyckoff_search(P, num_particles=n, generations=G, seed=31, session=s, do_quench=False)
        target = 1.0 - 1.05 * (1.0 - conv.best_cc)
        for i in range(args.warmup):
            lrun(s, P, 200, seed=50 + i, net=net, K=8, check_every=100)
        barrier(world)
        dev_ms, ttt_l, ttt_p, best_l, best_p, e2e = [], [], [], [], [], []
        l0 = s.launch_count()
        with ClockSampler(local) as clk:
            for i in range(args.steps):
                t0 = time.perf_counter()
                tr = lrun(s, P, G, seed=100 + i, net=net, K=8, check_every=100, target_cc=target)
                s.read_state()
                e2e.append(time.perf_counter() - t0)
                dev_ms.append(tr.device_ms)
                ttt_l.append(tr.time_to_target)
                best_l.append(tr.best_cc[-1])
        launches = s.launch_count() - l0
        for i in range(args.steps):
            r = run_wyckoff_search(P, num_particles=n, generations=G, seed=100 + i, chunk=100, session=s,
                                   do_quench=False, target_cc=target)
            ttt_p.append(r.time_to_target)
            best_p.append(r.best_cc)
        net.close()
    total_ms = max_over_ranks(float(sum(dev_ms)), world)
    value = world * n * G * args.steps / (total_ms / 1000.0)
    if rank == 0:
        clocks = clk.summary()
        groups, _ = schedule(G, P.refl.n_groups)
        cos_total = algorithmic_cos(P, groups, n)[0]
        ms = float(np.mean(dev_ms))
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks['sm_mhz'] or 1965.0
        peak = MUFU_PER_CLK_PER_SM * nsm * mhz * 1e6 / 1e9
        achieved = cos_total / (ms / 1000.0) / 1e9

        def med(v):
            v = [x for x in v if x is not None]
            return float(np.median(v)) if v else None
        line = {
            'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'fp32 fitness, bf16 network', 'data': 'synthetic',
            'config': {'workload': f'learned-proposal Wyckoff search: P2_1/c a=10.2 b=12.1 c=15.3 beta=100, 17 C/N/S '
                                   f'sites (68 atoms), {P.refl.n_refl} reflections to d_min 1.5 A, {n} replicas x {G} '
                                   f'generations, 8 candidates ranked per replica by a 64-256-256-1 MLP',
                       'training': {'records': int(len(X)), 'epochs': 8, 'seconds': train_s,
                                    'loss_first_last': [float(losses[0]), float(losses[-1])]},
                       'step': 'one learned search, one launch of each kernel per generation',
                       'parallelism': f'replicas only x{world}'},
            'time_to_target_wr2': {'target_wr2': 1.0 - target, 'reference_wr2_plain': 1.0 - conv.best_cc,
                                   'learned_median_s': med(ttt_l), 'plain_median_s': med(ttt_p),
                                   'learned_reached': f'{sum(t is not None for t in ttt_l)}/{len(ttt_l)}',
                                   'plain_reached': f'{sum(t is not None for t in ttt_p)}/{len(ttt_p)}',
                                   'best_wr2_learned': [1.0 - b for b in best_l],
                                   'best_wr2_plain': [1.0 - b for b in best_p]},
            'roofline': {'bound': 'sfu', 'achieved': achieved, 'peak': peak, 'unit': 'Gcos/s', 'frac': achieved / peak,
                         'traffic': None,
                         'note': f'{cos_total:.4g} algorithmic cosines per step (exact evaluations only)'},
            'e2e': {'value': world * n * G * args.steps / max_over_ranks(float(sum(e2e)), world), 'unit': 'trials/s',
                    'h2d_bytes_per_step': n * (51 * 4 + 48), 'd2h_bytes_per_step': n * (2 * 51 * 4 + 48)},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        print(json.dumps(line), flush=True)


FRAGMENT_GENERATIONS = 15000
FRAGMENT_SEEDS = (11, 12, 13, 14)


def main_fragment(args, world, rank, local):
    """Config 5 as a rigid fragment: cimetidine (17 non-H atoms, 6 torsions)
    on 4e of P2_1/c, 8192 replicas from random placements, every reflection
    at the final penalty weight, scored on its powder pattern (5895 points,
    575 reflections): chi^2 at the best scale from the three-part split-BF16
    contraction (the chosen form), from the dense FP32 render (plain), and
    in Gram form inside the fused search.  Per seed (the first --steps of
    FRAGMENT_SEEDS) each method searches up to FRAGMENT_GENERATIONS
    generations; time to target: wall seconds from the first evaluation to
    the first 500-generation boundary with a best Rwp <= 1.05 x the true
    structure's.  value: trials/s of the chosen method from CUDA events."""
    import torch
    from powder6_b200.contraction import FP32_DENSE, SPLIT3_BF16
    from powder6_b200.fragment import fragment_problem, run_fragment_pattern_search
    from powder6_b200.profile_search import GRAM_FP64, METHOD_NAMES, profile_problem
    torch.cuda.set_device(local)
    P, frag, _ = fragment_problem(seed=1)
    pp = profile_problem(P, seed=1)
    target = 1.05 * pp.rwp_true
    n = 8192
    methods = (SPLIT3_BF16, FP32_DENSE, GRAM_FP64)
    runs = {m: [] for m in methods}
    with ClockSampler(local) as clk:
        for seed in FRAGMENT_SEEDS[:max(1, args.steps)]:
            for m in methods:
                runs[m].append(run_fragment_pattern_search(P, frag, pp, m, n, FRAGMENT_GENERATIONS, seed=seed,
                                                           chunk=500, target_rwp=target))
    if rank != 0:
        return
    clocks = clk.summary()

    def summary(rs):
        hits = [r['time_to_target'] for r in rs if r['time_to_target'] is not None]
        us = [1000.0 * r['device_ms'] / max(1, r['generations']) for r in rs]
        return {'median_s': float(np.median(hits)) if hits else None, 'reached': f'{len(hits)}/{len(rs)}',
                'final_rwp': [r['best_rwp'] for r in rs],
                'generations_to_target': [r['generations_to_target'] for r in rs],
                'us_per_generation': float(np.median(us))}
    ttt = {METHOD_NAMES[m]: summary(runs[m]) for m in methods}
    chosen, plain, gram = (ttt[METHOD_NAMES[m]] for m in methods)
    both = [(a['time_to_target'], b['time_to_target']) for a, b in zip(runs[SPLIT3_BF16], runs[FP32_DENSE])
            if a['time_to_target'] is not None and b['time_to_target'] is not None]
    cr = runs[SPLIT3_BF16]
    value = n * sum(r['generations'] for r in cr) / (sum(r['device_ms'] for r in cr) / 1000.0)
    line = {
        'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
        'steps': len(cr), 'warmup': 0, 'ms_per_step': float(np.mean([r['device_ms'] for r in cr])),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'fp64 |F|^2, bf16 three-part split (6 products) fp32 accumulate, fp64 chi2', 'data': 'synthetic',
        'config': {'workload': f'rigid-fragment search, cimetidine (C10N6S, 17 non-H atoms, 6 torsions) on 4e of '
                               f'P2_1/c (10.2 x 12.1 x 15.3 A, beta 100), {P.refl.n_refl} reflections to 1.5 A, '
                               f'pattern {pp.n_points} points, {n} replicas from random placements, up to '
                               f'{FRAGMENT_GENERATIONS} generations per search',
                   'step': 'one search per seed and method', 'parallelism': f'replicas only x{world}'},
        'roofline': None,
        'e2e': None,
        'gpu_launches': None,
        'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        'time_to_target_rwp': {'target_rwp': target, 'converged_rwp': pp.rwp_true, 'methods': ttt,
                               'chosen': METHOD_NAMES[SPLIT3_BF16], 'plain': METHOD_NAMES[FP32_DENSE],
                               'chosen_s': chosen['median_s'], 'plain_s': plain['median_s'],
                               'ratio_seeds_both_reached': [b / a for a, b in both],
                               'gram_s': gram['median_s'],
                               'note': 'target 1.05 x the true structure\'s FP64 Rwp; chunks of 500 generations; '
                                       'seeds ' + ', '.join(str(x) for x in FRAGMENT_SEEDS[:len(cr)])},
    }
    print(json.dumps(line), flush=True)


def run_reference_profile(args, world, rank):
    if rank != 0:
        return
    from powder6_b200.profile_search import profile_problem
    pp = profile_problem()
    for _ in range(args.warmup):
        profile_cpu_rate(pp, 0.3)
    trials, dt = profile_cpu_rate(pp, 2.0 * args.steps)
    v = trials / dt
    sample = f'{trials} random structures, FP64 oracle port (per-reflection |F|^2, fitted-scale chi^2), one thread'
    print(json.dumps({
        'impl': 'reference', 'metric': 'trial structures evaluated/s', 'value': v, 'unit': 'trials/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1000 * dt / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': PROFILE_WORKLOAD + ' (sampled trials)'},
        'cpu_baseline': {'value': v, 'unit': 'trials/s', 'cores': 1, 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'trials/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


def main_profile(args, world, rank, local, emit=True):
    """The fixed-profile Wyckoff search.  One step = PROFILE_CHUNK generations
    of all 4096 replicas with the chosen method (search kernel, three-part
    split-BF16 contraction with the fitted scale, acceptance and exchange per
    generation).  value: trials/s from CUDA events on the search's stream,
    L2 flushed before each step; e2e: the same through the host API with
    host buffers (positions and states uploaded, the chunk, positions, bests
    and states read back).  The roofline is the contraction's (the largest
    share of a generation), timed alone on the same shapes."""
    import torch
    from powder6_b200.contraction import ContractionSession
    from powder6_b200.profile_search import SPLIT3_BF16, ProfileSearch, _ContractionInput, profile_problem
    from powder6_b200.swarm_wyckoff import STATE_DTYPE
    torch.cuda.set_device(local)
    pp = profile_problem()
    n = args.particles
    method = SPLIT3_BF16
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f'cuda:{local}')
    G = max(PROFILE_GENERATIONS, PROFILE_CHUNK * (args.steps + args.warmup))
    with ProfileSearch(pp, n, run_key=5 + rank) as ps:
        ps.start(G, seed=5 + rank, method=method)
        ps.synchronize()
        g0 = 0
        for _ in range(args.warmup):
            ps.run(g0, PROFILE_CHUNK, method)
            g0 += PROFILE_CHUNK
        ps.synchronize()
        barrier(world)
        l0 = ps.wy.launch_count() + ps.ct.query()['launches']
        times = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                ps.run(g0, PROFILE_CHUNK, method)
                ps.synchronize()
                times.append(ps.last_ms())
                g0 += PROFILE_CHUNK
        launches = ps.wy.launch_count() + ps.ct.query()['launches'] - l0
        total_ms = max_over_ranks(float(sum(times)), world)
        value = world * n * PROFILE_CHUNK * args.steps / (total_ms / 1000.0)
        # end to end: host positions and states in, the chunk, positions, bests and states out
        pos, _, st = ps.wy.read_state()
        pin_pos = torch.empty(len(pos), dtype=torch.float32, pin_memory=True).numpy()
        pin_pos[:] = pos
        pin_st = torch.empty(len(st) * STATE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True).numpy().view(
            STATE_DTYPE)
        pin_st[:] = st
        e2e = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ps.wy.sync_state(pin_pos, pin_st)
            ps.run(g0 % (G - PROFILE_CHUNK), PROFILE_CHUNK, method)
            ps.synchronize()
            cur, best, stb = ps.wy.read_state()
            e2e.append(time.perf_counter() - t0)
        e2e_value = world * n * PROFILE_CHUNK * args.steps / max_over_ranks(float(sum(e2e)), world)
        h2d = pin_pos.nbytes + pin_st.nbytes
        d2h = 2 * pin_pos.nbytes + pin_st.nbytes
    # the contraction alone on the same shapes (split, product, fitted reduction)
    rng = np.random.default_rng(3)
    I = rng.lognormal(0.0, 1.5, (n, pp.n_refl)).astype(np.float32)
    with ContractionSession(_ContractionInput(pp), max_replicas=n, device=local) as s:
        s.set_fitted(True)
        s.set_intensities(I)
        q = s.query()
        for _ in range(5):
            s.evaluate(method)
        s.synchronize()
        ct_ms = []
        for _ in range(20):
            s.evaluate(method)
            s.synchronize()
            ct_ms.append(s.last_ms())
    if rank != 0:
        return None
    clocks = clk.summary()
    ms = float(np.mean(times))
    ms_gen = ms / PROFILE_CHUNK
    ct_eval = float(np.median(ct_ms))
    n_mt = (n + 127) // 128
    flops = 6 * 2.0 * 128 * 256 * 64 * q['band_kblocks'] * n_mt
    peak = measured_peak('bf16_tflops')
    achieved = flops / (ct_eval / 1000.0) / 1e12
    line = {
        'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'fp64 |F|^2, bf16 three-part split (6 products) fp32 accumulate, fp64 chi2',
        'data': 'synthetic',
        'config': {'workload': PROFILE_WORKLOAD, 'method': 'split3-bf16', 'replicas': n,
                   'reflections': pp.n_refl, 'points': pp.n_points,
                   'step': f'{PROFILE_CHUNK} generations of all {n} replicas', 'us_per_generation': 1000 * ms_gen,
                   'l2': 'flushed before every step (256 MB write)', 'parallelism': f'replicas only x{world}'},
        'roofline': {'bound': 'tensor', 'achieved': achieved, 'peak': peak[0], 'unit': 'TFLOP/s',
                     'frac': achieved / peak[0] if peak[0] else None, 'traffic': None,
                     'note': f'contraction (split, tcgen05 product, fitted reduction) timed alone on the same '
                             f'shapes: {ct_eval:.4f} ms per evaluation, {100 * ct_eval / ms_gen:.0f} % of a '
                             f'generation; executed MMA flops {flops:.4g} (six bf16 products over each tile band); '
                             f'peak {peak[1]}'},
        'e2e': {'value': e2e_value, 'unit': 'trials/s', 'h2d_bytes_per_step': int(h2d),
                'd2h_bytes_per_step': int(d2h)},
        'gpu_launches': int(launches),
        'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
    }
    if not args.no_cpu_baseline and world == 1:
        trials, dt = profile_cpu_rate(pp, 10.0)
        line['cpu_baseline'] = {'value': trials / dt, 'unit': 'trials/s', 'cores': 1, 'kind': 'port',
                                'sample': f'{trials} random structures through the FP64 oracle (per-reflection '
                                          f'|F|^2 and the fitted-scale chi^2 over 7680 points), {dt:.1f} s'}
    if world == 1:
        line['time_to_target_rwp'] = profile_time_to_target(pp, n)
    if emit:
        print(json.dumps(line), flush=True)
    return line


PROFILE_GENERATIONS = 2000
PROFILE_CHUNK = 100
PROFILE_TTT_CHUNK = 50
PROFILE_SEEDS = 8
PROFILE_WORKLOAD = ('fixed-profile Wyckoff search: the Pnma PbSO4-like structure (Pb 4c, S 4c, O 4c, O 4c, O 8d) '
                    'against its powder pattern (Cu Ka1/Ka2, 5-81.8 deg at 0.01 deg: 7680 points, 112 reflections, '
                    'pseudo-Voigt at +/-20 FWHM, Poisson counts, peak 1e4), 4096 replicas, fitness 1 - Rwp at '
                    'the best scale - penalty')


def profile_cpu_rate(pp, seconds):
    """The FP64 oracle's trial evaluation on the host (one thread): the
    per-reflection mult |F|^2 of a random structure and the fitted-scale
    chi^2 over the whole pattern.  Returns (trials, seconds)."""
    from oracle import oracle as O
    prob = pp.problem
    ms = prob.tables.max_sites
    rng = np.random.default_rng(7)
    PT = pp.profile_t.astype(np.float64)
    t0 = time.perf_counter()
    done = 0
    while time.perf_counter() - t0 < seconds:
        x = np.zeros(ms * 3)
        for si, s in enumerate(prob.assignments[0].sites):
            x[si * 3:si * 3 + 3] = np.array(s.w.project(*rng.random(3))) % 1.0
        I = O.wy_reflection_intensities(prob, 0, x)
        O.profile_fitted_chi2(I[None, :], PT, pp.yobs, pp.w)
        done += 1
    return done, time.perf_counter() - t0


def profile_time_to_target(pp, n, seeds=PROFILE_SEEDS):
    """Time to target Rwp, the chosen method against the plain one, on the
    same search (proposals, ladders, schedule, seeds): the chosen form runs
    the pattern as the three-part split-BF16 product on the tensor cores
    (chi^2 within 1e-6 of FP64); the plain form renders every reflection at
    every point in FP32 on the CUDA cores, the reference's dense
    `columns`/`targets` stages; the band-limited FP32 product is shown
    beside them, and the Gram form (chi^2 at the best scale from v . I and
    I G I^T in FP64 inside the fused search: no pattern formed).  The target is 1.05 x the FP64 Rwp of the structure the
    pattern was made from (the converged value of a search that solves it).
    Wall time from the first evaluation of the random start (the host's
    drawing and upload of it excluded) to the first 50-generation boundary
    at or below the target; median over ``seeds`` seeds."""
    from powder6_b200.profile_search import FP32, FP32_DENSE, GRAM_FP64, METHOD_NAMES, SPLIT3_BF16, ProfileSearch, \
        run_profile_search
    target = 1.05 * pp.rwp_true
    out = {'target_rwp': target, 'converged_rwp': pp.rwp_true,
           'target_source': 'FP64 Rwp of the generating structure at its best scale (the noise floor)'}
    med = {}
    with ProfileSearch(pp, n, run_key=17) as ps:
        for m in (SPLIT3_BF16, FP32_DENSE, FP32, GRAM_FP64):
            runs = [run_profile_search(pp, n, PROFILE_GENERATIONS, seed=301 + k, method=m, chunk=PROFILE_TTT_CHUNK,
                                       target_rwp=target, search=ps, stop_at_target=True) for k in range(seeds)]
            hits = [r.time_to_target for r in runs if r.time_to_target is not None]
            gens = [r.generations_to_target for r in runs if r.generations_to_target is not None]
            med[m] = float(np.median(hits)) if hits else None
            out[METHOD_NAMES[m]] = {'median_s': med[m], 'reached': f'{len(hits)}/{len(runs)}',
                                    'median_generations': float(np.median(gens)) if gens else None,
                                    'final_rwp': [r.best_rwp for r in runs],
                                    'cpu_check_delta': [r.cpu_check.get('delta') for r in runs]}
    out['chosen'] = METHOD_NAMES[SPLIT3_BF16]
    out['plain'] = METHOD_NAMES[FP32_DENSE]
    out['chosen_s'] = med[SPLIT3_BF16]
    out['plain_s'] = med[FP32_DENSE]
    out['ratio'] = (med[FP32_DENSE] / med[SPLIT3_BF16]) if med[SPLIT3_BF16] and med[FP32_DENSE] else None
    out['ratio_vs_fp32_banded'] = (med[FP32] / med[SPLIT3_BF16]) if med[SPLIT3_BF16] and med[FP32] else None
    # the exact reformulation: no pattern formed, the whole search in one fused launch
    out['gram_s'] = med[GRAM_FP64]
    out['ratio_gram_vs_plain'] = (med[FP32_DENSE] / med[GRAM_FP64]) if med[GRAM_FP64] and med[FP32_DENSE] else None
    out['note'] = (f'chunks of {PROFILE_TTT_CHUNK} generations, {n} replicas, stop at the target; '
                   f'median over {seeds} seeds')
    return out


def measured_peak(key):
    f = ROOT / 'MEASURED_PEAKS.json'
    if f.exists():
        try:
            v = json.loads(f.read_text()).get(key)
            if v:
                return float(v), 'of measured (MEASURED_PEAKS.json ' + key + ')'
        except (ValueError, OSError):
            pass
    fallback = {'bf16_tflops': 1590.0, 'hbm_gbs': 6650.0}
    return fallback.get(key), 'of fallback'


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == 'reference':
        if args.workload == 'pt':
            run_reference_pt(args, world, rank)
        elif args.workload == 'contract':
            run_reference_ct(args, world, rank)
        elif args.workload == 'batch':
            run_reference_batch(args, world, rank)
        elif args.workload == 'refine':
            run_reference_refine(args, world, rank)
        elif args.workload == 'cf':
            run_reference_cf(args, world, rank)
        elif args.workload == 'profile':
            run_reference_profile(args, world, rank)
        elif args.workload == 'fragment':
            if rank == 0:
                print(json.dumps({'impl': 'reference', 'unavailable': 'the FP64 oracle restates the trial '
                                  'evaluation, not a fragment search; its pattern trial rate is the profile '
                                  'workload\'s reference arm'}), flush=True)
        else:
            run_reference(args, world, rank)
        return
    if args.workload in ('pt', 'contract', 'batch', 'learned', 'refine', 'cf', 'profile', 'fragment'):
        {'pt': main_pt, 'contract': main_ct, 'batch': main_batch, 'learned': main_learned,
         'refine': main_refine, 'cf': main_cf, 'profile': main_profile, 'fragment': main_fragment}[args.workload](
            args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from powder6_b200.swarm_wyckoff import (COS_FACTORED, COS_NAMES, WyckoffSession, build_ladders,
                                            default_cos_mode, initial_state, project_all, schedule)
    from powder6_b200.workloads import mulberry32, wyckoff_problem
    torch.cuda.set_device(local)
    P = wyckoff_problem(seed=1)
    n = args.particles
    G = args.generations
    groups, pen = schedule(G, P.refl.n_groups)
    if args.cos_mode < 0:
        args.cos_mode = default_cos_mode(P)
    sess = WyckoffSession(P, n, run_key=1000 + rank, cos_mode=args.cos_mode, device=local)
    assign = np.zeros(n, dtype=np.uint32)
    sess.set_assign(assign)
    ladders, temps = build_ladders(assign)
    sess.set_ladders(ladders, 8)
    sess.set_schedule(groups, pen)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    rnd = mulberry32(20261026 + rank)

    def fresh_inputs():
        pos = project_all(P, np.array([rnd() for _ in range(n * sess.coords_per_particle)], dtype=np.float32), assign)
        st = initial_state(n, temps, rnd)
        return pos, st

    def device_step(pos, st):
        sess.sync_state(pos, st)           # inputs resident before the timed kernel
        flush.zero_()
        torch.cuda.synchronize()
        sess.run(0, G, SWAP_EVERY, True)
        sess.synchronize(600)
        return sess.last_kernel_ms()

    inputs = [fresh_inputs() for _ in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        device_step(*inputs[i])
    barrier(world)
    torch.cuda.synchronize()
    l0 = sess.launch_count()
    with ClockSampler(local) as clk:
        times = [device_step(*inputs[args.warmup + i]) for i in range(args.steps)]
    torch.cuda.synchronize()
    barrier(world)
    launches = sess.launch_count() - l0
    total_ms = max_over_ranks(float(sum(times)), world)
    trials_per_step = n * G
    value = world * trials_per_step * args.steps / (total_ms / 1000.0)
    # end to end through the host-buffer C-ABI call: upload, search, read back
    pos, st = inputs[-1]
    torch.cuda.synchronize()
    e2e_times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        sess.run_host(pos, st, 0, G, SWAP_EVERY, True)
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(float(sum(e2e_times)), world)
    e2e_value = world * trials_per_step * args.steps / e2e_total
    h2d = n * sess.coords_per_particle * 4 + n * 48
    d2h = 2 * n * sess.coords_per_particle * 4 + n * 48
    if rank == 0:
        clocks = clk.summary()
        cos_total, nsteps = algorithmic_cos(P, groups, n)
        ms = float(np.mean(times))
        achieved = cos_total / (ms / 1000.0) / 1e9
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clocks['sm_mhz'] or 1965.0
        peak = MUFU_PER_CLK_PER_SM * nsm * mhz * 1e6 / 1e9
        traffic, inst_per_trial = None, None
        tf = ROOT / 'profiles' / 'wy_kernel_traffic.txt'
        if tf.exists():
            for ln in tf.read_text().splitlines():
                if ln.startswith('bytes_per_launch:'):
                    traffic = int(ln.split(':', 1)[1])
                if ln.startswith('warp_instructions_per_trial:'):
                    inst_per_trial = float(ln.split(':', 1)[1])
        sfu = {'bound': 'sfu', 'achieved': achieved, 'peak': peak, 'unit': 'Gcos/s', 'frac': achieved / peak,
               'traffic': traffic,
               'note': f'{cos_total:.4g} algorithmic cosines per launch (the reference\'s count); peak = '
                       f'{MUFU_PER_CLK_PER_SM} SFU ops/clk/SM x {nsm} SMs x {mhz:.0f} MHz (median SM clock under load)'}
        if args.cos_mode == COS_FACTORED and inst_per_trial:
            # the factored evaluation issues no cosine per term: the bound is instruction issue
            issue_peak = 4 * nsm * mhz * 1e6 / 1e9
            issued = inst_per_trial * trials_per_step / (ms / 1000.0) / 1e9
            roofline = {'bound': 'issue', 'achieved': issued, 'peak': issue_peak, 'unit': 'Gwarp-inst/s',
                        'frac': issued / issue_peak, 'traffic': traffic,
                        'note': f'{inst_per_trial:.0f} warp instructions per trial (ncu, small case of the same '
                                f'search) x trials/s; peak = 4 warp instructions/clk/SM x {nsm} SMs x {mhz:.0f} MHz',
                        'sfu_equivalent': sfu}
        else:
            roofline = sfu
        line = {
            'metric': 'trial structures evaluated/s', 'value': value, 'unit': 'trials/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'fp64' if args.cos_mode == COS_FACTORED else 'fp32',
            'data': 'synthetic',
            'config': {'workload': f'wyckoff-search Pnma PbSO4-like (Pb 4c, S 4c, O 4c, O 4c, O 8d; 24 atoms/cell), '
                                   f'{n} replicas x {G} generations per GPU, d_min 1.2 A '
                                   f'({P.refl.n_refl} reflections, {P.refl.n_groups} groups)',
                       'replicas_per_gpu': n, 'generations': G, 'step': 'one full search, one launch',
                       'l2': 'flushed before every step (256 MB write)', 'cos': COS_NAMES[args.cos_mode],
                       'parallelism': f'replicas only x{world}'},
            'roofline': roofline,
            'e2e': {'value': e2e_value, 'unit': 'trials/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h},
            'gpu_launches': int(launches),
            'clocks': {k: clocks[k] for k in ('sm_mhz', 'sm_max_mhz', 'reasons')},
        }
        if not args.no_cpu_baseline and world == 1:
            line['cpu_baseline'] = cpu_baseline(P, groups, pen, n)
        if world == 1 and G == GENERATIONS:
            line['time_to_target_wr2'] = wyckoff_time_to_target(P, n, sess)
    if world == 1 and G == GENERATIONS and n == PARTICLES and not args.no_sub_workloads:
        # the PT fit (NaCl, 64 chains x 2000 sweeps) and the split-BF16 contraction (16384 x 3000 x 12000)
        # under the same clock, each with its own roofline, CPU baseline, end-to-end figure and clocks
        import copy
        sub = {}
        a = copy.copy(args)
        a.chains, a.sweeps, a.pt_method = 64, 2000, 'rietveld'
        sub['pt'] = main_pt(a, world, rank, local, emit=False)
        a = copy.copy(args)
        a.method = 'split'
        sub['contract'] = main_ct(a, world, rank, local, emit=False)
        a = copy.copy(args)
        sub['profile'] = main_profile(a, world, rank, local, emit=False)
        if rank == 0:
            line['workloads'] = sub
    if rank == 0:
        print(json.dumps(line), flush=True)
    sess.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
