"""Benchmark: cell-updates/s of the local-inertial step on B200.

    python bench.py --gpus N --steps K --warmup W [--form batched|plain|served]
                    [--workload NAME] [--impl reference]

The default is the batched form (the headline of the metric): 64 seeded
quadtree scenarios of uneven size (about 43.65M cells in all), every
scenario with its own CFL dt, advanced together. A "step" of this benchmark
is one ensemble batch: up to 32 device time steps of every scenario. The
line also carries the same scenarios stepped one after another with the
plain form (``plain_sequential``, ``batched_over_plain``) and the largest
depth difference between the two after the same batches.

``--form plain`` times one plain solve of ``--workload`` (a batch of up to
32 time steps per bench step); ``--form served`` replays a Poisson request
stream through the server against the plain form one request at a time.

``value`` is device time with the state resident in HBM (CUDA events on the
library's stream around each batch); ``e2e`` is the same metric through the
public call with the host forcing inputs and the host trace read-back inside
the timed region.

Each run first advances, untimed, a third into its simulated duration (rain
and flow have reached the domain by then) and takes the warm-up batches:
that state is where the timed batches and the CPU baseline start.
``--impl reference`` times the reference algorithm's CPU implementation (the
CPU restatement of the step, all host threads) on the same workload, from
the same state and with the same ``config``; the CUDA step produces that
state untimed (it equals the restatement's own state bit for bit).

Multi-GPU: a solve does not shard (one domain per device); N ranks run N
independent replicas ("replicas only", weak scaling), timed by device events
with the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / 'nh-flood-2d_b200'))

METRIC = 'cell-updates/s'
PEAKS = ROOT / 'MEASURED_PEAKS.json'
FALLBACK_HBM = 6650.0
L2_FLUSH_BYTES = 256 << 20  # twice the B200's 126 MB L2


def algorithmic_bytes(w):
    """Minimum unique bytes a fully fused step moves per cell-update: depth
    r/w 8 + bed 4 + q r/w of the ~2 sides a cell owns 16 + their Manning n 8
    + max_depth r/w 8 + max_speed r/w 8 = 52 B; a rain pixel index +4 B when
    it rains; Horton rain time and capacity r/w 16 + f0/fc/k 12 = +28 B when
    Horton classes exist; multi-resolution connectivity: 2 cell ids + a
    length per side (12 B x S/N) and a 4-slot face table (20 B)."""
    b = 52.0
    if np.any(w.forcing.rain.millimetres > 0):
        b += 4
    from nhflood.input import HortonInfiltration
    if any(isinstance(p.infiltration, HortonInfiltration) for p in w.land_parameters.values()):
        b += 28
    if getattr(w.mesh, 'level', None) is not None:
        b += 12.0 * (w.mesh.s_num - 1) / w.cells + 20
    if getattr(w, 'gate', None) is not None and w.gate.enabled:
        b += 8  # the gate controller's per-cell gate index and pond flag
    return b


# DRAM bytes (read + write) of one step launch (the fused tiled step, or the
# lattice march), from the ncu captures summarised in profiles/
# (k_step_tiled_<workload>.md, k_lattice_march_dambreak.md).
# Timed state (the bench's NVTX timed region); keyed by workload and step form.
TRAFFIC_PER_LAUNCH = {('multires_quadtree', 'tiled'): 148.976896e6 + 20.993792e6,
                      ('dambreak_4096', 'tiled'): 1022.048512e6 + 189.920512e6,
                      ('dambreak_4096', 'lattice'): 1025.505024e6 + 201.589504e6}


def launches_per_batch(run) -> int:
    """Kernels one batch graph of a plain run launches: begin (+ rain-time
    copy, state copy-back and velocity on the fused step), and per step the
    fused step (+ its CFL pass on split plans) or the six multi-pass kernels,
    the hanging-edge and theta pre-passes, and the gate controller's
    passes."""
    eng = run.engine
    if eng.path.startswith('lattice'):  # gather, begin, scatter, velocity; per step the step and its CFL pass
        return 4 + run.params.batch_size * 2
    tiled = eng.path.startswith('tiled')
    pre = (1 if run.arrays.hang_cells else 0) + (0 if run.w.sita == 1.0 else 1)
    gate = run.arrays.gate
    once = 0
    if gate is not None:
        if tiled:  # exchange volumes with the end motion; start motion in the CFL pass (own launch at batch start)
            pre += 1
            once += 1
        else:  # bed motion at the start and the end, exchange volumes
            pre += 2 + (1 if len(gate.flux_sides) else 0)
    per_step = ((2 if 'cfl=pass' in eng.path else 1) if tiled else 6) + pre
    return (4 if tiled else 1) + once + run.params.batch_size * per_step


def combine_ranks(times, units, device, world):
    """Whole-job figures over the replicas: the slowest rank's times (max)
    and the units of all ranks (sum). times, units: equal-length lists of
    this rank's seconds (or ms) and processed units; returns both lists
    reduced over the process group (unchanged when world == 1)."""
    if world <= 1:
        return list(times), list(units)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in times], dtype=torch.float64, device=device)
    u = torch.tensor([float(x) for x in units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return t.tolist(), u.tolist()


def plain_config(w, spin_to, world, batch_size=32):
    """The plain workload's ``config``, identical in both arms."""
    return {'workload': w.name, 'cells': w.cells, 'sides': w.mesh.s_num - 1,
            'time_steps_per_bench_step': batch_size, 'spin_up_to_s': spin_to,
            'start_state': 'advanced by the CUDA step to the spin-up time, then the warm-up batches',
            'l2': 'flushed (256 MB write) before every timed batch', 'parallelism': f'replicas{world}'}


def reference_plain(args):
    """The reference arm of the plain form: the CPU restatement (all host
    threads) on the same workload, from the state the b200 arm's timed
    batches start from (produced by the CUDA step, untimed; it equals the CPU
    restatement's own state bit for bit)."""
    import torch
    w = make_workload(args.workload)
    spin_to = w.duration / 3 if args.spin_up is None else args.spin_up
    start = None
    if torch.cuda.is_available():
        from nhflood.native import CudaEngine
        from nhflood.plain import PlainRun
        start = PlainRun(w, lambda a, p: CudaEngine(a, p, device='cuda:0'))
        while start.elapsed < spin_to and not start.done:
            start.advance()
        for _ in range(args.warmup):
            start.advance()
    base = cpu_baseline(w, seconds_budget=max(5.0, args.cpu_seconds), start=start)
    if start is not None:
        start.close()
    line = {'metric': METRIC, 'value': base['value'], 'unit': METRIC, 'impl': 'reference', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'form': 'plain',
            'config': plain_config(w, spin_to, args.gpus),
            'cpu_baseline': base,
            'e2e': {'value': base['value'], 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def make_workload(name):
    from nhflood import workloads
    if name == 'plain_uniform_256':
        return workloads.plain_uniform_256()
    if name.startswith('dambreak_'):
        return workloads.dambreak(n=int(name.split('_')[1]))
    if name == 'multires_quadtree':
        return workloads.multires_quadtree()
    if name == 'multires_quadtree_4m':
        return workloads.multires_quadtree_4m()
    if name.startswith('gated_polder_'):
        return workloads.gated_polder(n=int(name.split('_')[2]))
    raise SystemExit(f'unknown workload {name}')


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.thread = None

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.FIELDS}',
                                      '--format=csv,noheader,nounits'], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(',')])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.thread:
            self.thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unavailable']}
        sm = [float(s[1]) for s in self.samples if s[1].replace('.', '').isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for s in self.samples for i, v in enumerate(s[5:9]) if v.strip().lower() == 'active'})
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(self.samples)}


def peak_hbm():
    try:
        return float(json.loads(PEAKS.read_text())['hbm_gbs']), 'measured'
    except Exception:
        return FALLBACK_HBM, 'fallback'


def cpu_baseline(workload, seconds_budget=15.0, threads=None, start=None):
    """The CPU restatement on the same workload, all host threads, bounded
    sample; with start (a PlainRun) it continues from that run's state."""
    sys.path.insert(0, str(ROOT / 'oracle'))
    from engine import OracleEngine, set_threads  # oracle/engine.py
    from nhflood.plain import PlainRun
    threads = threads or os.cpu_count()
    set_threads(threads)
    run = PlainRun(workload, lambda a, p: OracleEngine(a, p), batch_size=1)
    if start is not None:
        run.adopt(start)
    origin = run.elapsed
    steps = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds_budget and not run.done:
        steps += run.advance()
    el = time.perf_counter() - t0
    run.close()
    return {'value': workload.cells * steps / el, 'unit': METRIC, 'cores': threads, 'kind': 'port',
            'sample': f'{steps} time steps of {workload.name} from t={origin:.0f} s ({el:.1f} s of CPU restatement, OpenMP)'}


ENSEMBLE_PLAIN_BATCHES = 3  # plain batches of every member, and as many e2e ensemble batches


def ensemble_workloads(args, rank):
    from nhflood.workloads import ensemble_scenarios
    return ensemble_scenarios(seed=4 + rank, members=args.members)


def ensemble_config(ws, spin_to, world, batch_size=32):
    """The batched workload's ``config``, identical in both arms."""
    cells = np.array([w.cells for w in ws], np.int64)
    return {'workload': f'ensemble_{len(ws)}_quadtrees', 'members': len(ws), 'cells': int(cells.sum()),
            'cells_min': int(cells.min()), 'cells_max': int(cells.max()),
            'time_steps_per_bench_step': batch_size, 'spin_up_to_s': spin_to,
            'start_state': 'every member advanced by the CUDA step to the spin-up time, then the warm-up batches',
            'l2': 'inputs larger than L2 (43.65M cells resident)', 'parallelism': f'replicas{world}'}


def spin_up(ens, spin_to, warmup):
    """Advance (untimed) until every member has reached ``spin_to`` seconds,
    then ``warmup`` more batches: the state both arms start from."""
    while min(r.elapsed for r in ens.runs) < spin_to and not ens.done:
        ens.advance()
    for _ in range(warmup):
        ens.advance()


def ensemble_cpu_sample(runs, seconds_budget, threads=None):
    """The CPU restatement on every member in turn, continuing from that
    member's current state, one time step per call; each member gets a share
    of the budget in proportion to its cells (at least one step). Only the
    step calls are timed."""
    sys.path.insert(0, str(ROOT / 'oracle'))
    from engine import OracleEngine, set_threads  # oracle/engine.py
    from nhflood.plain import PlainRun
    threads = threads or os.cpu_count()
    set_threads(threads)
    total_cells = sum(r.w.cells for r in runs)
    cell_updates, seconds, steps = 0, 0.0, 0
    for member in runs:
        run = PlainRun(member.w, lambda a, p: OracleEngine(a, p), batch_size=1)
        run.adopt(member)
        share = seconds_budget * member.w.cells / total_cells
        spent, n = 0.0, 0
        while (n == 0 or spent < share) and not run.done:
            t0 = time.perf_counter()
            k = run.advance()
            spent += time.perf_counter() - t0
            n += k
            if k == 0:
                break
        cell_updates += n * member.w.cells
        seconds += spent
        steps += n
        run.close()
    return {'value': cell_updates / seconds if seconds else None, 'unit': METRIC, 'cores': threads, 'kind': 'port',
            'sample': (f'{steps} time steps over the {len(runs)} members, each member continuing from its state '
                       f'at the timed start ({seconds:.1f} s of CPU restatement, OpenMP)')}


def plain_breakdown(per_member, edges=(2e5, 7e5)):
    """The plain form's members in three size buckets (cells below 200k,
    200k to 700k, above): members, cells, share of the plain form's time and
    cell-updates/s. The largest bucket's rate is about what the plain form
    reaches once a mesh fills the GPU, so total plain time over (total
    cell-updates / that rate) bounds what batching can gain."""
    rows = np.array(per_member, dtype=np.float64).reshape(-1, 3)
    total_s = rows[:, 2].sum()
    names = ('small', 'mid', 'large')
    bounds = (0,) + tuple(edges) + (np.inf,)
    out = {}
    for name, lo, hi in zip(names, bounds[:-1], bounds[1:]):
        sel = rows[(rows[:, 0] >= lo) & (rows[:, 0] < hi)]
        if not len(sel):
            continue
        out[name] = {'members': int(len(sel)), 'cells': int(sel[:, 0].sum()),
                     'plain_time_share': float(sel[:, 2].sum() / total_s) if total_s else None,
                     'plain_rate': float(sel[:, 1].sum() / sel[:, 2].sum()) if sel[:, 2].sum() else None}
    if out:
        large = out.get('large') or out[max(out, key=lambda k: out[k]['cells'])]
        if large['plain_rate'] and total_s:
            out['bound_if_every_member_ran_at_the_large_rate'] = float(
                total_s / (rows[:, 1].sum() / large['plain_rate']))
    return out


def bench_batched(args, rank, world, local):
    """Batched form: 64 seeded quadtree scenarios (about 40M cells) in one
    ensemble (by default every scenario's own batch graph, all launched
    together; --tile / --grid select the one-launch schedule), against the
    same scenarios stepped one after another with the plain form from the
    same state; the max depth difference of the two is measured."""
    import torch
    from nhflood.ensemble import EnsembleRun
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    ws = ensemble_workloads(args, rank)
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    ens = EnsembleRun(ws, device=str(device), tile=args.tile, grid_blocks=args.grid, tune=not args.no_tune)
    t_setup = time.perf_counter() - t0
    stream = ens.ensemble.stream()
    spin_to = min(r.w.duration for r in ens.runs) / 3 if args.spin_up is None else args.spin_up
    t0 = time.perf_counter()
    spin_up(ens, spin_to, args.warmup)
    t_spin = time.perf_counter() - t0
    torch.cuda.synchronize(device)
    cpu = None
    if rank == 0 and world == 1 and os.environ.get('NHF_BENCH_NO_CPU') != '1':
        cpu = ensemble_cpu_sample(ens.runs, args.cpu_seconds)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    cell_updates = 0
    recorded = 0
    hang = sum(1 for r in ens.runs if r.arrays.hang_cells)
    if ens.schedule == 'member graphs':  # every member's own batch graph
        per_batch_kernels = sum(launches_per_batch(r) for r in ens.runs)
    else:  # per step: the ensemble step, its CFL pass, the hanging pre-pass if any member has hanging edges
        per_batch_kernels = 5 + ens.runs[0].params.batch_size * (2 + (1 if hang else 0))
    with ClockSampler(local) as clocks:
        torch.cuda.nvtx.range_push('timed')  # ncu --nvtx --nvtx-include timed/ captures the timed state
        for k in range(args.steps):
            if ens.done:
                break
            targets, origins = ens.begin()
            starts[k].record(stream)
            ens.ensemble.run_batch_async(targets, origins)
            ends[k].record(stream)
            cell_updates += ens.cell_updates(ens.finish(ens.ensemble.read_trace()))
            recorded += 1
        torch.cuda.synchronize(device)
        torch.cuda.nvtx.range_pop()
    device_s = sum(starts[i].elapsed_time(ends[i]) for i in range(recorded)) / 1e3
    # the same scenarios, one after another, each on a plain engine of its own
    # (the plain form's own tile and CFL choice) continuing from the member's state
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    plain_cells, plain_s = 0, 0.0
    plain_depth = []
    per_member = []  # (cells, cell-updates, seconds) of each member's plain batches
    for member in ens.runs:
        m_cells, m_s = plain_cells, plain_s
        r = PlainRun(member.w, lambda a, p: CudaEngine(a, p, device=str(device)), batch_size=member.params.batch_size)
        r.adopt(member)
        st = r.engine.stream()
        for _ in range(ENSEMBLE_PLAIN_BATCHES):
            if r.done:
                break
            tw, ow = r.begin()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            r.engine.run_batch_async(tw, ow)
            b.record(st)
            plain_cells += r.finish(r.engine.read_trace()) * r.w.cells
            b.synchronize()
            plain_s += a.elapsed_time(b) / 1e3
        plain_depth.append((r.elapsed, r.engine.get('depth')))
        per_member.append((r.w.cells, plain_cells - m_cells, plain_s - m_s))
        r.close()
    # end to end through the public call (host words in, host traces out),
    # the same batches the plain engines just ran
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    e2e_cells = 0
    h2d = 0
    for _ in range(ENSEMBLE_PLAIN_BATCHES):
        if ens.done:
            break
        e2e_cells += ens.cell_updates(ens.advance())
        h2d += ens.h2d_bytes
    torch.cuda.synchronize(device)
    e2e_s = time.perf_counter() - t0
    # batched against plain: the members' depths after the same batches
    max_err, compared = 0.0, 0
    for member, (elapsed, depth) in zip(ens.runs, plain_depth):
        if member.elapsed == elapsed:
            max_err = max(max_err, float(np.abs(member.engine.get('depth').astype(np.float64) - depth).max()))
            compared += 1
    (device_s, e2e_s), (cell_updates, e2e_cells) = combine_ranks([device_s, e2e_s], [cell_updates, e2e_cells],
                                                                 device, world)
    value = cell_updates / device_s
    plain = plain_cells / plain_s if plain_s else None
    if rank == 0:
        peak, kind = peak_hbm()
        cells = np.array([w.cells for w in ws], float)
        b_alg = float((cells * np.array([algorithmic_bytes(w) for w in ws])).sum() / cells.sum())
        achieved = value / world * b_alg / 1e9
        trace_bytes = ens.ensemble._trace.nbytes
        line = {
            'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': recorded,
            'warmup': args.warmup, 'ms_per_step': device_s * 1e3 / max(1, recorded), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'form': 'batched',
            'config': ensemble_config(ws, spin_to, world),
            'schedule': {'kind': ens.schedule, 'tile': ens.ensemble.tile or 'per member',
                         'grid_blocks': ens.ensemble.grid, 'tiles': ens.ensemble.tiles,
                         'autotuner_trials_tile_grid_rate': ens.tuned.trials if ens.tuned else None},
            'plain_sequential': {'value': plain, 'unit': METRIC,
                                 'sample': f'{ENSEMBLE_PLAIN_BATCHES} plain batches of each member from its state '
                                           'after the timed batches, one member after another'},
            'batched_over_plain': value / plain if plain else None,
            'plain_by_size': plain_breakdown(per_member),
            'max_depth_error_vs_plain_m': max_err,
            'members_compared_with_plain': compared,
            'gpu_launches': per_batch_kernels * recorded,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                         'traffic': None, 'peak_kind': kind, 'algorithmic_bytes_per_cell_update': b_alg,
                         'scope': 'whole batch of every member (step kernels, CFL passes, pre-passes)'},
            'e2e': {'value': e2e_cells / e2e_s if e2e_s else None, 'unit': METRIC,
                    'h2d_bytes_per_step': h2d // max(1, ENSEMBLE_PLAIN_BATCHES), 'd2h_bytes_per_step': trace_bytes},
            'clocks': clocks.summary(),
            'setup_seconds': {'generate': round(t_gen, 1), 'tuning_and_engines': round(t_setup, 1),
                              'spin_up': round(t_spin, 1)},
        }
        if cpu is not None:
            line['cpu_baseline'] = cpu
        print(json.dumps(line))
    ens.close()


def reference_batched(args):
    """The reference arm of the batched form: the CPU restatement of the step
    (all host threads) on the same 64 members, from the same start state and
    with the same ``config`` as the b200 arm. The start state is produced by
    the CUDA step, untimed: it equals the CPU restatement's own state bit for
    bit (the parity tests), and the CPU would need about half an hour to
    reach it. Only the CPU restatement's step calls are timed."""
    import torch
    from nhflood.ensemble import EnsembleRun
    ws = ensemble_workloads(args, 0)
    spin_to = min(w.duration for w in ws) / 3 if args.spin_up is None else args.spin_up
    cells = sum(w.cells for w in ws)
    if not torch.cuda.is_available():
        base = {'value': None, 'unit': METRIC, 'cores': os.cpu_count(), 'kind': 'port',
                'sample': 'not run: the start state needs the CUDA step'}
    else:
        ens = EnsembleRun(ws, device='cuda:0')
        spin_up(ens, spin_to, args.warmup)
        torch.cuda.synchronize()
        base = ensemble_cpu_sample(ens.runs, max(5.0, args.cpu_seconds))
        ens.close()
    line = {'metric': METRIC, 'value': base['value'], 'unit': METRIC, 'impl': 'reference', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'form': 'batched',
            'config': ensemble_config(ws, spin_to, args.gpus),
            'cpu_baseline': base,
            'e2e': {'value': base['value'], 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def _request_workload(params):
    from nhflood.workloads import multires_quadtree
    return multires_quadtree(**params)


def bench_served(args, rank, world, local):
    """Served form: a Poisson stream of flood-solve requests of uneven mesh
    size, admitted under an HBM budget and stepped together (continuous
    batching), replayed in real time; then the same stream through the plain
    form one request at a time."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    import torch
    from nhflood.serving import FloodServer, MadeAhead, Request, latency_summary, serve, serve_sequential
    from nhflood.workloads import served_requests
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    stream = served_requests(seed=5 + rank, count=args.requests)
    # the meshes are made by a process pool a window ahead of the arrivals
    # (the stream's meshes together would not fit host memory); a request's
    # mesh stands for its input files, so making it is not part of its latency
    pool = ProcessPoolExecutor(min(16, os.cpu_count() or 1), mp_context=mp.get_context('spawn'))
    t0 = time.perf_counter()
    source = MadeAhead(_request_workload, stream, pool, ahead=48)
    source.wait_first()
    t_gen = time.perf_counter() - t0
    reqs = source.requests()
    # warm-up: one small request through both paths (module loads, first graph)
    warm_workload = _request_workload(dict(stream[0]['params'], width=1000.0, duration=60))
    warm = [Request(-1, 0.0, warm_workload)]
    server = FloodServer(hbm_budget=args.hbm_budget, tile=args.tile or 256, device=str(device))
    serve(warm, server, realtime=False)
    serve_sequential([Request(-1, 0.0, warm_workload)], tile=args.tile or 256, device=str(device), realtime=False)
    server = FloodServer(hbm_budget=args.hbm_budget, tile=args.tile or 256, device=str(device))
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        served = serve(reqs, server, realtime=True)
        served_wall = time.perf_counter() - t0
    server.close()
    source = MadeAhead(_request_workload, stream, pool, ahead=48)
    source.wait_first()
    again = source.requests()
    t0 = time.perf_counter()
    sequential = serve_sequential(again, tile=args.tile or 256, device=str(device), realtime=True)
    seq_wall = time.perf_counter() - t0
    pool.shutdown()
    by_id = {c.id: c for c in sequential}
    max_err = 0.0
    for c in served:
        o = by_id[c.id]
        max_err = max(max_err, float(np.abs(c.depth - o.depth).max()), float(np.abs(c.max_depth - o.max_depth).max()))
    cell_updates = sum(c.cell_updates for c in served)
    value = cell_updates / served_wall
    seq_value = sum(c.cell_updates for c in sequential) / seq_wall
    if rank == 0:
        cells = np.array([r.cells for r in reqs])
        line = {
            'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': server.rounds,
            'warmup': 1, 'ms_per_step': served_wall * 1e3 / max(1, server.rounds), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'form': 'served',
            'config': {'workload': f'served_{len(reqs)}_requests', 'arrival_rate_per_s': 2.0,
                       'cells_total': int(cells.sum()), 'cells_min': int(cells.min()), 'cells_max': int(cells.max()),
                       'hbm_budget_bytes': args.hbm_budget, 'tile': args.tile or 256, 'parallelism': f'replicas{world}',
                       'l2': 'inputs larger than L2 once several solves are resident'},
            'timing': 'wall clock of the whole session, arrivals replayed in real time',
            'latency': latency_summary(served),
            'plain_sequential': {'value': seq_value, 'unit': METRIC, 'latency': latency_summary(sequential),
                                 'wall_s': seq_wall},
            'served_over_plain': value / seq_value,
            'max_depth_error_vs_plain_m': max_err,
            'peak_resident_bytes_estimate': server.peak_used,
            'session_wall_s': served_wall,
            'gpu_launches': None,
            'e2e': {'value': value, 'unit': METRIC, 'h2d_bytes_per_step': None, 'd2h_bytes_per_step': None},
            'clocks': clocks.summary(),
            'setup_seconds': {'generate': round(t_gen, 1)},
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--workload', default=os.environ.get('NHF_BENCH_WORKLOAD', 'multires_quadtree'))
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--cpu-seconds', type=float, default=15.0)
    ap.add_argument('--form', default=os.environ.get('NHF_BENCH_FORM', 'batched'),
                    choices=['plain', 'batched', 'served'])
    ap.add_argument('--requests', type=int, default=512, help='served: requests in the stream (config 5: 512)')
    ap.add_argument('--hbm-budget', type=float, default=150e9, help='served: admission budget in bytes')
    ap.add_argument('--members', type=int, default=64)
    ap.add_argument('--tile', type=int, default=None, help='batched: one-launch tile size (default: autotuned)')
    ap.add_argument('--grid', type=int, default=None,
                    help='batched: 0 persistent, -1 block per tile, -2 member graphs (default: autotuned)')
    ap.add_argument('--no-tune', action='store_true', help='batched: member graphs without the autotuner')
    ap.add_argument('--path', default='auto', help="plain form's step: 'auto', 'multipass', 'tile256', 'tile512', 'tile1024'")
    ap.add_argument('--spin-up', type=float, default=None,
                    help='simulated seconds advanced (untimed) before the warm-up; default a third of the run')
    args = ap.parse_args()

    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))

    if args.impl == 'reference':
        if rank != 0:
            return
        if args.form == 'batched':
            reference_batched(args)
        elif args.form == 'plain':
            reference_plain(args)
        else:
            print(json.dumps({'impl': 'reference', 'form': args.form,
                              'unavailable': 'the served form has no CPU counterpart; time the batched or plain form'}))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
        torch.cuda.set_device(local)
    if args.form in ('batched', 'served'):
        (bench_batched if args.form == 'batched' else bench_served)(args, rank, world, local)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun

    w = make_workload(args.workload)
    def factory(a, p):
        p.path = args.path
        return CudaEngine(a, p, device=str(device))
    run = PlainRun(w, factory)
    eng = run.engine
    stream = eng.stream()
    # spin-up (untimed): the timed batches start a third into the run, where
    # rain and flow have reached the domain, not on the initial dry state
    spin_to = w.duration / 3 if args.spin_up is None else args.spin_up
    while run.elapsed < spin_to and not run.done:
        run.advance()
    spin_up_s = run.elapsed
    # warm-up batches (untimed)
    for _ in range(args.warmup):
        run.advance()
    torch.cuda.synchronize(device)
    # the CPU restatement on a bounded sample from the same state the timed batches start from
    cpu = None
    if rank == 0 and world == 1 and os.environ.get('NHF_BENCH_NO_CPU') != '1':
        cpu = cpu_baseline(w, seconds_budget=args.cpu_seconds, start=run)
    if world > 1:
        dist.barrier()
    # device-resident timing: events around each graph replay on the library stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    cell_steps = 0
    launches = 0
    tiled = eng.path.startswith('tiled')
    per_batch_launches = launches_per_batch(run)
    recorded = 0
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=device)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize(device)
        torch.cuda.nvtx.range_push('timed')  # ncu --nvtx --nvtx-include timed/ captures the timed state
        for k in range(args.steps):
            if run.done:
                break
            recorded += 1
            tw, ow = run.begin()
            with torch.cuda.stream(stream):
                flush.fill_(k)  # evict the state from L2 between timed batches
            starts[k].record(stream)
            eng.run_batch_async(tw, ow)
            ends[k].record(stream)
            n = run.finish(eng.read_trace())
            cell_steps += n * w.cells
            launches += per_batch_launches
        torch.cuda.synchronize(device)
        torch.cuda.nvtx.range_pop()
    timed = [starts[i].elapsed_time(ends[i]) for i in range(recorded)]
    device_ms = float(sum(timed))
    # end-to-end through the public call: host inputs in, host trace out
    e2e_cells = 0
    e2e_batches = max(3, min(args.steps, 20))
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(e2e_batches):
        if run.done:
            break
        tw, ow = run.begin()
        rows = eng.run_batch(tw, ow)
        h2d += run.h2d_bytes
        d2h += rows.nbytes
        e2e_cells += run.finish(rows) * w.cells
    torch.cuda.synchronize(device)
    e2e_s = time.perf_counter() - t0
    (device_ms, e2e_s), (cell_steps, e2e_cells) = combine_ranks([device_ms, e2e_s], [cell_steps, e2e_cells],
                                                                device, world)
    value = cell_steps / (device_ms / 1e3) if device_ms > 0 else 0.0
    e2e = e2e_cells / e2e_s if e2e_s > 0 else 0.0
    if rank == 0:
        peak, kind = peak_hbm()
        b_alg = algorithmic_bytes(w)
        per_rank = value / world
        achieved = per_rank * b_alg / 1e9 if b_alg else None
        line = {
            'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': device_ms / max(1, len(timed)), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': plain_config(w, spin_to, world, run.params.batch_size),
            'step_form': eng.path, 'spun_up_to_s': spin_up_s,
            'gpu_launches': launches,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak if achieved else None,
                         'traffic': TRAFFIC_PER_LAUNCH.get((w.name, eng.path.split('(')[0])),
                         'traffic_unit': 'bytes per step launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)',
                         'algorithmic_bytes_per_launch': b_alg * w.cells,
                         'peak_kind': kind, 'algorithmic_bytes_per_cell_update': b_alg,
                         'scope': ('whole batch graph (' + ('lattice march and close pass, gather and scatter'
                                   if eng.path.startswith('lattice') else 'fused step kernel, its CFL pass'
                                   if 'cfl=pass' in eng.path else 'fused step kernel' if tiled
                                   else 'multi-pass kernels') + ', per-batch epilogue)')},
            'e2e': {'value': e2e, 'unit': METRIC, 'h2d_bytes_per_step': h2d // max(1, e2e_batches),
                    'd2h_bytes_per_step': d2h // max(1, e2e_batches)},
            'clocks': clocks.summary(),
            'simulated_seconds': run.elapsed,
        }
        if cpu is not None:
            line['cpu_baseline'] = cpu
        print(json.dumps(line))
    run.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
