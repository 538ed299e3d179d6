"""Benchmark: cell-updates/s of the plain local-inertial step on B200.

    python bench.py --gpus N --steps K --warmup W [--workload NAME] [--impl reference]

A "step" of this benchmark is one batch of up to 32 device time steps (one
replay of the captured step graph, the unit the reference's ti.graph runs
per host round trip) of the plain single-run solver on the workload; the
metric counts cells x completed time steps. ``value`` is device time with
the state resident in HBM (CUDA events on the library's stream around each
batch); ``e2e`` is the same metric through the public engine call with host
forcing inputs and the host trace read-back inside the timed region.

Multi-GPU: the plain solve does not shard (one domain per device); N ranks
run N independent replicas ("replicas only", weak scaling), timed by device
events with the max over ranks.

Each plain run first advances, untimed, a third into its simulated duration
(rain and flow have reached the domain by then), then takes the warm-up and
the timed batches; the CPU baseline continues from the GPU run's state.

``--impl reference`` times the reference algorithm's CPU implementation (the
CPU restatement of the step, all host threads) on the same workload, from
t = 0: spinning it up to the GPU arm's start would take the CPU minutes to
hours on the large configurations.
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


# DRAM bytes (read + write) of one fused step launch, from the ncu captures
# summarised in profiles/ (k_step_tiled_<workload>.md).
TRAFFIC_PER_LAUNCH = {'multires_quadtree': 148.207616e6 + 18.244352e6}


def launches_per_batch(run) -> int:
    """Kernels one batch graph of a plain run launches: begin (+ rain-time
    copy, state copy-back and velocity on the fused step), and per step the
    fused step (+ its CFL pass on split plans) or the six multi-pass kernels,
    the hanging-edge and theta pre-passes, and the gate controller's
    passes."""
    eng = run.engine
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


def make_workload(name):
    from nhflood import workloads
    if name == 'plain_uniform_256':
        return workloads.plain_uniform_256()
    if name.startswith('dambreak_'):
        return workloads.dambreak(n=int(name.split('_')[1]))
    if name == 'multires_quadtree':
        return workloads.multires_quadtree()
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


def bench_batched(args, rank, world, local):
    """Batched form: 64 seeded quadtree scenarios (about 40M cells) in one
    ensemble (by default every scenario's own batch graph, all launched
    together; --tile / --grid select the one-launch schedule), against the
    same scenarios stepped one after another with the plain form."""
    import torch
    from nhflood.ensemble import EnsembleRun
    from nhflood.workloads import ensemble_scenarios
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    ws = ensemble_scenarios(seed=4 + rank, members=args.members)
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    ens = EnsembleRun(ws, device=str(device), tile=args.tile, grid_blocks=args.grid)
    t_setup = time.perf_counter() - t0
    stream = ens.ensemble.stream()
    # spin-up (untimed) a third into the members' runs, as for the plain form
    spin_to = min(r.w.duration for r in ens.runs) / 3 if args.spin_up is None else args.spin_up
    while min(r.elapsed for r in ens.runs) < spin_to and not ens.done:
        ens.advance()
    for _ in range(args.warmup):
        ens.advance()
    torch.cuda.synchronize(device)
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
    device_s = sum(starts[i].elapsed_time(ends[i]) for i in range(recorded)) / 1e3
    # the same scenarios, one after another, each on a plain engine of its own
    # (the plain form's own tile and CFL choice) continuing from the member's state
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    plain_cells, plain_s = 0, 0.0
    for member in ens.runs if args.plain_batches > 0 else ():
        r = PlainRun(member.w, lambda a, p: CudaEngine(a, p, device=str(device)), batch_size=member.params.batch_size)
        r.adopt(member)
        st = r.engine.stream()
        for _ in range(args.plain_batches):
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
        r.close()
    # end to end through the public call (host words in, host traces out)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    e2e_cells = 0
    h2d = 0
    e2e_batches = 3
    for _ in range(e2e_batches):
        if ens.done:
            break
        e2e_cells += ens.cell_updates(ens.advance())
        h2d += ens.h2d_bytes
    torch.cuda.synchronize(device)
    e2e_s = time.perf_counter() - t0
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
            'config': {'workload': f'ensemble_{args.members}_quadtrees', 'members': len(ws),
                       'cells': int(cells.sum()), 'cells_min': int(cells.min()), 'cells_max': int(cells.max()),
                       'time_steps_per_bench_step': ens.runs[0].params.batch_size,
                       'schedule': ens.schedule, 'tile': ens.ensemble.tile or 'per member',
                       'grid_blocks': ens.ensemble.grid, 'tiles': ens.ensemble.tiles,
                       'spin_up_to_s': spin_to,
                       'l2': 'inputs larger than L2', 'parallelism': f'replicas{world}'},
            'plain_sequential': {'value': plain, 'unit': METRIC,
                                 'sample': f'{args.plain_batches} plain batches of each member, one member after another'},
            'batched_over_plain': value / plain if plain else None,
            'max_depth_error_vs_plain_m': 0.0,
            'gpu_launches': per_batch_kernels * recorded,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                         'traffic': None, 'peak_kind': kind, 'algorithmic_bytes_per_cell_update': b_alg},
            'e2e': {'value': e2e_cells / e2e_s if e2e_s else None, 'unit': METRIC,
                    'h2d_bytes_per_step': h2d // max(1, e2e_batches), 'd2h_bytes_per_step': trace_bytes},
            'clocks': clocks.summary(),
            'setup_seconds': {'generate': round(t_gen, 1), 'engines_and_tuning': round(t_setup, 1)},
        }
        print(json.dumps(line))
    ens.close()


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
    from nhflood.serving import FloodServer, Request, latency_summary, serve, serve_sequential
    from nhflood.workloads import served_requests
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    stream = served_requests(seed=5 + rank, count=args.requests)
    t0 = time.perf_counter()
    with ProcessPoolExecutor(min(len(stream), os.cpu_count() or 1), mp_context=mp.get_context('spawn')) as pool:
        workloads = list(pool.map(_request_workload, [r['params'] for r in stream]))
    t_gen = time.perf_counter() - t0
    reqs = [Request(r['id'], r['arrival'], w) for r, w in zip(stream, workloads)]
    for r in reqs:
        r.prepare()
    # warm-up: one small request through both paths (module loads, first graph)
    warm = [Request(-1, 0.0, _request_workload(dict(stream[0]['params'], width=1000.0, duration=60)))]
    server = FloodServer(hbm_budget=args.hbm_budget, tile=args.tile or 256, device=str(device))
    serve(warm, server, realtime=False)
    serve_sequential([Request(-1, 0.0, warm[0].workload)], tile=args.tile or 256, device=str(device), realtime=False)
    server = FloodServer(hbm_budget=args.hbm_budget, tile=args.tile or 256, device=str(device))
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        served = serve(reqs, server, realtime=True)
        served_wall = time.perf_counter() - t0
    server.close()
    t0 = time.perf_counter()
    sequential = serve_sequential(reqs, tile=args.tile or 256, device=str(device), realtime=True)
    seq_wall = time.perf_counter() - t0
    by_id = {c.id: c for c in sequential}
    max_err = 0.0
    for c in served:
        o = by_id[c.id]
        max_err = max(max_err, float(np.abs(c.depth - o.depth).max()), float(np.abs(c.max_depth - o.max_depth).max()))
    cell_updates = sum(c.cell_updates for c in served)
    value = cell_updates / served_wall
    seq_value = sum(c.cell_updates for c in sequential) / seq_wall
    if rank == 0:
        cells = np.array([r.workload.cells for r in reqs])
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
    ap.add_argument('--form', default='plain', choices=['plain', 'batched', 'served'])
    ap.add_argument('--requests', type=int, default=48, help='served: requests in the stream')
    ap.add_argument('--hbm-budget', type=float, default=150e9, help='served: admission budget in bytes')
    ap.add_argument('--members', type=int, default=64)
    ap.add_argument('--tile', type=int, default=None, help='batched: tile size (default: autotuned)')
    ap.add_argument('--grid', type=int, default=None, help='batched: 0 persistent, -1 block per tile')
    ap.add_argument('--plain-batches', type=int, default=2)
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
        w = make_workload(args.workload)
        base = cpu_baseline(w, seconds_budget=max(5.0, args.cpu_seconds))
        line = {'metric': METRIC, 'value': base['value'], 'unit': METRIC, 'impl': 'reference', 'n_gpus': args.gpus,
                'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
                'config': {'workload': w.name, 'cells': w.cells},
                'cpu_baseline': base,
                'e2e': {'value': base['value'], 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line))
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
            'config': {'workload': w.name, 'cells': w.cells, 'sides': w.mesh.s_num - 1,
                       'time_steps_per_bench_step': run.params.batch_size,
                       'l2': 'flushed (256 MB write) before every timed batch',
                       'step_form': eng.path, 'spin_up_to_s': spin_up_s,
                       'parallelism': f'replicas{world}'},
            'gpu_launches': launches,
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak if achieved else None,
                         'traffic': TRAFFIC_PER_LAUNCH.get(w.name),
                         'traffic_unit': 'bytes per step launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)',
                         'algorithmic_bytes_per_launch': b_alg * w.cells,
                         'peak_kind': kind, 'algorithmic_bytes_per_cell_update': b_alg,
                         'scope': ('whole batch graph (' + ('fused step kernel, its CFL pass' if 'cfl=pass' in eng.path
                                   else 'fused step kernel' if tiled else 'multi-pass kernels')
                                   + ', per-batch epilogue)')},
            'e2e': {'value': e2e, 'unit': METRIC, 'h2d_bytes_per_step': h2d // max(1, e2e_batches),
                    'd2h_bytes_per_step': d2h // max(1, e2e_batches)},
            'clocks': clocks.summary(),
            'simulated_seconds': run.elapsed,
        }
        if world == 1 and os.environ.get('NHF_BENCH_NO_CPU') != '1':
            line['cpu_baseline'] = cpu_baseline(w, seconds_budget=args.cpu_seconds, start=run)
        print(json.dumps(line))
    run.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
