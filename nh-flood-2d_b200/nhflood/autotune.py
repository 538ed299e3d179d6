"""Autotuner of the batched form's schedule.

Candidates: the member-graph schedule (every member's own batch graph with
the plain form's own step choice, all launched together on their own
streams) and the one-launch schedule (one fused step launch per slot for all
members) at tile sizes 256 and 1024 cells, each with two grid schedules:
persistent (resident blocks per SM x SMs, each block walking the tile list)
and one block per tile. Each candidate runs fresh engines of the same
scenarios from t = 0 (one warm-up batch, then timed batches with CUDA
events on the launching stream); the fastest cell-updates/s wins. Results
are cached in a JSON file keyed by the device name and a signature of the
meshes, so a given ensemble is tuned once per device.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np

TILES = (256, 1024)
GRIDS = (0, -1)  # 0: persistent grid, -1: one block per tile
MEMBER_GRAPHS = -2  # the member-graph schedule (tile 0)


@dataclass
class Schedule:
    tile: int
    grid: int
    rate: float = 0.0          # cell-updates/s measured for the winner
    trials: list | None = None  # [(tile, grid, rate or None)]


def default_cache() -> Path:
    env = os.environ.get('NHF_AUTOTUNE_CACHE')
    if env:
        return Path(env)
    return Path.home() / '.cache' / 'nhflood' / 'autotune.json'


def signature(workloads, batch_size: int, device_name: str) -> str:
    h = hashlib.sha256()
    h.update(device_name.encode())
    h.update(str(batch_size).encode())
    for w in workloads:
        level = getattr(w.mesh, 'level', None)
        h.update(np.array([w.cells, w.mesh.s_num, 0 if level is None else int(level.max()) + 1,
                           int(w.sita == 1.0)], np.int64).tobytes())
    return h.hexdigest()[:24]


def load(cache: Path) -> dict:
    try:
        return json.loads(Path(cache).read_text())
    except (OSError, ValueError):
        return {}


def store(cache: Path, key: str, schedule: Schedule) -> None:
    cache = Path(cache)
    data = load(cache)
    data[key] = asdict(schedule)
    cache.parent.mkdir(parents=True, exist_ok=True)
    tmp = cache.with_suffix(f'.{os.getpid()}.tmp')
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(tmp, cache)


def measure(workloads, tile: int, grids, batch_size: int, device: str, batches: int = 2) -> dict:
    """cell-updates/s of each grid schedule for one tile size (None when the
    tile size does not fit a member)."""
    import torch
    from .ensemble import EnsembleRun
    from .native import CudaEnsemble
    try:
        run = EnsembleRun(workloads, tile=tile, grid_blocks=grids[0], batch_size=batch_size, device=device)
    except RuntimeError:
        return {g: None for g in grids}
    out = {}
    ensembles = {grids[0]: run.ensemble}
    try:
        for g in grids[1:]:
            ensembles[g] = CudaEnsemble([r.engine for r in run.runs], g)
        run.advance()  # warm-up (also builds the first graph)
        for g in grids[1:]:
            run.ensemble = ensembles[g]
            run.advance()
        times = {g: 0.0 for g in grids}
        cells = {g: 0 for g in grids}
        for _ in range(batches):
            for g in grids:
                if run.done:
                    break
                ens = ensembles[g]
                run.ensemble = ens
                targets, origins = run.begin()
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                stream = ens.stream()
                start.record(stream)
                ens.run_batch_async(targets, origins)
                end.record(stream)
                completed = run.finish(ens.read_trace())
                end.synchronize()
                times[g] += start.elapsed_time(end) / 1e3
                cells[g] += run.cell_updates(completed)
        for g in grids:
            out[g] = cells[g] / times[g] if times[g] > 0 else None
    finally:
        for ens in ensembles.values():
            ens.close()
        run.close()
    return out


def measure_member_graphs(workloads, batch_size: int, device: str, batches: int = 2):
    """cell-updates/s of the member-graph schedule."""
    import torch
    from .ensemble import EnsembleRun
    run = EnsembleRun(workloads, grid_blocks=MEMBER_GRAPHS, batch_size=batch_size, device=device)
    try:
        run.advance()  # warm-up (builds every member's graph)
        seconds, cells = 0.0, 0
        stream = run.ensemble.stream()
        for _ in range(batches):
            if run.done:
                break
            targets, origins = run.begin()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            run.ensemble.run_batch_async(targets, origins)
            end.record(stream)
            completed = run.finish(run.ensemble.read_trace())
            end.synchronize()
            seconds += start.elapsed_time(end) / 1e3
            cells += run.cell_updates(completed)
        return cells / seconds if seconds > 0 else None
    finally:
        run.close()


def choose_schedule(workloads, *, batch_size: int = 32, device: str = 'cuda:0', cache=None,
                    tiles=TILES, grids=GRIDS, retune: bool = False, device_name: str | None = None,
                    measure_fn=None, member_graphs_fn=None) -> Schedule:
    """The fastest schedule: tile 0 and grid -2 stand for the member graphs."""
    cache = default_cache() if cache is None else Path(cache)
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(torch.device(device))
    key = signature(workloads, batch_size, device_name)
    if not retune:
        hit = load(cache).get(key)
        if hit:
            return Schedule(**hit)
    measure_fn = measure_fn or measure
    trials = []
    rate = (member_graphs_fn or measure_member_graphs)(workloads, batch_size, device)
    trials.append((0, MEMBER_GRAPHS, rate))
    for tile in tiles:
        rates = measure_fn(workloads, tile, list(grids), batch_size, device)
        trials.extend((tile, g, r) for g, r in rates.items())
    usable = [t for t in trials if t[2]]
    if not usable:
        raise RuntimeError('no schedule ran the ensemble')
    tile, grid, rate = max(usable, key=lambda t: t[2])
    schedule = Schedule(tile=tile, grid=grid, rate=rate, trials=[list(t) for t in trials])
    store(cache, key, schedule)
    return schedule
