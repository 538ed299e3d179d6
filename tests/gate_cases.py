"""Gate-controller cases rebuilt from the reference's gate tests
(tests/test_gate_solver.py:22-75 setup/run, :134-142 level boundary,
:253-262 event steps): square cells of given land classes, a seed checkpoint
with the initial depth and bed, a one-pixel rain raster and a gate block
whose default is one gate on cell 2 controlled by cell 1."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from nhflood.input import ForceConfig
from nhflood.output import write_checkpoint
from nhflood.raster import from_origin
from nhflood.run_record import sha256
from runner import run as run_case
from scenarios import domain, rectangles_mesh, write_line, write_rain, write_series

THREE = [(i * 10, (i + 1) * 10, 0, 10) for i in range(3)]


def centre(cell):
    x0, x1, y0, y1 = cell
    return ((x0 + x1) / 2, (y0 + y1) / 2)


def level_boundary(path: Path, rows, line=((0, 0), (0, 10)), name='river', kind='level'):
    path.mkdir(parents=True, exist_ok=True)
    return [dict(name=name, kind=kind, line=write_line(path / f'{name}.geojson', line),
                 series=write_series(path / f'{name}.csv', rows))]


def setup(path: Path, *, cells=None, types=None, bed=None, depth=None, gate=None, rain=0., warmup=0,
          yield_step=1, boundaries=None, land=None, rain_intervals=None):
    """Returns (domain config, force config, side topology, depth, bed); the
    depth and bed arrays carry the sentinel cell 0."""
    path.mkdir(parents=True, exist_ok=True)
    cells = cells or THREE
    types = types or [1, 11, 10]
    bed = np.r_[0, bed if bed is not None else [0] * len(cells)].astype(np.float32)
    depth = np.r_[0, depth if depth is not None else [2] * len(cells)].astype(np.float32)
    topo, _ = rectangles_mesh(path, cells, bed, types)
    config = dict(land_type=11, pond_land_type=10, enabled=True, trigger_level=1, opening_seconds=1,
                  open_elevation=-.1, gates=[dict(name='A', inside_point=centre(cells[1]),
                                                  control_point=centre(cells[0]))])
    if gate is not None:
        config.update(gate)
    x1, y1 = max(c[1] for c in cells), max(c[3] for c in cells)
    intervals = rain_intervals or [(0, 3600)]
    bands = np.full((len(intervals), 1, 1), rain, dtype=np.float32)
    rain_cfg = write_rain(path, bands, from_origin(0, y1, x1, y1), intervals)
    force = ForceConfig(boundaries=boundaries or [], gate=config, rainfall=rain_cfg)
    zeros, words = np.zeros(len(depth), np.float32), np.zeros(len(depth), np.uint32)
    seed = path / 'seed.fdb'
    write_checkpoint(seed, depth=depth, bed=bed, q=np.zeros(len(topo), np.float32), rain_time=zeros,
                     infiltration=zeros, max_depth=depth, max_speed=zeros, first_time_hi=words,
                     first_time_lo=words, clock_hi=0, clock_lo=0, gate_open=False,
                     metadata_json=json.dumps(dict(run_state=False, ne_sha256=sha256(path / 'ne.txt'),
                                                   ns_sha256=sha256(path / 'ns.txt'),
                                                   gate_config=force.gate.model_dump_json())))
    land = land or {t: dict(manning_n=0, infiltration='none') for t in set(types)}
    dc = domain(path, duration=3600, warmup=warmup, yield_step=yield_step, restart=str(seed), land=land)
    return dc, force, topo, depth, bed


def event_steps(path: Path, step: float, end: float, width=30, height=10):
    """A zero-rain raster whose intervals end every ``step`` seconds up to
    ``end``: every interval end is a step event (tests/test_gate_solver.py:253-262)."""
    count = round(end / step)
    times = [i * step for i in range(count + 1)] + [3600]
    return write_rain(path, np.zeros((len(times) - 1, 1, 1), np.float32), from_origin(0, height, width, height),
                      list(zip(times, times[1:])))


def run(dc, force, seconds, *, output=None, restart=None, engine='oracle'):
    """_solve to an exact clock tick (tests/test_gate_solver.py:62-75)."""
    seconds = round(seconds * 2 ** 40) / 2 ** 40
    changes = {}
    if output is not None:
        changes['domain_dir'] = str(output)
    if restart is not None:
        changes['restart_state'] = str(restart)
    dc = dc.model_copy(update=changes)
    Path(dc.domain_dir).mkdir(parents=True, exist_ok=True)
    return run_case(dc, force, engine, end_time=seconds)
