"""Small NE/NS cases rebuilt from the reference tests' fixtures.

The reference's physics tests (tests/test_solver_forcing.py:64-122 two
cells, tests/test_positivity.py:23-57 3x3 grid, tests/test_face_flux.py:
273-333 coarse/fine channel, tests/test_pressure_gradient.py:23-67 split-face
quadtree, tests/test_open_boundary.py:327-361 uniform strip) write tiny text
meshes, a one-pixel rain raster and seed checkpoints, then run the real
solver. This module writes the same inputs with this project's own code so
that the same known answers can be checked against the CPU restatement and
the CUDA step.
"""
from __future__ import annotations

import csv
import json
from collections import defaultdict
from datetime import datetime, timedelta, timezone
from pathlib import Path

import numpy as np

from nhflood.input import DomainConfig, ForceConfig
from nhflood.output import write_checkpoint
from nhflood.raster import from_origin, write_geotiff
from nhflood.run_record import sha256

START = datetime(2023, 9, 7, 8, tzinfo=timezone.utc)
EPSG = 2326


def iso(seconds: float) -> str:
    return (START + timedelta(seconds=seconds)).isoformat()


def write_line(path: Path, points) -> str:
    path.write_text(json.dumps({'type': 'LineString', 'coordinates': [list(map(float, p)) for p in points],
                                'crs': {'type': 'name', 'properties': {'name': f'EPSG:{EPSG}'}}}))
    return str(path)


def write_series(path: Path, rows) -> str:
    path.write_text('time,value\n' + ''.join(f'{iso(t)},{v}\n' for t, v in rows))
    return str(path)


def write_rain(path: Path, bands, transform, intervals) -> dict:
    """bands: [n, rows, cols] millimetres; intervals: [(start_s, end_s)]."""
    write_geotiff(path / 'rain.tif', np.asarray(bands, dtype=np.float32), transform, EPSG)
    with open(path / 'intervals.csv', 'w', newline='') as out:
        w = csv.writer(out)
        w.writerow(['interval_start', 'interval_end'])
        for a, b in intervals:
            w.writerow([iso(a), iso(b)])
    return dict(raster=str(path / 'rain.tif'), intervals=str(path / 'intervals.csv'))


def seed_checkpoint(path: Path, ne: Path, ns: Path, *, depth, bed=None, q=None, rain_time=None,
                    infiltration=None) -> str:
    """A ``run_state: False`` checkpoint carrying an initial state."""
    depth = np.asarray(depth, dtype=np.float32)
    zeros = np.zeros_like(depth)
    side_count = len(ns.read_text().splitlines()) + 1
    words = np.zeros(len(depth), dtype=np.uint32)
    write_checkpoint(path, depth=depth, bed=zeros if bed is None else np.asarray(bed, np.float32),
                     q=np.zeros(side_count, np.float32) if q is None else np.asarray(q, np.float32),
                     rain_time=zeros if rain_time is None else rain_time,
                     infiltration=zeros if infiltration is None else infiltration,
                     max_depth=depth.copy(), first_time_hi=words, first_time_lo=words, max_speed=zeros,
                     clock_hi=0, clock_lo=0, gate_open=False,
                     metadata_json=json.dumps(dict(run_state=False, ne_sha256=sha256(ne), ns_sha256=sha256(ns),
                                                   gate_config='null')))
    return str(path)


# ----------------------------------------------------------------- meshes

def two_cell_mesh(path: Path, *, bed=0., land_type=10, connected=False):
    """Two 10 m cells centred at x = 5 and 15 (y = 5), isolated or sharing side 2."""
    ne, ns = [], []
    for ei, x in ((1, 5.0), (2, 15.0)):
        f = 4 * (ei - 1) + 1
        left = 2 if (connected and ei == 2) else f
        ne.append(f'{ei},1,1,1,1,{left},{f + 1},{f + 2},{f + 3},{x},5,{bed},{land_type}')
        rows = [(f, 2, 0, ei, 0, 0, x - 5, 5), (f + 1, 2, ei, 0, 0, 0, x + 5, 5),
                (f + 2, 1, 0, 0, 0, ei, x, 0), (f + 3, 1, 0, 0, ei, 0, x, 10)]
        for sid, o, l, r, b, t, sx, sy in rows:
            if connected and sid == 5:
                continue
            if connected and sid == 2:
                l, r = 1, 2
            ns.append(f'{sid},{o},{l},{r},{b},{t},10,{sx},{sy},0,0')
    (path / 'ne.txt').write_text('\n'.join(ne) + '\n')
    (path / 'ns.txt').write_text('\n'.join(ns) + '\n')


def grid_cell(row, col):
    return row * 3 + col + 1


def grid_vertical(row, col):
    return row * 4 + col + 1


def grid_horizontal(row, col):
    return 13 + row * 3 + col


def grid3_mesh(path: Path, bed=0.):
    """3 x 3 grid of 10 m cells with explicit side numbering."""
    ne, ns = [], []
    for r in range(3):
        for c in range(3):
            ne.append(f'{grid_cell(r, c)},1,1,1,1,{grid_vertical(r, c)},{grid_vertical(r, c + 1)},'
                      f'{grid_horizontal(r, c)},{grid_horizontal(r + 1, c)},{5 + 10 * c},{5 + 10 * r},{bed},10')
    for r in range(3):
        for c in range(4):
            left = grid_cell(r, c - 1) if c else 0
            right = grid_cell(r, c) if c < 3 else 0
            ns.append(f'{grid_vertical(r, c)},2,{left},{right},0,0,10,{10 * c},{5 + 10 * r},0,0')
    for r in range(4):
        for c in range(3):
            bottom = grid_cell(r - 1, c) if r else 0
            top = grid_cell(r, c) if r < 3 else 0
            ns.append(f'{grid_horizontal(r, c)},1,0,0,{bottom},{top},10,{5 + 10 * c},{10 * r},0,0')
    (path / 'ne.txt').write_text('\n'.join(ne) + '\n')
    (path / 'ns.txt').write_text('\n'.join(ns) + '\n')


def rectangles_mesh(path: Path, cells, bed, land_type=10):
    """Square cells (x0, x1, y0, y1); each face is split at the corners of its
    neighbours; sides are numbered in sorted (orient, coordinate, a, b) order.
    land_type is one class for every cell or a list with one per cell."""
    types = list(land_type) if np.ndim(land_type) else [land_type] * len(cells)
    breaks = {1: defaultdict(set), 2: defaultdict(set)}
    for x0, x1, y0, y1 in cells:
        breaks[2][x0].update((y0, y1)); breaks[2][x1].update((y0, y1))
        breaks[1][y0].update((x0, x1)); breaks[1][y1].update((x0, x1))
    owner = defaultdict(dict)
    faces = []
    for ei, (x0, x1, y0, y1) in enumerate(cells, 1):
        per = []
        # (orient, coordinate, span, role): role 'hi' = cell is right/top of the side
        for orient, coord, a, b, role in ((2, x0, y0, y1, 'hi'), (2, x1, y0, y1, 'lo'),
                                          (1, y0, x0, x1, 'hi'), (1, y1, x0, x1, 'lo')):
            pts = sorted(p for p in breaks[orient][coord] if a <= p <= b)
            keys = [(orient, coord, u, w) for u, w in zip(pts, pts[1:])]
            for k in keys:
                owner[k][role] = ei
            per.append(keys)
        faces.append(per)
    sid = {k: i for i, k in enumerate(sorted(owner), 1)}
    ne = []
    for ei, ((x0, x1, y0, y1), per) in enumerate(zip(cells, faces), 1):
        ids = [sid[k] for keys in per for k in keys]
        ne.append(','.join(map(str, [ei, *(len(k) for k in per), *ids, (x0 + x1) / 2, (y0 + y1) / 2,
                                     bed[ei], types[ei - 1]])))
    ns = []
    topo = np.zeros((len(sid) + 1, 3), dtype=np.int64)
    side_xy = np.zeros((len(sid) + 1, 2))
    for k, i in sid.items():
        orient, coord, u, w = k
        lo, hi = owner[k].get('lo', 0), owner[k].get('hi', 0)
        x, y = (coord, (u + w) / 2) if orient == 2 else ((u + w) / 2, coord)
        nb = (lo, hi, 0, 0) if orient == 2 else (0, 0, lo, hi)
        ns.append(','.join(map(str, [i, orient, *nb, w - u, x, y, 0, 0])))
        topo[i] = (orient, lo, hi)
        side_xy[i] = (x, y)
    (path / 'ne.txt').write_text('\n'.join(ne) + '\n')
    (path / 'ns.txt').write_text('\n'.join(ns) + '\n')
    return topo, side_xy


def channel_cells(length=1024):
    """A 2 m wide channel: 2 m cells, then 1 m cells across the width."""
    half = length // 2
    cells = [(x, x + 2, 0, 2) for x in range(0, half, 2)]
    for x in range(half, length):
        cells += [(x, x + 1, 0, 1), (x, x + 1, 1, 2)]
    return cells


def strip_grid_mesh(path: Path, nx: int, ny: int, dx: int):
    """Uniform strip; sides numbered when first met (left, right, bottom, top per cell)."""
    sides = {}

    def side(orient, x, y, lower, higher):
        key = (orient, x, y)
        if key not in sides:
            sides[key] = [len(sides) + 1, orient, 0, 0, 0, 0, dx, x, y, 0, 0]
        row = sides[key]
        base = 2 if orient == 2 else 4
        if lower:
            row[base] = lower
        if higher:
            row[base + 1] = higher
        return row[0]

    ne = []
    for j in range(ny):
        for i in range(nx):
            cell = j * nx + i + 1
            x, y = (i + .5) * dx, (j + .5) * dx
            ids = [side(2, i * dx, y, 0, cell), side(2, (i + 1) * dx, y, cell, 0),
                   side(1, x, j * dx, 0, cell), side(1, x, (j + 1) * dx, cell, 0)]
            ne.append(','.join(map(str, [cell, 1, 1, 1, 1, *ids, x, y, 0, 10])))
    (path / 'ne.txt').write_text('\n'.join(ne) + '\n')
    (path / 'ns.txt').write_text('\n'.join(','.join(map(str, r)) for r in sides.values()) + '\n')


# ----------------------------------------------------------------- configs

def domain(path: Path, *, duration, warmup=0, land=None, yield_step=None, restart='', stations=None,
           out='out', **kw):
    land = land or {10: dict(manning_n=.03, infiltration='none')}
    return DomainConfig(ne=str(path / 'ne.txt'), ns=str(path / 'ns.txt'), epsg_code=EPSG,
                        domain_dir=str(path / out), start=START, duration=duration, warmup_duration=warmup,
                        land_parameters=land, yield_step=yield_step or duration, restart_state=restart,
                        stations=stations or {}, **kw)


def two_cell_case(path: Path, bands, duration, *, land_type=10, q=0., warmup=0, level=None, bed=0.,
                  connected=False, level_rows=None, q_rows=None, yield_step=None, infiltration='none',
                  stations=None):
    """The reference's two-cell experiment (test_solver_forcing.py:64-122)."""
    path.mkdir(parents=True, exist_ok=True)
    two_cell_mesh(path, bed=bed, land_type=land_type, connected=connected)
    values = np.asarray(bands, dtype=np.float32).reshape(-1, 1, 2)
    n = len(values)
    rain = write_rain(path, values, from_origin(0, 10, 10, 10),
                      [(i * duration / n, (i + 1) * duration / n) for i in range(n)])
    boundaries = []
    for name, val, kind, x in (('river', q, 'discharge', 0), ('sea', level, 'level', 20)):
        if val is None or (kind == 'discharge' and q == 0):
            continue
        rows = [(0, val), (duration, val)]
        if name == 'river' and q_rows:
            rows = q_rows
        if name == 'sea' and level_rows:
            rows = level_rows
        boundaries.append(dict(name=name, kind=kind, line=write_line(path / f'{name}.geojson', [[x, 1], [x, 9]]),
                               series=write_series(path / f'{name}.csv', rows)))
    dc = domain(path, duration=duration, warmup=warmup, yield_step=yield_step,
                land={land_type: dict(manning_n=.03, infiltration=infiltration)}, stations=stations)
    fc = ForceConfig(boundaries=boundaries, rainfall=rain)
    return dc, fc


def all_cells_filtered(path: Path):
    """The two-cell rain case with both cells marked z = -9999: the NE/NS
    filter leaves no cell and no side, only the sentinels."""
    dc, fc = two_cell_case(path, [[6, 6]], 10)
    lines = []
    for line in (path / 'ne.txt').read_text().splitlines():
        fields = line.split(',')
        fields[-2] = '-9999'
        lines.append(','.join(fields))
    (path / 'ne.txt').write_text('\n'.join(lines) + '\n')
    return dc, fc
