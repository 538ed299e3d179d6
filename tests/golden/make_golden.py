"""Generate golden vectors for the host-side inputs of the step by running
the reference's own NumPy/pydantic code.

Three parts of nh-flood-2d run without Taichi, rasterio or fastdb4py:
  * preprocess/hydraulics.py – map_land_parameters (side Manning n, cell
    Horton parameters), open_boundary_face_fractions (θ < 1 boundary faces),
    connected_still_water (the warm-up fill);
  * preprocess/gate.py – GateLayout.load (gate components, control cells,
    validation);
  * input/domain.py, input/force.py – the config schema and absolute_time;
and, from files that import Taichi, rasterio or fastdb4py at the top, the
plain-Python definitions of core/clock.py, core/pressure.py,
preprocess/domain.py, preprocess/force.py, core/run_record.py, core/gate.py
and core/output.py, compiled from their unchanged source (``definitions``).
The script runs that code from a reference checkout, feeds it seeded
synthetic meshes, configs and states, and writes what it returns
(or the error they raise) to host_golden.json and host_golden.npz next to
it. tests/test_golden_host.py replays every case through nhflood.

    python tests/golden/make_golden.py --reference PATH   (or NHF_REFERENCE=PATH)

The reference's preprocess/__init__.py imports its Taichi domain pass, so
the package object is registered without running that file; the two
modules themselves are imported as they are. The meshes are 2:1 quadtrees
built here (a 2 m base grid with random cells split into four 1 m cells).
"""
from __future__ import annotations

import argparse
import ast
import csv
import importlib
import json
import math
import os
import sys
import types
from collections import defaultdict
from dataclasses import dataclass
from datetime import datetime, timedelta, timezone
from pathlib import Path
from types import SimpleNamespace as NS

import numpy as np

HERE = Path(__file__).resolve().parent


def definitions(path: Path, names, namespace, inside=None) -> dict:
    """Compile the named top-level definitions of one reference file (or the
    named methods of its class ``inside``) from its unchanged source, and run
    them in ``namespace``. The rest of the file, which needs Taichi,
    rasterio or fastdb4py, is not run."""
    tree = ast.parse(path.read_text(), filename=str(path))
    body = tree.body
    if inside is not None:
        body = next(n for n in body if isinstance(n, ast.ClassDef) and n.name == inside).body
    keep = []
    for node in body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            keep.append(node)
        elif isinstance(node, ast.Assign) and all(isinstance(t, ast.Name) and t.id in names for t in node.targets):
            keep.append(node)
    found = {getattr(n, 'name', None) or n.targets[0].id for n in keep}
    if found != set(names):
        raise LookupError(f'{path}: missing {sorted(set(names) - found)}')
    for node in keep:
        if inside is not None:
            node.decorator_list = []
    exec(compile(ast.Module(keep, type_ignores=[]), str(path), 'exec'), namespace)
    return namespace


def load_reference(root: Path):
    src = root / 'src'
    sys.path.insert(0, str(src))
    importlib.import_module('nh_flood_2d')
    package = types.ModuleType('nh_flood_2d.preprocess')
    package.__path__ = [str(src / 'nh_flood_2d' / 'preprocess')]
    sys.modules['nh_flood_2d.preprocess'] = package
    ref = NS(hydraulics=importlib.import_module('nh_flood_2d.preprocess.hydraulics'),
             gate=importlib.import_module('nh_flood_2d.preprocess.gate'),
             input=importlib.import_module('nh_flood_2d.input'),
             force=importlib.import_module('nh_flood_2d.input.force'))
    pkg = src / 'nh_flood_2d'
    ref.pkg = pkg
    ref.clock = NS(**definitions(pkg / 'core/clock.py', ['_TICKS_PER_SECOND', '_MAX_TICKS', '_seconds_to_ticks',
                                                         '_words'], dict(math=math, np=np)))
    ref.series = NS(**definitions(pkg / 'preprocess/force.py', ['TimeSeries', 'RainField'],
                                  dict(np=np, csv=csv, dataclass=dataclass, absolute_time=ref.force.absolute_time)))
    ref.budget = NS(**definitions(pkg / 'core/run_record.py', ['WaterBudget'], dict(np=np, csv=csv)))
    ref.balance = NS(**definitions(pkg / 'core/gate.py', ['append_gate_balance'], dict(csv=csv, Path=Path)))
    ref.report = definitions(pkg / 'core/gate.py', ['report'], dict(np=np), inside='GateController')['report']
    ref.pressure = NS(**definitions(pkg / 'core/pressure.py', ['HangingGeometry', 'hanging_geometry'],
                                    dict(np=np, dataclass=dataclass)))
    ref.domain = definitions(pkg / 'preprocess/domain.py', ['_filter_ne_ns'], dict(Path=Path))
    output_names = ['STATION_FIELDS', '_float_array', '_uint_array', 'append_station_samples', 'list_depth_frames']
    ref.output = NS(**definitions(pkg / 'core/output.py', output_names, dict(np=np, csv=csv, Path=Path)))
    return ref


# ---------------------------------------------------------------- meshes

def quadtree(rng, nx, ny, split_fraction):
    """Cells (x0, x1, y0, y1) of a 2 m grid with some cells split in four;
    sides split at every neighbour corner; face CSR per direction
    (0 west, 1 east, 2 south, 3 north)."""
    cells = []
    for j in range(ny):
        for i in range(nx):
            x0, y0 = 2 * i, 2 * j
            if rng.random() < split_fraction:
                cells += [(x0 + a, x0 + a + 1, y0 + b, y0 + b + 1) for b in (0, 1) for a in (0, 1)]
            else:
                cells.append((x0, x0 + 2, y0, y0 + 2))
    breaks = {1: defaultdict(set), 2: defaultdict(set)}
    for x0, x1, y0, y1 in cells:
        breaks[2][x0].update((y0, y1)); breaks[2][x1].update((y0, y1))
        breaks[1][y0].update((x0, x1)); breaks[1][y1].update((x0, x1))
    owner = defaultdict(dict)
    faces = []
    for cell, (x0, x1, y0, y1) in enumerate(cells, 1):
        per = []
        for orient, coord, a, b, role in ((2, x0, y0, y1, 'hi'), (2, x1, y0, y1, 'lo'),
                                          (1, y0, x0, x1, 'hi'), (1, y1, x0, x1, 'lo')):
            points = sorted(p for p in breaks[orient][coord] if a <= p <= b)
            keys = [(orient, coord, u, w) for u, w in zip(points, points[1:])]
            for key in keys:
                owner[key][role] = cell
            per.append(keys)
        faces.append(per)
    side_id = {key: i for i, key in enumerate(sorted(owner), 1)}
    topology = np.zeros((len(side_id) + 1, 3), dtype=np.int32)
    length = np.zeros(len(side_id) + 1, dtype=np.float32)
    side_xy = np.zeros((len(side_id) + 1, 2), dtype=np.float64)
    for key, i in side_id.items():
        orient, coord, u, w = key
        topology[i] = (orient, owner[key].get('lo', 0), owner[key].get('hi', 0))
        length[i] = w - u
        side_xy[i] = (coord, (u + w) / 2) if orient == 2 else ((u + w) / 2, coord)
    n = len(cells) + 1
    face_ptr = np.zeros((n, 4), dtype=np.int32)
    face_count = np.zeros((n, 4), dtype=np.int32)
    flat = []
    for cell, per in enumerate(faces, 1):
        for d, keys in enumerate(per):
            face_ptr[cell, d] = len(flat)
            face_count[cell, d] = len(keys)
            flat += [side_id[k] for k in keys]
    bounds = np.zeros((n, 4), dtype=np.float64)
    bounds[1:] = [(x0, y0, x1, y1) for x0, x1, y0, y1 in cells]
    area = np.zeros(n, dtype=np.float64)
    area[1:] = (bounds[1:, 2] - bounds[1:, 0]) * (bounds[1:, 3] - bounds[1:, 1])
    return dict(topology=topology, length=length, face_ptr=face_ptr, face_count=face_count,
                flat=np.array(flat, dtype=np.int32), bounds=bounds, area=area, side_xy=side_xy,
                centre=np.column_stack([(bounds[:, 0] + bounds[:, 2]) / 2, (bounds[:, 1] + bounds[:, 3]) / 2]))


def exterior_cells(mesh, side):
    """Cells on one outer edge ('west', 'east', 'south', 'north'), id order."""
    b = mesh['bounds']
    column = {'west': 0, 'south': 1, 'east': 2, 'north': 3}[side]
    value = b[1:, column].min() if side in ('west', 'south') else b[1:, column].max()
    cells = np.flatnonzero(b[:, column] == value)
    return cells[cells != 0].astype(np.int64)


def smooth_bed(rng, mesh, relief):
    centre_x = (mesh['bounds'][:, 0] + mesh['bounds'][:, 2]) / 2
    centre_y = (mesh['bounds'][:, 1] + mesh['bounds'][:, 3]) / 2
    bed = np.zeros(len(centre_x))
    for _ in range(4):
        kx, ky, phase = rng.uniform(.05, .4), rng.uniform(.05, .4), rng.uniform(0, 2 * np.pi)
        bed += rng.uniform(.2, 1) * np.sin(kx * centre_x + ky * centre_y + phase)
    bed = relief * bed / np.abs(bed).max() + rng.normal(0, relief / 20, bed.shape)
    bed[0] = 0
    return bed.astype(np.float32)


# ---------------------------------------------------------------- cases

def decimal(rng, low, high, digits):
    return float(round(rng.uniform(low, high), digits))


def land_cases(ref, rng, mesh, arrays):
    out = []
    n = len(mesh['bounds'])
    for case in range(8):
        classes = sorted(rng.choice([0, 1, 3, 7, 10, 11, 42, 200, 255], size=rng.integers(1, 6), replace=False))
        types_ = rng.choice(classes, size=n).astype(np.uint8)
        table = {}
        for c in classes:
            if case == 7 and c == classes[-1]:
                continue  # a class without parameters: rejected
            if rng.random() < .5:
                f0 = decimal(rng, 0, 120, 3)
                table[str(int(c))] = dict(manning_n=decimal(rng, 0, .2, 5), infiltration=dict(
                    f0_mm_h=f0, fc_mm_h=decimal(rng, 0, f0, 3), k_per_h=decimal(rng, 0, 8, 4)))
            else:
                table[str(int(c))] = dict(manning_n=decimal(rng, 0, .2, 5), infiltration='none')
        parsed = {int(k): ref.input.domain.LandParameters.model_validate(v) for k, v in table.items()}
        arrays[f'land{case}_types'] = types_
        try:
            side_n, f0, fc, k = ref.hydraulics.map_land_parameters(parsed, types_, mesh['topology'])
        except ValueError as error:
            out.append(dict(table=table, error=str(error)))
            continue
        for name, value in (('side_n', side_n), ('f0', f0), ('fc', fc), ('k', k)):
            arrays[f'land{case}_{name}'] = value
        out.append(dict(table=table, error=None))
    return out


def face_fraction_cases(ref, rng, mesh, arrays):
    topology = mesh['topology']
    exterior = np.flatnonzero(((topology[:, 1] == 0) ^ (topology[:, 2] == 0)))
    out = []
    for case in range(4):
        selected = np.zeros(len(topology), dtype=bool)
        selected[rng.choice(exterior, size=max(1, int(len(exterior) * (case + 1) / 6)), replace=False)] = True
        result = ref.hydraulics.open_boundary_face_fractions(selected, mesh['length'], topology, mesh['face_ptr'],
                                                             mesh['face_count'], mesh['flat'])
        arrays[f'faces{case}_selected'] = selected
        arrays[f'faces{case}_result'] = result
        out.append(case)
    return out


def level_boundary(name, cells, level):
    return NS(name=name, kind='level', cells=np.asarray(cells, dtype=np.int64), series=NS(at=lambda t, v=level: v))


def still_water_cases(ref, rng, mesh, arrays):
    topology = mesh['topology']
    out = []
    for case in range(16):
        bed = smooth_bed(rng, mesh, relief=3.0)
        crest = np.full(len(topology), -999.0, dtype=np.float32)
        ridge = rng.choice(len(topology), size=len(topology) // 12, replace=False)
        crest[ridge] = rng.uniform(-1, 4, ridge.size).astype(np.float32)
        closed = (rng.random(len(topology)) < .04).astype(np.uint8)
        edges = rng.permutation(['west', 'east', 'south', 'north'])[:1 if case % 2 else rng.integers(2, 5)]
        specs = []
        for i, edge in enumerate(edges):
            cells = exterior_cells(mesh, edge)
            cells = cells[rng.random(cells.size) < .6] if cells.size > 2 else cells
            # shared decimal levels make one body per level; a level that is
            # not an F32 value checks the F64 comparison
            level = [0.5, 0.5, 1.1, -0.3][i] if case % 3 == 0 else decimal(rng, -1.5, 2.5, 2)
            specs.append(dict(name=f'{edge}_{i}', kind='level', cells=cells.tolist(), level=level))
        if case % 4 == 1:
            specs.append(dict(name='inflow', kind='discharge', cells=exterior_cells(mesh, 'north').tolist(),
                              level=9.0))
        boundaries = [level_boundary(s['name'], s['cells'], s['level']) if s['kind'] == 'level'
                      else NS(name=s['name'], kind='discharge', cells=np.asarray(s['cells']),
                              series=NS(at=lambda t: 9.0)) for s in specs]
        arrays[f'still{case}_bed'] = bed
        arrays[f'still{case}_crest'] = crest
        arrays[f'still{case}_closed'] = closed
        try:
            depth, meta = ref.hydraulics.connected_still_water(bed, crest, closed, topology, boundaries, mesh['area'])
        except ValueError as error:
            out.append(dict(boundaries=specs, error=str(error)))
            continue
        arrays[f'still{case}_depth'] = depth
        out.append(dict(boundaries=specs, error=None, meta=meta))
    return out


def gate_mesh(rng):
    """A 2 m grid, 14 x 6: river (1) west of x = 10, pond (11) east of it, two
    gate strips (10) in the column x = 10-12 and one gate cell at (9, 7)."""
    mesh = quadtree(rng, 14, 6, 0.0)
    centre_x = (mesh['bounds'][:, 0] + mesh['bounds'][:, 2]) / 2
    centre_y = (mesh['bounds'][:, 1] + mesh['bounds'][:, 3]) / 2
    types_ = np.where(centre_x < 10, 1, 11).astype(np.uint8)
    # the lower and upper strip, with a pond cell between them, and the gate cell at (9, 7)
    types_[(centre_x > 10) & (centre_x < 12) & (centre_y < 6)] = 10
    types_[(centre_x > 10) & (centre_x < 12) & (centre_y > 8)] = 10
    types_[(centre_x > 8) & (centre_x < 10) & (centre_y > 6) & (centre_y < 8)] = 10
    types_[0] = 0
    return mesh, types_, centre_x, centre_y


def gate_cases(ref, rng, arrays):
    mesh, types_, cx, cy = gate_mesh(rng)
    arrays['gate_bounds'] = mesh['bounds']
    arrays['gate_topology'] = mesh['topology']
    arrays['gate_types'] = types_
    bed = np.where(types_ == 10, 2.0, 0.5).astype(np.float32)
    bed[0] = 0
    arrays['gate_bed'] = bed
    strip_low = (11.0, 3.0)      # inside the lower strip
    strip_high = (11.0, 10.0)    # inside the upper strip
    island = (9.0, 7.0)          # a gate cell between river and the pond cell between the strips
    river = (3.0, 3.0)
    pond = (20.0, 6.0)
    corner = (10.0, 6.0)         # a corner shared by four cells: first id wins
    base = [('north', strip_high, river), ('south', strip_low, pond), ('island', island, river)]
    variants = [
        dict(gates=base),
        dict(gates=base, open_elevation=2.0),
        dict(gates=base, open_elevation=float(np.nextafter(np.float32(2.0), np.float32(3.0)))),
        dict(gates=base[:2]),
        dict(gates=[base[0], ('south', strip_low, pond), ('again', (11.0, 1.0), river)]),
        dict(gates=[base[0], ('south', strip_low, strip_high), base[2]]),
        dict(gates=[base[0], ('south', river, pond), base[2]]),
        dict(gates=[base[0], ('south', (99.0, 3.0), pond), base[2]]),
        dict(gates=[base[0], ('south', strip_low, corner), base[2]]),
        dict(gates=base, pond_land_type=12),
        dict(gates=base, overlap=True),
        dict(gates=base, level_on='gate'),
        dict(gates=base, level_on='river'),
        dict(gates=[base[0], base[1], ('island', (8.0, 6.0), river)]),
        dict(gates=[base[0], base[1], ('island', island, (12.0, 8.0))]),
    ]
    out = []
    for i, v in enumerate(variants):
        land_types = types_.copy()
        if v.get('overlap'):
            land_types[land_types == 10] = 11
        pond_type = v.get('pond_land_type', 11)
        config = NS(land_type=10, pond_land_type=pond_type, open_elevation=v.get('open_elevation', 1.0),
                    gates=[NS(name=n, inside_point=p, control_point=q) for n, p, q in v['gates']])
        boundaries = []
        if v.get('level_on') == 'gate':
            boundaries.append(NS(kind='level', cells=np.flatnonzero(land_types == 10)[:1]))
        elif v.get('level_on') == 'river':
            boundaries.append(NS(kind='level', cells=np.flatnonzero(land_types == 1)[:3]))
        spec = dict(land_type=10, pond_land_type=pond_type, open_elevation=config.open_elevation,
                    gates=[dict(name=n, inside_point=list(p), control_point=list(q)) for n, p, q in v['gates']],
                    overlap=bool(v.get('overlap')), level_cells=[b.cells.tolist() for b in boundaries])
        try:
            layout = ref.gate.GateLayout.load(config, NS(bounds=mesh['bounds']), land_types, mesh['topology'],
                                              boundaries, bed)
        except ValueError as error:
            out.append(dict(spec, error=str(error)))
            continue
        out.append(dict(spec, error=None, cell_gate=layout.cell_gate.tolist(), controls=layout.controls.tolist(),
                        cells=[c.tolist() for c in layout.cells]))
    return out


def hanging_cases(ref, rng, arrays):
    """hanging_geometry on a uniform grid (None), and on quadtrees."""
    out = []
    for case, (nx, ny, split) in enumerate([(6, 5, 0.0), (12, 9, 0.3), (10, 10, 0.6), (7, 3, 0.15)]):
        mesh = quadtree(rng, nx, ny, split)
        x, y = mesh['centre'][:, 0], mesh['centre'][:, 1]
        sx, sy = mesh['side_xy'][:, 0], mesh['side_xy'][:, 1]
        for key, value in (('x', x), ('y', y), ('sx', sx), ('sy', sy), ('topology', mesh['topology'])):
            arrays[f'hang{case}_{key}'] = value
        result = ref.pressure.hanging_geometry(x, y, sx, sy, mesh['topology'])
        if result is None:
            out.append(dict(none=True))
            continue
        for key in ('edge_index', 'offsets', 'gradient_slots', 'cells', 'axes'):
            arrays[f'hang{case}_{key}'] = getattr(result, key)
        out.append(dict(none=False))
    return out


def ne_ns_text(rng, mesh, missing_fraction):
    """NE lines (id, 4 face counts, side ids, x, y, z, class) and NS lines
    (id, orient, left, right, bottom, top, length, x, y, z, attr) of a
    quadtree, with some cells given the z = -9999 marker."""
    ne = []
    for cell in range(1, len(mesh['bounds'])):
        ids = [mesh['flat'][mesh['face_ptr'][cell, d] + k] for d in range(4) for k in range(mesh['face_count'][cell, d])]
        z = '-9999' if rng.random() < missing_fraction else repr(float(np.float32(rng.uniform(-5, 40))))
        if z == '-9999' and rng.random() < .3:
            z = '-9999.0'
        x, y = mesh['centre'][cell]
        ne.append(','.join(map(str, [cell, *mesh['face_count'][cell].tolist(), *ids, x, y, z, int(rng.integers(1, 5))])))
    ns = []
    for side in range(1, len(mesh['topology'])):
        orient, lo, hi = mesh['topology'][side].tolist()
        nb = (lo, hi, 0, 0) if orient == 2 else (0, 0, lo, hi)
        x, y = mesh['side_xy'][side]
        ns.append(','.join(map(str, [side, orient, *nb, float(mesh['length'][side]), x, y, 0, 0])))
    return '\n'.join(ne) + '\n', '\n'.join(ns) + '\n'


def filter_cases(ref, rng, work: Path):
    out = []
    for case, (nx, ny, split, missing) in enumerate([(5, 4, 0.3, 0.0), (8, 6, 0.4, 0.15), (6, 6, 0.5, 0.5)]):
        ne_text, ns_text = ne_ns_text(rng, quadtree(rng, nx, ny, split), missing)
        (work / 'ne.txt').write_text(ne_text)
        (work / 'ns.txt').write_text(ns_text)
        ref.domain['_filter_ne_ns'](str(work / 'ne.txt'), str(work / 'ns.txt'), str(work / 'ne_out.txt'),
                                    str(work / 'ns_out.txt'))
        out.append(dict(ne=ne_text, ns=ns_text, ne_out=(work / 'ne_out.txt').read_text(),
                        ns_out=(work / 'ns_out.txt').read_text()))
    return out


def hanging_gate_cases(ref, arrays):
    """GateLayout.load on a refined quadtree: two gate strips (class 10) of
    mixed 2 m and 1 m cells, joined within each strip through hanging
    subedges, between river (1) and pond (11) cells."""
    rng = np.random.default_rng(7)
    mesh = quadtree(rng, 12, 8, 0.4)
    cx, cy = mesh['centre'][:, 0], mesh['centre'][:, 1]
    types_ = np.where(cx < 10, 1, 11).astype(np.uint8)
    strip = (cx > 10) & (cx < 14)
    types_[strip] = 1
    types_[strip & ((cy < 6) | (cy > 10))] = 10
    types_[0] = 0
    bed = np.where(types_ == 10, 2.0, 0.5).astype(np.float32)
    bed[0] = 0
    for key, value in (('bounds', mesh['bounds']), ('topology', mesh['topology']), ('types', types_), ('bed', bed)):
        arrays[f'hgate_{key}'] = value
    low, high, river = ('low', (12.0, 3.0), (5.0, 3.0)), ('high', (11.0, 13.0), (5.0, 13.0)), (5.0, 8.0)
    variants = [
        dict(gates=[low, high]),
        dict(gates=[('low', (12.0, 2.0), (10.0, 4.0)), ('high', (13.0, 11.0), (10.0, 16.0))]),
        dict(gates=[low]),
        dict(gates=[low, ('high', (11.0, 13.0), (12.0, 12.0))]),
        dict(gates=[low, ('high', (12.0, 8.0), river)]),
        dict(gates=[low, high], open_elevation=2.5),
    ]
    out = []
    for v in variants:
        config = NS(land_type=10, pond_land_type=11, open_elevation=v.get('open_elevation', 1.0),
                    gates=[NS(name=n, inside_point=p, control_point=q) for n, p, q in v['gates']])
        spec = dict(land_type=10, pond_land_type=11, open_elevation=config.open_elevation,
                    gates=[dict(name=n, inside_point=list(p), control_point=list(q)) for n, p, q in v['gates']],
                    overlap=False, level_cells=[])
        try:
            layout = ref.gate.GateLayout.load(config, NS(bounds=mesh['bounds']), types_, mesh['topology'], [], bed)
        except ValueError as error:
            out.append(dict(spec, error=str(error)))
            continue
        out.append(dict(spec, error=None, cell_gate=layout.cell_gate.tolist(), controls=layout.controls.tolist(),
                        cells=[c.tolist() for c in layout.cells]))
    return out


def output_cases(ref, work: Path):
    """The checkpoint and frame array rules and stations.csv rows."""
    values = [[0.0, 1.5, -2.25], [], [[1.0, 2.0]], [1.0, float('nan')], [1.0, float('inf')], [1e39], [0, 1, 4294967295],
              [0, 4294967296], [-1, 2], [1.5, 2.0], [True, False], [7], [3.0, 4.0], 5]
    arrays = []
    for value in values:
        case = dict(value=[repr(v) if isinstance(v, float) else v for v in value] if isinstance(value, list) else value)
        for kind, check in (('float', ref.output._float_array), ('uint', ref.output._uint_array)):
            try:
                result = check(value if not isinstance(value, list) else np.array(value), 'field')
                case[kind] = dict(dtype=str(result.dtype), values=result.tolist())
            except ValueError as error:
                case[kind] = dict(error=str(error))
        arrays.append(case)
    path = work / 'stations.csv'
    rng = np.random.default_rng(11)
    for k in range(3):
        samples = {name: dict(cell_id=int(rng.integers(1, 1000)), depth=float(np.float32(rng.uniform(0, 2))),
                              level=float(rng.uniform(-5, 20)), u=float(rng.normal()), v=float(rng.normal()))
                   for name in rng.permutation(['gauge_b', 'Gauge_a', 'gauge_c', 'z1'])[:int(rng.integers(1, 5))]}
        ref.output.append_station_samples(path, elapsed_seconds=300 * k, time=f'2023-09-07T08:{5 * k:02d}:00+00:00',
                                          samples=samples)
        arrays.append(dict(stations_call=dict(elapsed_seconds=300 * k, time=f'2023-09-07T08:{5 * k:02d}:00+00:00',
                                              samples=samples)))
    frame_sets = [['depth_900.fdb', 'depth_0.fdb', 'depth_10800.fdb', 'depth_2700.fdb'], ['depth_0900.fdb', 'depth_-5.fdb'],
                  ['depth_1e3.fdb'], ['depth_.fdb'], [], ['depth_300.fdb', 'other.fdb', 'depth_300.txt']]
    frames = []
    for k, names in enumerate(frame_sets):
        root = work / f'frames{k}'
        (root / 'frames').mkdir(parents=True)
        for name in names:
            (root / 'frames' / name).write_bytes(b'')
        try:
            listed = [[seconds, Path(p).name] for seconds, p in ref.output.list_depth_frames(root)]
            frames.append(dict(names=names, listed=listed))
        except ValueError as error:
            frames.append(dict(names=names, error=str(error).replace(str(root), '{root}')))
    return dict(cases=arrays, stations_csv=path.read_text(), frames=frames, timelines=bed_timeline_cases(ref))


def bed_timeline_cases(ref):
    """BedTimeline.at (core/output.py:299-343) over seeded bed events and gate
    openings; the base bed comes from a stand-in for the bed.fdb reader."""
    rng = np.random.default_rng(17)
    out = []
    for case in range(3):
        n = 24
        bed = rng.uniform(-2, 5, n).astype(np.float32)
        bed[0] = 0
        events = [dict(elapsed_seconds=float(t), cell_ids=rng.choice(np.arange(1, n), 3, replace=False).tolist(),
                       new_bed=[float(np.float32(v)) for v in rng.uniform(-3, 3, 3)])
                  for t in rng.permutation([0.0, 450.0, 1200.5, 3600.0])]
        origin = float(rng.choice([0.0, 1800.0, 7.125]))
        formal = round(origin * 2 ** 40)
        gates = []
        for g in range(2):
            cells = list(range(3 + 8 * g, 7 + 8 * g))
            command = None if (case, g) == (1, 1) else float(rng.uniform(0, 900))
            ticks = None if command is None else formal + round(command * 2 ** 40)
            gates.append(dict(cell_ids=cells, closed_elevation=[float(bed[c]) for c in cells], command_seconds=command,
                              command_clock_ticks=None if ticks is None else [ticks >> 32, ticks & 0xffffffff]))
        manifest = dict(bed_events=events, gate_control=dict(gates=gates, clock_origin_before_start_s=origin,
                                                              opening_seconds=float(rng.uniform(60, 1200)),
                                                              open_elevation=-1.0))
        names = dict(np=np, Path=Path, json=json, _uint_array=ref.output._uint_array,
                     _float_array=ref.output._float_array, read_bed=lambda path, count, b=bed: b.copy())
        timeline_class = definitions(ref.pkg / 'core/output.py', ['read_manifest', 'BedTimeline'], names)['BedTimeline']
        timeline = timeline_class('output', manifest)
        times = [0.0, 100.0, 450.0, 700.25, 1200.5, 2000.0, 3600.0, 9000.0]
        out.append(dict(bed=bed.tolist(), manifest=manifest, times=times,
                        beds=[timeline.at(t).astype(np.float32).tolist() for t in times]))
    return out


class ClockField:
    """A stand-in for a device field of StepClock: it keeps what is uploaded
    and returns the trace rows it is given."""

    def __init__(self):
        self.value, self.rows = None, None

    def from_numpy(self, array):
        self.value = np.array(array)

    def fill(self, value):
        self.value = value

    def to_numpy(self):
        return np.array(self.rows, dtype=np.uint32)


def trace_rows(start_ticks, statuses, rng):
    """Trace rows whose completed steps end at increasing tick counts."""
    rows, now = [], start_ticks
    for status in statuses:
        row = [0] * 10
        row[3] = status
        if status == 1:
            now += int(rng.integers(1, 1 << 40))
            row[1], row[2] = now >> 32, now & 0xffffffff
        rows.append(row)
    return rows


def clock_protocol_cases(ref, pkg: Path):
    """StepClock.begin / read_trace (core/clock.py:71-92,187-203) on a
    stand-in clock: the words uploaded, the host tick mirror and the errors."""
    names = dict(math=math, np=np, _seconds_to_ticks=ref.clock._seconds_to_ticks, _words=ref.clock._words,
                 _TICKS_PER_SECOND=ref.clock._TICKS_PER_SECOND)
    fns = definitions(pkg / 'core/clock.py', ['host_now_seconds', 'begin', 'read_trace'], names, inside='StepClock')

    class Clock:
        DONE, COMPLETED, BAD_CFL, BAD_DT, OVERSHOOT = 0, 1, 2, 3, 4
        host_now_seconds = property(fns['host_now_seconds'])
        begin, read_trace = fns['begin'], fns['read_trace']

        def __init__(self, seconds):
            self._host_now_ticks = ref.clock._seconds_to_ticks(seconds)
            self._batch_pending = False
            self.next, self.origin, self.trace = ClockField(), ClockField(), ClockField()

    rng = np.random.default_rng(13)
    out = []
    for initial, script in [
        (0.0, [('begin', 10.0, 0.0), ('trace', [1, 1, 1, 0, 0]), ('begin', 20.0, 'now'), ('trace', [1] * 32)]),
        (0.0, [('begin', 10.0, 2e-6), ('begin', 10.0, 5e-7), ('begin', 11.0, 0.0)]),
        (1234.5, [('begin', 1234.0, 1234.5), ('begin', 1234.5, 1234.5 + 1e-7), ('trace', [0] * 4)]),
        (0.0, [('trace', [1, 0]), ('begin', 5.0, math.nan), ('begin', 5.0, 0.0), ('trace', [1, 2, 1])]),
        (7.25, [('begin', 9.0, 7.25), ('trace', [1, 1, 9, 1]), ('begin', 9.0, 'now'), ('trace', [1, 3])]),
        (0.0, [('begin', 3.0, 0.0), ('trace', [1, 4, 0]), ('begin', 3.0, 'now'), ('trace', [1, 1, 5])]),
    ]:
        clock, steps = Clock(initial), []
        for op in script:
            step = dict(op=op[0])
            try:
                if op[0] == 'begin':
                    origin = clock.host_now_seconds if op[2] == 'now' else op[2]
                    step.update(target=op[1], origin=repr(float(origin)))
                    clock.begin(op[1], origin)
                    step.update(next=clock.next.value.tolist(), origin_words=clock.origin.value.tolist())
                else:
                    clock.trace.rows = trace_rows(clock._host_now_ticks, op[1], rng)
                    step.update(rows=clock.trace.rows)
                    clock.read_trace()
            except (ValueError, RuntimeError) as error:
                step.update(error=type(error).__name__, message=str(error))
            step.update(now=str(clock._host_now_ticks), pending=clock._batch_pending)
            steps.append(step)
        out.append(dict(initial=initial, steps=steps))
    return out


# ---------------------------------------------------------------- clock, series, rain

def tick_cases(ref, rng):
    values = [0.0, -0.0, 1.0, 0.5, 2.0 ** -41, 3 * 2.0 ** -41, 5 * 2.0 ** -41, 2.0 ** -40, 1e-6, 1e-12, 0.1, 1 / 3,
              3600.000001, 16777215.999999, 2.0 ** 24 - 2.0 ** -29, 2.0 ** 24, 1.5e7, -1e-300, math.nan, math.inf,
              -math.inf, 1e300, 5e-324]
    values += (10.0 ** rng.uniform(-13, 7.2, 120)).tolist()
    values += ((rng.integers(1, 1 << 20, 40) * 2 + 1).astype(float) * 2.0 ** -41).tolist()  # exact half ticks
    out = []
    for value in values:
        try:
            ticks = ref.clock._seconds_to_ticks(value)
        except ValueError as error:
            out.append(dict(seconds=repr(float(value)), error=str(error)))
            continue
        out.append(dict(seconds=repr(float(value)), ticks=str(ticks), words=ref.clock._words(ticks).tolist()))
    return out


ORIGIN = datetime(2023, 9, 7, 8, tzinfo=timezone.utc)


def series_cases(ref, rng, work: Path):
    out = []
    for case in range(10):
        n = int(rng.integers(2, 12)) if case != 6 else 1
        steps = rng.choice([0.25, 0.5, 1, 7.5, 60, 300, 1e-3], size=n) * rng.integers(1, 5, size=n)
        times = np.concatenate([[0.0], np.cumsum(steps[1:])])
        times -= float(rng.uniform(0, 0.5 * times[-1]))
        if case == 7:
            times[-1] = times[-2]
        values = [repr(float(round(v, 4))) for v in rng.normal(0, 5, n)]
        if case == 8:
            values[0] = 'nan'
        lines = ['time,value']
        for t, v in zip(times, values):
            offset = timezone(timedelta(hours=int(rng.integers(-11, 13)), minutes=int(rng.choice([0, 30]))))
            lines.append(f'{(ORIGIN + timedelta(seconds=float(t))).astimezone(offset).isoformat()},{v}')
        text = '\n'.join(lines) + '\n'
        end = float(times[-1]) + (5.0 if case == 9 else -float(rng.uniform(0, 0.1 * (times[-1] - times[0]))))
        path = work / f'series{case}.csv'
        path.write_text(text)
        spec = dict(csv=text, begin=0.0, end=max(end, 0.0))
        try:
            series = ref.series.TimeSeries.load(path, ORIGIN, spec['begin'], spec['end'])
        except ValueError as error:
            out.append(dict(spec, error=str(error).replace(str(path), '{path}')))
            continue
        queries = np.concatenate([series.times, rng.uniform(series.times[0] - 10, series.times[-1] + 10, 30)])
        out.append(dict(spec, error=None, times=series.times.tolist(), values=series.values.tolist(),
                        queries=queries.tolist(), at=[series.at(q) for q in queries]))
    return out


def rain_cases(ref, rng):
    out = []
    for case in range(6):
        bands, pixels = int(rng.integers(1, 8)), int(rng.integers(1, 6))
        durations = rng.choice([60.0, 300.0, 0.5, 1800.0, 7.25], size=bands)
        starts = -float(rng.uniform(0, 100)) + np.concatenate([[0.0], np.cumsum(durations[:-1])])
        ends = starts + durations
        mm = rng.uniform(0, 30, (bands, pixels)).astype(np.float32).astype(float)
        mapping = rng.integers(0, pixels, 20).astype(np.int32)
        mapping[0] = 0
        field = ref.series.RainField(starts, ends, mm, mapping)
        queries = np.concatenate([starts, ends, rng.uniform(starts[0] - 5, ends[-1] + 5, 20)])
        out.append(dict(starts=starts.tolist(), ends=ends.tolist(), millimetres=mm.tolist(), pixel_index=mapping.tolist(),
                        queries=queries.tolist(), index=[field.index_at(q) for q in queries],
                        rates=[field.rates(i).tolist() for i in range(bands)]))
    return out


# ---------------------------------------------------------------- budget rows and gate reports

def budget_cases(ref, rng, work: Path):
    out = []
    for case in range(6):
        nb = int(rng.integers(0, 4)) if case else 0
        boundaries = [NS(kind=str(rng.choice(['level', 'discharge'])), name=f'edge{i}') for i in range(nb)]
        initial = float(rng.uniform(0, 1e4)) if case else 0.0
        path = work / f'budget{case}.csv'
        budget = ref.budget.WaterBudget(path, boundaries, initial)
        calls = []
        for k in range(4):
            for _ in range(int(rng.integers(1, 6))):
                dt = float(np.float32(rng.uniform(0.01, 1)))
                rain = float(rng.uniform(0, 5)) if case else 0.0
                values = rng.normal(0, 3, nb) if case else np.zeros(nb)
                budget.add_forcing(dt, rain, values)
                calls.append(['forcing', dt, rain, values.tolist()])
            terms = rng.normal(0, 10, 4 + 6 * nb) if case else np.zeros(4 + 6 * nb)
            budget.set_device_terms(terms)
            calls.append(['terms', terms.tolist()])
            date, seconds = ORIGIN + timedelta(seconds=300 * k), 300 * k
            storage = float(rng.uniform(0, 2e4)) if case else 0.0
            phase = 'warmup' if k == 0 else 'simulation'
            budget.output(date, seconds, storage, phase)
            calls.append(['output', date.isoformat(), seconds, storage, phase])
        budget.close()
        out.append(dict(boundaries=[[b.kind, b.name] for b in boundaries], initial=initial, calls=calls,
                        csv=path.read_text()))
    return out


class Field:
    """A stand-in for a device field: to_numpy() returns a copy."""

    def __init__(self, array):
        self.array = np.asarray(array)

    def to_numpy(self):
        return self.array.copy()


def report_cases(ref, rng, arrays, gates, work: Path):
    """GateController.report on seeded controller state for the first valid
    gate layout, and gate_balance.csv rows appended from three reports."""
    spec = next(g for g in gates if g['error'] is None and len(g['gates']) == 3)
    types_ = arrays['gate_types']
    n_gates = len(spec['gates'])
    cells = [np.array(c, dtype=np.int32) for c in spec['cells']]
    layout = NS(cells=cells, controls=np.array(spec['controls'], dtype=np.int32))
    bed = arrays['gate_bed']
    pond = (types_ == spec['pond_land_type']).astype(np.int32)
    pond[0] = 0
    area = np.full(len(types_), 4.0)
    out = []
    path = work / 'gate_balance.csv'
    for case in range(3):
        origin_seconds = float(rng.choice([0.0, 3600.0, 1234.5]))
        formal = ref.clock._seconds_to_ticks(origin_seconds)
        commanded = rng.integers(0, 2, n_gates).astype(np.int32)
        flow_seen = rng.integers(0, 2, n_gates).astype(np.int32)
        opened = rng.integers(0, 2, n_gates).astype(np.int32)

        def words():
            ticks = formal + rng.integers(0, 1 << 52, n_gates).astype(np.uint64)
            return np.stack([ticks >> np.uint64(32), ticks & np.uint64(0xffffffff)], axis=1).astype(np.uint32)

        command, first_flow, opened_at = words(), words(), words()
        totals = rng.normal(0, 50, 4 * n_gates + 8 + 6 * n_gates)
        depth = rng.uniform(0, 2, len(types_)).astype(np.float32)
        initial_storage = float(rng.uniform(0, 500))
        initial_channel = rng.uniform(0, 50, n_gates)
        config = NS(gates=[NS(name=g['name']) for g in spec['gates']], opening_seconds=float(rng.uniform(60, 900)),
                    trigger_level=float(rng.uniform(0, 3)), pond_land_type=spec['pond_land_type'],
                    open_elevation=spec['open_elevation'])
        clock_seconds = float(rng.uniform(0, 2e5))
        controller = NS(budget=NS(flush=lambda t=totals: t.copy()), commanded=Field(commanded), command=Field(command),
                        flow_seen=Field(flow_seen), first_flow=Field(first_flow), opened=Field(opened),
                        opened_at=Field(opened_at), formal_tick=formal, config=config, closed=Field(bed),
                        layout=layout, channel_source_offset=4 * n_gates + 8, initial_channel_storage=initial_channel,
                        offset=4 * n_gates, pond=Field(pond), initial_storage=initial_storage)
        report = ref.report(controller, depth, area, clock_seconds)
        ref.balance.append_gate_balance(path, ORIGIN + timedelta(seconds=clock_seconds), clock_seconds, report)
        out.append(dict(origin_seconds=origin_seconds, commanded=commanded.tolist(), command=command.tolist(),
                        flow_seen=flow_seen.tolist(), first_flow=first_flow.tolist(), opened=opened.tolist(),
                        opened_at=opened_at.tolist(), totals=totals.tolist(), depth=depth.tolist(),
                        initial_storage=initial_storage, initial_channel=initial_channel.tolist(),
                        opening_seconds=config.opening_seconds, trigger_level=config.trigger_level,
                        clock_seconds=clock_seconds, report=report))
    return dict(gate_case=gates.index(spec), area=4.0, cases=out, balance_csv=path.read_text())


# ---------------------------------------------------------------- configs

DOMAIN = dict(ne='NE', ns='NS', epsg_code=2326, domain_dir='OUT', start='2023-09-07T16:00:00+08:00',
              duration=3600, warmup_duration=0,
              land_parameters={'10': dict(manning_n=0.03, infiltration='none')})
FORCE = dict(boundaries=[dict(name='river', kind='discharge', line='line.geojson', series='q.csv')],
             rainfall=dict(raster='rain.tif', intervals='rain.csv'))
GATE = dict(land_type=10, pond_land_type=11, enabled=True, trigger_level=1.5, opening_seconds=600,
            open_elevation=0.5, gates=[dict(name='g1', inside_point=[1, 2], control_point=[3, 4])])

DOMAIN_CHANGES = [
    {}, {'afa': 0}, {'afa': 1}, {'afa': 1.01}, {'sita': -0.1}, {'sita': 0.7}, {'sita': 1.5}, {'min_h': 0},
    {'min_h': 1e-3}, {'start': '2023-09-07T16:00:00'}, {'start': 1694054400}, {'start': '2023-09-07T08:00:00Z'},
    {'duration': 0}, {'duration': 16777215}, {'duration': 16777215, 'warmup_duration': 1},
    {'warmup_duration': -1}, {'warmup_duration': 600}, {'land_parameters': {}},
    {'land_parameters': {'256': dict(manning_n=0.03, infiltration='none')}},
    {'land_parameters': {'-1': dict(manning_n=0.03, infiltration='none')}},
    {'land_parameters': {'0': dict(manning_n=0.0, infiltration='none')}},
    {'land_parameters': {'10': dict(manning_n=-0.01, infiltration='none')}},
    {'land_parameters': {'10': dict(manning_n=0.03, infiltration=dict(f0_mm_h=5, fc_mm_h=10, k_per_h=2))}},
    {'land_parameters': {'10': dict(manning_n=0.03, infiltration=dict(f0_mm_h=60, fc_mm_h=10, k_per_h=4))}},
    {'land_parameters': {'10': dict(manning_n=0.03, infiltration=dict(f0_mm_h=60, fc_mm_h=10))}},
    {'land_parameters': {'10': dict(manning_n=0.03, infiltration='horton')}},
    {'land_parameters': {'10': dict(manning_n=0.03)}},
    {'land_parameters': {'10': dict(manning_n=0.03, infiltration='none', extra=1)}},
    {'manning': {'10': 0.03}}, {'yield_step': 0}, {'yield_step': 60}, {'yield_step': 300.5},
    {'yield_step': 300.0}, {'stations': {'a': [1, 2]}}, {'stations': {'a': [1]}}, {'stations': {'a': [1, 2, 3]}},
    {'restart_state': 'state.fdb'}, {'observation_dir': 'obs'}, {'ne': 'MISSING'}, {'epsg_code': '2326'},
    {'epsg_code': 2326.5}, {'duration': '3600'},
]
FORCE_CHANGES = [
    {}, {'boundaries': []},
    {'boundaries': [FORCE['boundaries'][0], dict(FORCE['boundaries'][0])]},
    {'boundaries': [dict(FORCE['boundaries'][0], kind='flow')]},
    {'boundaries': [dict(FORCE['boundaries'][0], name='')]},
    {'boundaries': [dict(FORCE['boundaries'][0], kind='level'), dict(FORCE['boundaries'][0], name='sea')]},
    {'rainfall': dict(raster='rain.tif')}, {'gate': None}, {'gate': GATE},
    {'gate': dict(GATE, pond_land_type=10)}, {'gate': dict(GATE, opening_seconds=0)},
    {'gate': dict(GATE, gates=[])}, {'gate': dict(GATE, land_type=256)},
    {'gate': dict(GATE, gates=[GATE['gates'][0], GATE['gates'][0]])},
    {'gate': dict(GATE, gates=[dict(GATE['gates'][0], inside_point=[1])])},
    {'gate': dict(GATE, extra=True)}, {'gate': {k: v for k, v in GATE.items() if k != 'enabled'}},
    {'pipes': []},
]
TIMES = ['2023-09-07T08:00:00Z', '2023-09-07T16:00:00+08:00', '2023-09-07T08:00:00', '2023-09-07',
         '2023-09-07T08:00:00.123456-03:30', '2023-09-07 08:00:00+00:00', '2023-02-29T00:00:00Z']


def validate(model, text):
    from pydantic import ValidationError
    try:
        value = model.model_validate_json(text)
    except ValidationError as error:
        return dict(accepted=False, errors=sorted([[str(p) for p in e['loc']] for e in error.errors()]))
    return dict(accepted=True, dump=value.model_dump(mode='json'))


def config_cases(ref, work: Path):
    (work / 'NE').write_text('mesh\n')
    (work / 'NS').write_text('mesh\n')

    def place(d):
        return {k: (str(work / v) if k in ('ne', 'ns', 'domain_dir') and isinstance(v, str) else v)
                for k, v in d.items()}

    def unplace(value):
        if isinstance(value, dict):
            return {k: unplace(v) for k, v in value.items()}
        if isinstance(value, str) and value.startswith(str(work) + '/'):
            return value[len(str(work)) + 1:]
        return value

    out = []
    for change in DOMAIN_CHANGES:
        config = {**DOMAIN, **change}
        result = validate(ref.input.DomainConfig, json.dumps(place(config)))
        out.append(dict(kind='domain', config=config, **unplace(result)))
    for change in FORCE_CHANGES:
        config = {**FORCE, **change}
        result = validate(ref.input.ForceConfig, json.dumps(config))
        out.append(dict(kind='force', config=config, **result))
    times = []
    for text in TIMES:
        try:
            times.append(dict(text=text, value=ref.force.absolute_time(text).isoformat()))
        except ValueError as error:
            times.append(dict(text=text, error=str(error)))
    return out, times


def main():
    import tempfile
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument('--reference', type=Path, default=os.environ.get('NHF_REFERENCE'),
                        help='a checkout of nh-flood-2d (or set NHF_REFERENCE)')
    args = parser.parse_args()
    if args.reference is None:
        parser.error('give --reference PATH or set NHF_REFERENCE')
    args.reference = Path(args.reference)
    ref = load_reference(args.reference)
    rng = np.random.default_rng(20261204)
    arrays = {}
    mesh = quadtree(rng, 12, 9, 0.3)
    for key in ('topology', 'length', 'face_ptr', 'face_count', 'flat', 'bounds', 'area'):
        arrays[f'mesh_{key}'] = mesh[key]
    golden = dict(land=land_cases(ref, rng, mesh, arrays), faces=face_fraction_cases(ref, rng, mesh, arrays),
                  still=still_water_cases(ref, rng, mesh, arrays), gate=gate_cases(ref, rng, arrays))
    golden['hanging'] = hanging_cases(ref, rng, arrays)
    golden['ticks'] = tick_cases(ref, rng)
    golden['rain'] = rain_cases(ref, rng)
    with tempfile.TemporaryDirectory() as work:
        golden['configs'], golden['times'] = config_cases(ref, Path(work))
        golden['series'] = series_cases(ref, rng, Path(work))
        golden['budget'] = budget_cases(ref, rng, Path(work))
        golden['report'] = report_cases(ref, rng, arrays, golden['gate'], Path(work))
        golden['filter'] = filter_cases(ref, rng, Path(work))
        golden['output'] = output_cases(ref, Path(work))
    golden['hanging_gate'] = hanging_gate_cases(ref, arrays)
    golden['clock_protocol'] = clock_protocol_cases(ref, args.reference / 'src' / 'nh_flood_2d')
    (HERE / 'host_golden.json').write_text(json.dumps(golden, separators=(',', ':')) + '\n')
    np.savez_compressed(HERE / 'host_golden.npz', **arrays)
    summary = {k: (sum(c.get('error') is not None for c in v if isinstance(c, dict)), len(v))
               for k, v in golden.items() if isinstance(v, list)}
    print('cases (errors, total):', summary)


if __name__ == '__main__':
    main()
