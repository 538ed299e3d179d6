"""Frames, extrema, checkpoints and station samples (host I/O only).

Same file names, table names and columns as the reference's core/output.py
(lines 20-348); the container is nhflood.fdb (same schema, own byte format).
"""
from __future__ import annotations

import csv
import json
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import fdb

STATION_FIELDS = ('elapsed_seconds', 'time', 'station', 'cell_id', 'depth', 'level', 'u', 'v')
_CHECKPOINT_FLOATS = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed')
_CHECKPOINT_INTS = ('clock_hi', 'clock_lo', 'gate_open')
_CHECKPOINT_TIME = ('first_time_hi', 'first_time_lo')


@dataclass
class Extrema:
    max_depth: np.ndarray
    first_time_hi: np.ndarray
    first_time_lo: np.ndarray
    max_speed: np.ndarray


@dataclass
class Checkpoint:
    depth: np.ndarray
    bed: np.ndarray
    q: np.ndarray
    rain_time: np.ndarray
    infiltration: np.ndarray
    max_depth: np.ndarray
    first_time_hi: np.ndarray
    first_time_lo: np.ndarray
    max_speed: np.ndarray
    clock_hi: int
    clock_lo: int
    gate_open: bool
    metadata_json: str


def _float_array(value, name):
    array = np.asarray(value, dtype=np.float32)
    if array.ndim != 1 or not np.all(np.isfinite(array)):
        raise ValueError(f'{name} must be a finite one-dimensional F32 array')
    return array


def _uint_array(value, name):
    array = np.asarray(value)
    if (array.ndim != 1 or not np.issubdtype(array.dtype, np.number)
            or not np.all(np.isfinite(array)) or np.any(array != np.floor(array))
            or np.any(array < 0) or np.any(array > np.iinfo(np.uint32).max)):
        raise ValueError(f'{name} must be a one-dimensional U32 array')
    return array.astype(np.uint32)


def write_bed(path, bed):
    fdb.save(path, [('F32Value', 'bed', {'value': _float_array(bed, 'bed')})])


def _read_named(path, feature, name, column, expected_count=None):
    values = fdb.load(path).table(feature, name)[column]
    if expected_count is not None and len(values) != expected_count:
        raise ValueError(f'{path}: {name} has {len(values)} rows, expected {expected_count}')
    return values


def read_bed(path, expected_count=None):
    return _read_named(path, 'F32Value', 'bed', 'value', expected_count)


def write_depth_frame(path, depth):
    values = _float_array(depth, 'depth')
    if np.any(values < 0):
        raise ValueError('depth must be nonnegative')
    fdb.save(path, [('F32Value', 'depth', {'value': values})])


def read_depth_frame(path, expected_count=None):
    values = _read_named(path, 'F32Value', 'depth', 'value', expected_count)
    if not np.all(np.isfinite(values)) or np.any(values < 0):
        raise ValueError(f'{path}: invalid depth frame')
    return values


def list_depth_frames(output_root):
    """(elapsed seconds, path) pairs in numeric order."""
    frames = []
    for path in (Path(output_root) / 'frames').glob('depth_*.fdb'):
        try:
            seconds = int(path.stem.removeprefix('depth_'))
        except ValueError as exc:
            raise ValueError(f'Invalid depth frame name: {path}') from exc
        frames.append((seconds, path))
    return sorted(frames)


def write_extrema(path, max_depth, first_time_hi, first_time_lo, max_speed):
    arrays = {
        'max_depth': _float_array(max_depth, 'max_depth'),
        'max_speed': _float_array(max_speed, 'max_speed'),
        'first_time_hi': _uint_array(first_time_hi, 'first_time_hi'),
        'first_time_lo': _uint_array(first_time_lo, 'first_time_lo'),
    }
    if len({len(a) for a in arrays.values()}) != 1:
        raise ValueError('extrema arrays must have the same number of cells')
    fdb.save(path, [('F32Value', 'max_depth', {'value': arrays['max_depth']}),
                    ('F32Value', 'max_speed', {'value': arrays['max_speed']}),
                    ('IndexLike', 'first_time_hi', {'index': arrays['first_time_hi']}),
                    ('IndexLike', 'first_time_lo', {'index': arrays['first_time_lo']})])


def read_extrema(path, expected_count=None):
    db = fdb.load(path)
    result = Extrema(db.table('F32Value', 'max_depth')['value'],
                     db.table('IndexLike', 'first_time_hi')['index'],
                     db.table('IndexLike', 'first_time_lo')['index'],
                     db.table('F32Value', 'max_speed')['value'])
    sizes = {len(result.max_depth), len(result.first_time_hi), len(result.first_time_lo), len(result.max_speed)}
    if len(sizes) != 1 or (expected_count is not None and len(result.max_depth) != expected_count):
        raise ValueError(f'{path}: extrema cell count differs from mesh')
    return result


def write_checkpoint(path, *, depth, bed, q, rain_time, infiltration, max_depth, first_time_hi,
                     first_time_lo, max_speed, clock_hi, clock_lo, gate_open, metadata_json):
    """Persist a completed step; metadata_json is kept verbatim (output.py:171-211)."""
    arrays = {name: _float_array(value, name) for name, value in
              [('depth', depth), ('bed', bed), ('q', q), ('rain_time', rain_time),
               ('infiltration', infiltration), ('max_depth', max_depth), ('max_speed', max_speed)]}
    if len({len(arrays[n]) for n in ('depth', 'bed', 'rain_time', 'infiltration', 'max_depth', 'max_speed')}) != 1:
        raise ValueError('checkpoint cell arrays must have the same length')
    times = {name: _uint_array(value, name) for name, value in
             [('first_time_hi', first_time_hi), ('first_time_lo', first_time_lo)]}
    if any(len(v) != len(arrays['depth']) for v in times.values()):
        raise ValueError('checkpoint first-time arrays must match cell count')
    if np.any(arrays['depth'] < 0):
        raise ValueError('checkpoint depth must be nonnegative')
    if not isinstance(metadata_json, str):
        raise TypeError('metadata_json must be a JSON string')
    json.loads(metadata_json)
    if not isinstance(gate_open, (bool, np.bool_)):
        raise TypeError('gate_open must be boolean')
    ints = [_uint_array([v], n) for n, v in
            [('clock_hi', clock_hi), ('clock_lo', clock_lo), ('gate_open', int(gate_open))]]
    tables = [('F32Value', n, {'value': a}) for n, a in arrays.items()]
    tables += [('IndexLike', n, {'index': a}) for n, a in zip(_CHECKPOINT_INTS, ints)]
    tables += [('IndexLike', n, {'index': a}) for n, a in times.items()]
    tables.append(('U8Value', 'state_meta', {'value': np.frombuffer(metadata_json.encode('utf-8'), np.uint8)}))
    fdb.save(path, tables)


def read_checkpoint(path, expected_cells=None, expected_sides=None):
    db = fdb.load(path)
    floats = {n: db.table('F32Value', n)['value'] for n in _CHECKPOINT_FLOATS}
    ints = {n: db.table('IndexLike', n)['index'] for n in _CHECKPOINT_INTS}
    times = {n: db.table('IndexLike', n)['index'] for n in _CHECKPOINT_TIME}
    metadata_json = db.table('U8Value', 'state_meta')['value'].tobytes().decode('utf-8')
    if len({len(floats[n]) for n in ('depth', 'bed', 'rain_time', 'infiltration', 'max_depth', 'max_speed')}) != 1:
        raise ValueError(f'{path}: inconsistent checkpoint cell counts')
    if any(len(v) != len(floats['depth']) for v in times.values()):
        raise ValueError(f'{path}: inconsistent checkpoint first-time counts')
    if expected_cells is not None and len(floats['depth']) != expected_cells:
        raise ValueError(f'{path}: checkpoint cell count differs from mesh')
    if expected_sides is not None and len(floats['q']) != expected_sides:
        raise ValueError(f'{path}: checkpoint side count differs from mesh')
    if any(len(v) != 1 for v in ints.values()):
        raise ValueError(f'{path}: checkpoint scalar count must be one')
    if any(not np.all(np.isfinite(v)) for v in floats.values()) or np.any(floats['depth'] < 0):
        raise ValueError(f'{path}: invalid checkpoint F32 state')
    if ints['gate_open'][0] not in (0, 1):
        raise ValueError(f'{path}: invalid checkpoint gate state')
    json.loads(metadata_json)
    return Checkpoint(floats['depth'], floats['bed'], floats['q'], floats['rain_time'],
                      floats['infiltration'], floats['max_depth'], times['first_time_hi'],
                      times['first_time_lo'], floats['max_speed'], int(ints['clock_hi'][0]),
                      int(ints['clock_lo'][0]), bool(ints['gate_open'][0]), metadata_json)


def resolve_station_cells(points, geometry):
    """Station -> smallest real cell id whose closed rectangle holds the point
    (output.py:246-268)."""
    left, bottom, right, top = (geometry.bounds[1:, i] for i in range(4))
    resolved = {}
    for name, (x, y) in points.items():
        if not np.isfinite(x) or not np.isfinite(y):
            raise ValueError(f'Station {name}: coordinates must be finite')
        hit = np.flatnonzero((left <= x) & (x <= right) & (bottom <= y) & (y <= top))
        if not len(hit):
            raise ValueError(f'Station {name}: ({x}, {y}) lies outside the mesh')
        resolved[name] = int(hit[0] + 1)
    return resolved


def append_station_samples(path, *, elapsed_seconds, time, samples):
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    needs_header = not path.exists()
    with path.open('a', newline='') as stream:
        writer = csv.DictWriter(stream, fieldnames=STATION_FIELDS)
        if needs_header:
            writer.writeheader()
        for name in sorted(samples):
            sample = samples[name]
            writer.writerow({'elapsed_seconds': elapsed_seconds, 'time': time, 'station': name,
                             **{k: sample[k] for k in ('cell_id', 'depth', 'level', 'u', 'v')}})


def write_manifest(path, manifest):
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    temporary = path.with_name(f'.{path.name}.{os.getpid()}.tmp')
    temporary.write_text(json.dumps(manifest, ensure_ascii=False, indent=2) + '\n')
    os.replace(temporary, path)


def read_manifest(path):
    return json.loads(Path(path).read_text())


class BedTimeline:
    """Working bed at a frame time: bed.fdb plus recorded bed events, then the
    gate beds re-derived from the manifest's ``gate_control`` block with the
    device's F32 opening arithmetic (output.py:299-343)."""

    def __init__(self, output_root, manifest=None, expected_count=None):
        output_root = Path(output_root)
        manifest = read_manifest(output_root.parent / 'manifest.json') if manifest is None else manifest
        self.bed = read_bed(output_root / 'bed.fdb', expected_count)
        self.events = sorted(manifest.get('bed_events', []), key=lambda e: e['elapsed_seconds'])
        self.gate_control = manifest.get('gate_control', {})
        self.cursor = 0
        self.seconds = float('-inf')

    def _gate_beds(self, elapsed_seconds):
        control = self.gate_control
        f32 = np.float32
        for gate in control.get('gates', []):
            cells = np.asarray(gate['cell_ids'], dtype=np.int64)
            closed = np.asarray(gate['closed_elevation'], dtype=f32)
            fraction = f32(0.)
            command = gate['command_seconds']
            if command is not None and elapsed_seconds >= command:
                hi, lo = gate['command_clock_ticks']
                tick = round((elapsed_seconds + control['clock_origin_before_start_s']) * 2 ** 40)
                age_ticks = max(tick - ((int(hi) << 32) | int(lo)), 0)
                age = f32(age_ticks >> 32) / f32(256.) + f32(age_ticks & 0xffffffff) * f32(2. ** -40)
                fraction = np.minimum(age / f32(control['opening_seconds']), f32(1.))
            opened = f32(control['open_elevation'])
            self.bed[cells] = closed + (opened - closed) * fraction
            if fraction >= 1.:
                self.bed[cells] = opened

    def at(self, elapsed_seconds):
        if elapsed_seconds < self.seconds:
            raise ValueError('BedTimeline requires nondecreasing frame times')
        while self.cursor < len(self.events) and self.events[self.cursor]['elapsed_seconds'] <= elapsed_seconds:
            event = self.events[self.cursor]
            ids = _uint_array(event['cell_ids'], 'bed event cell_ids')
            new_bed = _float_array(event['new_bed'], 'bed event new_bed')
            if len(ids) != len(new_bed) or np.any(ids >= len(self.bed)):
                raise ValueError('bed event has invalid cell ids or values')
            self.bed[ids] = new_bed
            self.cursor += 1
        self.seconds = elapsed_seconds
        self._gate_beds(elapsed_seconds)
        return self.bed


def read_bed_at(output_root, elapsed_seconds, manifest=None, expected_count=None):
    return BedTimeline(output_root, manifest, expected_count).at(elapsed_seconds)
