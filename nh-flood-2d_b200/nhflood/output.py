"""Solver outputs on disk: the bed, depth frames, extrema, checkpoints,
station samples, the manifest, and the bed replay of frame times.

What is shared with nh-flood-2d (core/output.py), so that downstream tools
and restart files carry over: the file names, the FDB table names and
columns, the stations.csv columns, and which arrays are accepted or refused,
with the same messages. The container bytes are nhflood.fdb's own format.

Every FDB file kind is described once, as a layout: an ordered list of
(feature, table) pairs. ``_store`` writes the arrays of a layout and
``_fetch`` reads them back. The functions below only validate and assemble.
"""
from __future__ import annotations

import csv
import json
import os
import re
from collections import deque
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import fdb

STATION_FIELDS = ('elapsed_seconds', 'time', 'station', 'cell_id', 'depth', 'level', 'u', 'v')
_U32_MAX = 0xFFFFFFFF


# ------------------------------------------------------------ array rules
# Acceptance rules of a stored array (core/output.py:53-66): F32 arrays are
# finite and one-dimensional; U32 arrays are one-dimensional whole numbers in
# [0, 2**32).

def _float_array(value, name):
    array = np.asarray(value, dtype=np.float32)
    if array.ndim == 1 and bool(np.isfinite(array).all()):
        return array
    raise ValueError(f'{name} must be a finite one-dimensional F32 array')


def _uint_array(value, name):
    array = np.asarray(value)
    valid = array.ndim == 1 and np.issubdtype(array.dtype, np.number)
    if valid:
        whole = np.isfinite(array).all() and (array == np.floor(array)).all()
        valid = bool(whole and (array >= 0).all() and (array <= _U32_MAX).all())
    if not valid:
        raise ValueError(f'{name} must be a one-dimensional U32 array')
    return array.astype(np.uint32)


# ---------------------------------------------------------------- layouts

_COLUMN = {'F32Value': 'value', 'IndexLike': 'index', 'U8Value': 'value'}


@dataclass(frozen=True)
class _Table:
    feature: str
    name: str

    @property
    def column(self) -> str:
        return _COLUMN[self.feature]


def _f32(*names):
    return tuple(_Table('F32Value', n) for n in names)


def _u32(*names):
    return tuple(_Table('IndexLike', n) for n in names)


_CELL_F32 = ('depth', 'bed', 'rain_time', 'infiltration', 'max_depth', 'max_speed')
_STATE_F32 = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed')
_SCALARS = ('clock_hi', 'clock_lo', 'gate_open')
_TIMES = ('first_time_hi', 'first_time_lo')

BED_LAYOUT = _f32('bed')
FRAME_LAYOUT = _f32('depth')
EXTREMA_LAYOUT = _f32('max_depth', 'max_speed') + _u32(*_TIMES)
CHECKPOINT_LAYOUT = _f32(*_STATE_F32) + _u32(*_SCALARS) + _u32(*_TIMES) + (_Table('U8Value', 'state_meta'),)


def _store(path, layout, arrays: dict) -> None:
    fdb.save(path, [(t.feature, t.name, {t.column: arrays[t.name]}) for t in layout])


def _fetch(path, layout) -> dict:
    db = fdb.load(path)
    return {t.name: db.table(t.feature, t.name)[t.column] for t in layout}


def _counted(path, name, values, expected_count):
    if expected_count is not None and len(values) != expected_count:
        raise ValueError(f'{path}: {name} has {len(values)} rows, expected {expected_count}')
    return values


# --------------------------------------------------------- bed and frames

def write_bed(path, bed):
    _store(path, BED_LAYOUT, {'bed': _float_array(bed, 'bed')})


def read_bed(path, expected_count=None):
    return _counted(path, 'bed', _fetch(path, BED_LAYOUT)['bed'], expected_count)


def write_depth_frame(path, depth):
    values = _float_array(depth, 'depth')
    if (values < 0).any():
        raise ValueError('depth must be nonnegative')
    _store(path, FRAME_LAYOUT, {'depth': values})


def read_depth_frame(path, expected_count=None):
    values = _counted(path, 'depth', _fetch(path, FRAME_LAYOUT)['depth'], expected_count)
    if not np.isfinite(values).all() or (values < 0).any():
        raise ValueError(f'{path}: invalid depth frame')
    return values


_FRAME_NAME = re.compile(r'depth_(.*)')


def list_depth_frames(output_root):
    """(elapsed seconds, path) of every frames/depth_<seconds>.fdb, by time."""
    found = []
    for path in (Path(output_root) / 'frames').glob('depth_*.fdb'):
        label = _FRAME_NAME.fullmatch(path.stem).group(1)
        try:
            found.append((int(label), path))
        except ValueError as exc:
            raise ValueError(f'Invalid depth frame name: {path}') from exc
    found.sort()
    return found


# ---------------------------------------------------------------- extrema

@dataclass
class Extrema:
    max_depth: np.ndarray
    first_time_hi: np.ndarray
    first_time_lo: np.ndarray
    max_speed: np.ndarray


def write_extrema(path, max_depth, first_time_hi, first_time_lo, max_speed):
    arrays = {'max_depth': _float_array(max_depth, 'max_depth'),
              'max_speed': _float_array(max_speed, 'max_speed'),
              'first_time_hi': _uint_array(first_time_hi, 'first_time_hi'),
              'first_time_lo': _uint_array(first_time_lo, 'first_time_lo')}
    if len({a.size for a in arrays.values()}) > 1:
        raise ValueError('extrema arrays must have the same number of cells')
    _store(path, EXTREMA_LAYOUT, arrays)


def read_extrema(path, expected_count=None):
    arrays = _fetch(path, EXTREMA_LAYOUT)
    sizes = {len(a) for a in arrays.values()}
    if len(sizes) > 1 or (expected_count is not None and sizes != {expected_count}):
        raise ValueError(f'{path}: extrema cell count differs from mesh')
    return Extrema(arrays['max_depth'], arrays['first_time_hi'], arrays['first_time_lo'], arrays['max_speed'])


# ------------------------------------------------------------- checkpoints

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


def write_checkpoint(path, *, depth, bed, q, rain_time, infiltration, max_depth, first_time_hi,
                     first_time_lo, max_speed, clock_hi, clock_lo, gate_open, metadata_json):
    """A completed step's state and its metadata text (kept byte for byte)."""
    given = dict(depth=depth, bed=bed, q=q, rain_time=rain_time, infiltration=infiltration,
                 max_depth=max_depth, max_speed=max_speed)
    arrays = {name: _float_array(given[name], name) for name in _STATE_F32}
    cells = len(arrays['depth'])
    if any(len(arrays[name]) != cells for name in _CELL_F32):
        raise ValueError('checkpoint cell arrays must have the same length')
    for name, value in (('first_time_hi', first_time_hi), ('first_time_lo', first_time_lo)):
        arrays[name] = _uint_array(value, name)
    if len(arrays['first_time_hi']) != cells or len(arrays['first_time_lo']) != cells:
        raise ValueError('checkpoint first-time arrays must match cell count')
    if (arrays['depth'] < 0).any():
        raise ValueError('checkpoint depth must be nonnegative')
    if not isinstance(metadata_json, str):
        raise TypeError('metadata_json must be a JSON string')
    json.loads(metadata_json)
    if not isinstance(gate_open, (bool, np.bool_)):
        raise TypeError('gate_open must be boolean')
    for name, value in (('clock_hi', clock_hi), ('clock_lo', clock_lo), ('gate_open', int(gate_open))):
        arrays[name] = _uint_array([value], name)
    arrays['state_meta'] = np.frombuffer(metadata_json.encode('utf-8'), np.uint8)
    _store(path, CHECKPOINT_LAYOUT, arrays)


def read_checkpoint(path, expected_cells=None, expected_sides=None):
    a = _fetch(path, CHECKPOINT_LAYOUT)
    cells = len(a['depth'])
    if any(len(a[name]) != cells for name in _CELL_F32):
        raise ValueError(f'{path}: inconsistent checkpoint cell counts')
    if any(len(a[name]) != cells for name in _TIMES):
        raise ValueError(f'{path}: inconsistent checkpoint first-time counts')
    if expected_cells is not None and cells != expected_cells:
        raise ValueError(f'{path}: checkpoint cell count differs from mesh')
    if expected_sides is not None and len(a['q']) != expected_sides:
        raise ValueError(f'{path}: checkpoint side count differs from mesh')
    if any(len(a[name]) != 1 for name in _SCALARS):
        raise ValueError(f'{path}: checkpoint scalar count must be one')
    if not all(np.isfinite(a[name]).all() for name in _STATE_F32) or (a['depth'] < 0).any():
        raise ValueError(f'{path}: invalid checkpoint F32 state')
    if int(a['gate_open'][0]) not in (0, 1):
        raise ValueError(f'{path}: invalid checkpoint gate state')
    metadata_json = a['state_meta'].tobytes().decode('utf-8')
    json.loads(metadata_json)
    return Checkpoint(a['depth'], a['bed'], a['q'], a['rain_time'], a['infiltration'], a['max_depth'],
                      a['first_time_hi'], a['first_time_lo'], a['max_speed'], int(a['clock_hi'][0]),
                      int(a['clock_lo'][0]), bool(a['gate_open'][0]), metadata_json)


# ---------------------------------------------------------------- stations

def resolve_station_cells(points, geometry):
    """Station name -> the smallest real cell id whose closed rectangle holds
    the point; a point on a shared edge belongs to the lower id
    (core/output.py:246-268)."""
    box = geometry.bounds[1:]
    resolved = {}
    for name, (x, y) in points.items():
        if not (np.isfinite(x) and np.isfinite(y)):
            raise ValueError(f'Station {name}: coordinates must be finite')
        inside = (box[:, 0] <= x) & (x <= box[:, 2]) & (box[:, 1] <= y) & (y <= box[:, 3])
        if not inside.any():
            raise ValueError(f'Station {name}: ({x}, {y}) lies outside the mesh')
        resolved[name] = int(np.argmax(inside)) + 1
    return resolved


def append_station_samples(path, *, elapsed_seconds, time, samples):
    """One stations.csv row per station, stations in name order; the header
    is written with the first rows."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    fresh = not path.exists()
    rows = [{'elapsed_seconds': elapsed_seconds, 'time': time, 'station': name,
             'cell_id': samples[name]['cell_id'], 'depth': samples[name]['depth'],
             'level': samples[name]['level'], 'u': samples[name]['u'], 'v': samples[name]['v']}
            for name in sorted(samples)]
    with path.open('a', newline='') as stream:
        writer = csv.DictWriter(stream, fieldnames=STATION_FIELDS)
        if fresh:
            writer.writeheader()
        writer.writerows(rows)


# ---------------------------------------------------------------- manifest

def write_manifest(path, manifest):
    """manifest.json, replaced in one step through a sibling temporary file."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    staging = path.parent / f'.{path.name}.{os.getpid()}.tmp'
    staging.write_text(json.dumps(manifest, ensure_ascii=False, indent=2) + '\n')
    os.replace(staging, path)


def read_manifest(path):
    return json.loads(Path(path).read_text())


# -------------------------------------------------------------- bed replay

@dataclass
class _GateOpening:
    """One gate of the manifest's gate_control report: its cells' closed beds
    and, once commanded, the F32 opening fraction at a frame time, computed
    as the device computes it (core/gate.py:115-135, core/output.py:323-341)."""
    cells: np.ndarray
    closed: np.ndarray
    command_seconds: float | None
    command_tick: int
    origin: float
    opening_seconds: np.float32
    open_elevation: np.float32

    @classmethod
    def from_report(cls, gate, control):
        hi, lo = gate['command_clock_ticks'] if gate.get('command_clock_ticks') else (0, 0)
        return cls(np.asarray(gate['cell_ids'], dtype=np.int64), np.asarray(gate['closed_elevation'], np.float32),
                   gate['command_seconds'], (int(hi) << 32) | int(lo), control['clock_origin_before_start_s'],
                   np.float32(control['opening_seconds']), np.float32(control['open_elevation']))

    def fraction(self, elapsed_seconds) -> np.float32:
        if self.command_seconds is None or elapsed_seconds < self.command_seconds:
            return np.float32(0.)
        tick = round((elapsed_seconds + self.origin) * 2 ** 40)
        age = max(tick - self.command_tick, 0)
        seconds = np.float32(age >> 32) / np.float32(256.) + np.float32(age & _U32_MAX) * np.float32(2. ** -40)
        return np.minimum(seconds / self.opening_seconds, np.float32(1.))

    def apply(self, bed, elapsed_seconds):
        f = self.fraction(elapsed_seconds)
        bed[self.cells] = self.closed + (self.open_elevation - self.closed) * f
        if f >= 1.:
            bed[self.cells] = self.open_elevation


class BedTimeline:
    """The working bed at nondecreasing frame times: bed.fdb, then the
    manifest's bed events up to each time in time order, then the gate beds
    of its gate_control report."""

    def __init__(self, output_root, manifest=None, expected_count=None):
        root = Path(output_root)
        if manifest is None:
            manifest = read_manifest(root.parent / 'manifest.json')
        self.bed = read_bed(root / 'bed.fdb', expected_count)
        self._events = deque(sorted(manifest.get('bed_events', []), key=lambda e: e['elapsed_seconds']))
        control = manifest.get('gate_control', {})
        self._gates = [_GateOpening.from_report(g, control) for g in control.get('gates', [])]
        self.seconds = float('-inf')

    def _apply_event(self, event):
        ids = _uint_array(event['cell_ids'], 'bed event cell_ids')
        values = _float_array(event['new_bed'], 'bed event new_bed')
        if len(ids) != len(values) or (ids >= len(self.bed)).any():
            raise ValueError('bed event has invalid cell ids or values')
        self.bed[ids] = values

    def at(self, elapsed_seconds):
        if elapsed_seconds < self.seconds:
            raise ValueError('BedTimeline requires nondecreasing frame times')
        while self._events and self._events[0]['elapsed_seconds'] <= elapsed_seconds:
            self._apply_event(self._events.popleft())
        self.seconds = elapsed_seconds
        for gate in self._gates:
            gate.apply(self.bed, elapsed_seconds)
        return self.bed


def read_bed_at(output_root, elapsed_seconds, manifest=None, expected_count=None):
    return BedTimeline(output_root, manifest, expected_count).at(elapsed_seconds)
