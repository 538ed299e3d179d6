"""Absolute-time forcing: boundary series, exterior-edge selection and rain.

Same contract as the reference's preprocess/force.py:83-218:
  * ``TimeSeries``     – CSV ``time,value`` relative to the domain start,
                         linear interpolation (np.interp);
  * ``load_line``      – GeoJSON LineString/MultiLineString with a declared
                         CRS equal to the mesh EPSG;
  * ``load_boundaries``– an exterior edge belongs to a boundary when its
                         overlap with the line has positive length; each cell
                         is weighted by its selected edge length;
  * ``RainField``      – interval CSV + one raster band of millimetres per
                         interval, sampled at the pixel of each cell centre;
  * ``Forcing.load``   – boundaries, rain and the step-splitting events.
The GIS stack (shapely, rasterio) is absent; the geometric selection below is
exact for the axis-aligned exterior edges of Cartesian meshes.
"""
from __future__ import annotations

import csv
import json
import re
from dataclasses import dataclass

import numpy as np

from .input import absolute_time
from .raster import read_geotiff


@dataclass
class TimeSeries:
    times: np.ndarray   # seconds from simulation start, F64
    values: np.ndarray

    @classmethod
    def load(cls, path, origin, begin, end):
        with open(path, newline='') as file:
            rows = list(csv.DictReader(file))
        times = np.array([(absolute_time(r['time']) - origin).total_seconds() for r in rows])
        values = np.array([float(r['value']) for r in rows])
        if len(times) < 2 or not np.all(np.isfinite(values)) or np.any(np.diff(times) <= 0):
            raise ValueError(f'{path}: need finite values and strictly increasing times (at least two)')
        if times[0] > begin or times[-1] < end:
            raise ValueError(f'{path}: series does not cover [{begin}, {end}] seconds from start')
        return cls(times, values)

    def at(self, seconds) -> float:
        return float(np.interp(seconds, self.times, self.values))


def _epsg_of(name: str) -> int | None:
    match = re.search(r'EPSG:+(\d+)', name, flags=re.IGNORECASE)
    return int(match.group(1)) if match else None


def load_line(path, epsg) -> list[np.ndarray]:
    """Polylines (each [k, 2] F64) of a GeoJSON line file."""
    with open(path) as file:
        data = json.load(file)
    if 'crs' not in data:
        raise ValueError(f'{path}: GeoJSON must declare its CRS')
    if _epsg_of(str(data['crs'].get('properties', {}).get('name', ''))) != int(epsg):
        raise ValueError(f'{path}: boundary CRS differs from mesh EPSG:{epsg}')
    if data['type'] == 'FeatureCollection':
        geometries = [f['geometry'] for f in data['features']]
    elif data['type'] == 'Feature':
        geometries = [data['geometry']]
    else:
        geometries = [data]
    lines = []
    for g in geometries:
        if g.get('type') == 'LineString':
            parts = [g['coordinates']]
        elif g.get('type') == 'MultiLineString':
            parts = g['coordinates']
        else:
            raise ValueError(f'{path}: expected nonempty LineString or MultiLineString')
        for part in parts:
            pts = np.asarray(part, dtype=np.float64).reshape(-1, 2)
            if len(pts) < 2 or not np.all(np.isfinite(pts)):
                raise ValueError(f'{path}: expected nonempty LineString or MultiLineString')
            lines.append(pts)
    if not lines:
        raise ValueError(f'{path}: expected nonempty LineString or MultiLineString')
    return lines


def overlap_lengths(segments: np.ndarray, lines: list[np.ndarray]) -> np.ndarray:
    """Length of the overlap of each axis-aligned segment with the polylines.

    Only collinear pieces have positive length: a vertical edge at x = c
    overlaps line pieces with both endpoints at x = c, a horizontal edge at
    y = c those with both endpoints at y = c.
    """
    a, b = segments[:, 0], segments[:, 1]
    vertical = a[:, 0] == b[:, 0]
    fixed = np.where(vertical, a[:, 0], a[:, 1])
    lo = np.where(vertical, np.minimum(a[:, 1], b[:, 1]), np.minimum(a[:, 0], b[:, 0]))
    hi = np.where(vertical, np.maximum(a[:, 1], b[:, 1]), np.maximum(a[:, 0], b[:, 0]))
    total = np.zeros(len(segments))
    for pts in lines:
        for p, q in zip(pts[:-1], pts[1:]):
            if p[0] == q[0] and p[1] != q[1]:
                m = vertical & (fixed == p[0])
                plo, phi = min(p[1], q[1]), max(p[1], q[1])
            elif p[1] == q[1] and p[0] != q[0]:
                m = ~vertical & (fixed == p[1])
                plo, phi = min(p[0], q[0]), max(p[0], q[0])
            else:
                continue
            total[m] += np.clip(np.minimum(hi[m], phi) - np.maximum(lo[m], plo), 0.0, None)
    return total


@dataclass
class Boundary:
    name: str
    kind: str
    cells: np.ndarray
    weights: np.ndarray
    side_ids: np.ndarray
    series: TimeSeries

    def distribute(self, q):
        return self.weights * q


def select_boundary(name, kind, lines, series, geometry, claimed) -> Boundary:
    """Exterior edges overlapping ``lines`` with positive length; each cell is
    weighted by its selected edge length (force.py:136-160)."""
    edges = geometry.exterior_edges
    selected = np.flatnonzero(overlap_lengths(edges.segments, lines) > 0)
    side_ids = edges.side_ids[selected]
    if len(side_ids) == 0:
        raise ValueError(f'{name}: boundary selects no exterior edges; '
                         'snap the line to mesh exterior edges in GIS')
    cells, inverse = np.unique(edges.cell_ids[selected], return_inverse=True)
    if np.any(claimed[cells]):
        raise ValueError(f'{name}: boundary cells overlap another boundary')
    claimed[cells] = True
    lengths = np.bincount(inverse, weights=edges.lengths[selected])
    weights = lengths / lengths.sum(dtype=np.float64)
    return Boundary(name, kind, cells, weights, side_ids, series)


def load_boundaries(config, geometry, epsg, origin, begin, end) -> list[Boundary]:
    if not config:
        return []
    claimed = np.zeros(len(geometry.x), dtype=bool)
    return [select_boundary(b.name, b.kind, load_line(b.line, epsg), TimeSeries.load(b.series, origin, begin, end),
                            geometry, claimed) for b in config]


@dataclass
class RainField:
    starts: np.ndarray
    ends: np.ndarray
    millimetres: np.ndarray  # [bands, unique sampled pixels]
    pixel_index: np.ndarray  # cell -> sampled pixel; cell 0 unused

    @classmethod
    def load(cls, config, geometry, epsg, origin, begin, end):
        with open(config.intervals, newline='') as file:
            rows = list(csv.DictReader(file))
        starts = np.array([(absolute_time(r['interval_start']) - origin).total_seconds() for r in rows])
        ends = np.array([(absolute_time(r['interval_end']) - origin).total_seconds() for r in rows])
        if not len(rows) or np.any(ends <= starts) or np.any(starts[1:] != ends[:-1]):
            raise ValueError('Rainfall intervals must be continuous, positive and nonoverlapping')
        if starts[0] > begin or ends[-1] < end:
            raise ValueError('Rainfall intervals do not cover the simulation window')
        raster = read_geotiff(config.raster)
        if raster.epsg != int(epsg):
            raise ValueError('Rainfall CRS differs from mesh CRS')
        if raster.count != len(rows):
            raise ValueError('Rainfall band count differs from interval count')
        return cls.from_raster(raster, geometry, starts, ends)

    @classmethod
    def from_raster(cls, raster, geometry, starts, ends):
        rr, cc = raster.rowcol(geometry.x[1:], geometry.y[1:])
        if np.any((rr < 0) | (rr >= raster.height) | (cc < 0) | (cc >= raster.width)):
            raise ValueError('Cell centre is outside the rainfall raster')
        pixels, inverse = np.unique(rr * raster.width + cc, return_inverse=True)
        rain = raster.data[:, pixels // raster.width, pixels % raster.width].astype(np.float32).astype(float)
        bad = ~np.isfinite(rain) | (rain < 0)
        if raster.nodata is not None:
            bad |= rain == np.float32(raster.nodata)
        if np.any(bad):
            raise ValueError('Rainfall at a cell centre is NoData, nonfinite or negative')
        mapping = np.zeros(len(geometry.x), dtype=np.int32)
        mapping[1:] = inverse.reshape(-1)
        return cls(np.asarray(starts, float), np.asarray(ends, float), rain, mapping)

    def index_at(self, seconds) -> int:
        return int(np.searchsorted(self.ends, seconds, side='right'))

    def rates(self, index) -> np.ndarray:
        return self.millimetres[index] * (0.001 / (self.ends[index] - self.starts[index]))


@dataclass
class Forcing:
    boundaries: list[Boundary]
    rain: RainField
    events: np.ndarray

    @classmethod
    def load(cls, domain, config, geometry):
        begin, end = 0., domain.duration
        boundaries = load_boundaries(config.boundaries, geometry, domain.epsg_code, domain.start, begin, end)
        rain = RainField.load(config.rainfall, geometry, domain.epsg_code, domain.start, begin, end)
        return cls.assemble(boundaries, rain, end)

    @classmethod
    def assemble(cls, boundaries, rain, end):
        events = np.unique(np.concatenate([rain.ends, [0., end]] + [b.series.times for b in boundaries]))
        return cls(boundaries, rain, events)
