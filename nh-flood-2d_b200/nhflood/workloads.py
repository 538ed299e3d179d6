"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: every mesh, bed, land-class map, rain field
and boundary series is generated here from a seed, in memory, with the
arrays the NE/NS preprocessing would produce (index 0 is the exterior
sentinel). ``write_inputs`` writes the same case as NE/NS text, GeoJSON,
CSV, GeoTIFF and JSON configs for the file-based drop-in path.

  plain_uniform_256   256 x 256 cells at 10 m, planar 0.001 slope rising
                      towards +y plus 8 Gaussian hills, 2 land classes split
                      by a random half-plane, 50 mm/h rain for 1800 s, an
                      absorbing south level boundary (a level far below the
                      bed sets those cells to zero depth), 3600 s.
  multires_quadtree   2:1-balanced 3-level quadtree (20/10/5 m) over
                      20 km x 20 km around a carved meandering channel,
                      fractal bed, 4 land classes (3 Horton), translating
                      Gaussian storm, tidal east boundary, 7200 s.
  dambreak_4096       4096 x 4096 cells at 1 m, fractal bed + 0.002 slope,
                      2 m reservoir over the western 10 %, absorbing
                      perimeter level boundary, 1800 s.
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from datetime import datetime, timezone
from pathlib import Path

import numpy as np

from .forcing import Boundary, Forcing, RainField, TimeSeries, select_boundary
from .geometry import MeshGeometry
from .input import DomainConfig, LandParameters
from .output import Checkpoint
from .preprocess import MeshData, boundary_flags
from .raster import Raster, from_origin

START = datetime(2023, 9, 7, 8, tzinfo=timezone.utc)
EPSG = 2326


@dataclass
class Workload:
    name: str
    mesh: MeshData
    geometry: MeshGeometry
    forcing: Forcing
    land_parameters: dict
    duration: int
    yield_step: int = 300
    afa: float = 0.5
    sita: float = 1.0
    min_h: float = 0.02
    initial_depth: np.ndarray | None = None
    rain_raster: Raster | None = None
    meta: dict = field(default_factory=dict)

    @property
    def sbf(self):
        return boundary_flags(self.mesh.topology)

    @property
    def cells(self) -> int:
        return self.mesh.e_num - 1

    def domain_config(self, domain_dir) -> DomainConfig:
        Path(domain_dir).mkdir(parents=True, exist_ok=True)
        return DomainConfig.model_construct(
            ne='', ns='', epsg_code=EPSG, domain_dir=str(domain_dir), afa=self.afa, sita=self.sita,
            min_h=self.min_h, start=START, duration=self.duration, warmup_duration=0,
            land_parameters=self.land_parameters, yield_step=self.yield_step, restart_state='',
            stations={}, observation_dir='')

    def initial_state(self) -> Checkpoint | None:
        """A run_state=False seed state (the reference's way to inject an initial
        condition), or None for a dry cold start."""
        if self.initial_depth is None:
            return None
        e, s = self.mesh.e_num, self.mesh.s_num
        zeros = np.zeros(e, np.float32)
        words = np.zeros(e, np.uint32)
        depth = self.initial_depth.astype(np.float32)
        meta = json.dumps(dict(run_state=False, ne_sha256=None, ns_sha256=None, gate_config='null'))
        return Checkpoint(depth, self.mesh.z.astype(np.float32), np.zeros(s, np.float32), zeros.copy(),
                          zeros.copy(), depth.copy(), words, words.copy(), zeros.copy(), 0, 0, False, meta)

    def step_arrays(self):
        from .model import build_step_arrays
        return build_step_arrays(self.mesh, self.sbf, self.geometry, self.forcing, self.land_parameters, self.sita)

    def write_inputs(self, path) -> tuple[Path, Path]:
        """Write NE/NS text, forcing files and domain/force JSON; returns the JSON paths."""
        from .preprocess import write_ne_ns
        from .raster import write_geotiff
        path = Path(path)
        path.mkdir(parents=True, exist_ok=True)
        write_ne_ns(self.mesh, path / 'ne.txt', path / 'ns.txt')
        rain = self.forcing.rain
        raster = self.rain_raster
        write_geotiff(path / 'rain.tif', raster.data.astype(np.float32), raster.transform, EPSG)
        with open(path / 'intervals.csv', 'w') as f:
            f.write('interval_start,interval_end\n')
            for a, b in zip(rain.starts, rain.ends):
                f.write(f'{_iso(a)},{_iso(b)}\n')
        boundaries = []
        for b in self.forcing.boundaries:
            line = self.meta['lines'][b.name]
            (path / f'{b.name}.geojson').write_text(json.dumps(
                {'type': 'MultiLineString', 'coordinates': [p.tolist() for p in line],
                 'crs': {'type': 'name', 'properties': {'name': f'EPSG:{EPSG}'}}}))
            (path / f'{b.name}.csv').write_text('time,value\n' + ''.join(
                f'{_iso(t)},{repr(float(v))}\n' for t, v in zip(b.series.times, b.series.values)))
            boundaries.append(dict(name=b.name, kind=b.kind, line=str(path / f'{b.name}.geojson'),
                                   series=str(path / f'{b.name}.csv')))
        domain = dict(ne=str(path / 'ne.txt'), ns=str(path / 'ns.txt'), epsg_code=EPSG,
                      domain_dir=str(path / 'run'), afa=self.afa, sita=self.sita, min_h=self.min_h,
                      start=START.isoformat(), duration=self.duration, warmup_duration=0,
                      land_parameters={str(k): v.model_dump(mode='json') for k, v in self.land_parameters.items()},
                      yield_step=self.yield_step)
        force = dict(boundaries=boundaries, rainfall=dict(raster=str(path / 'rain.tif'),
                                                           intervals=str(path / 'intervals.csv')))
        (path / 'domain.json').write_text(json.dumps(domain, indent=2))
        (path / 'force.json').write_text(json.dumps(force, indent=2))
        return path / 'domain.json', path / 'force.json'


def _iso(seconds: float) -> str:
    from datetime import timedelta
    return (START + timedelta(seconds=float(seconds))).isoformat()


# ------------------------------------------------------------ mesh builders

def uniform_grid(nx: int, ny: int, dx: float, bed: np.ndarray, land: np.ndarray, tile: int = 32) -> MeshData:
    """nx x ny grid of square cells numbered tile by tile (tile x tile blocks in
    row-major block order, row-major inside a block), so that consecutive cell
    indices form compact tiles. Each cell owns its east and north sides (and
    its exterior west/south sides on the domain edge); sides are numbered in
    owner order, so tiles away from the edges have identical relative
    numbering."""
    n = nx * ny
    e = n + 1
    jj, ii = np.divmod(np.arange(n, dtype=np.int64), nx)          # row-major grid positions
    ntx = (nx + tile - 1) // tile
    key = ((jj // tile) * ntx + ii // tile) * (tile * tile) + (jj % tile) * tile + (ii % tile)
    order = np.argsort(key, kind='stable')                         # grid position of each cell id - 1
    cid = np.empty(n, np.int64)
    cid[order] = np.arange(1, e)                                   # cell id of each grid position
    grid_id = cid.reshape(ny, nx)
    i, j = ii[order], jj[order]                                    # grid position by cell id - 1
    x = np.zeros(e, np.float32)
    y = np.zeros(e, np.float32)
    x[1:] = (i + 0.5) * dx
    y[1:] = (j + 0.5) * dx
    z = np.zeros(e, np.float32)
    z[1:] = np.asarray(bed, np.float32).reshape(-1)[order]
    land_type = np.zeros(e, np.uint8)
    land_type[1:] = np.asarray(land).reshape(-1)[order]
    # owned sides per cell: slot 0 east, 1 north, 2 west (edge), 3 south (edge)
    owner = np.arange(1, e, dtype=np.int64)
    has = np.stack([np.ones(n, bool), np.ones(n, bool), i == 0, j == 0], axis=1)
    count = has.sum(axis=1)
    first = np.zeros(n + 1, np.int64)
    first[1:] = np.cumsum(count)
    slot_rank = np.cumsum(has, axis=1) - 1                         # rank among the cell's owned sides
    sid = np.where(has, 1 + first[:-1, None] + slot_rank, 0)       # side id per (cell, slot)
    s = 1 + int(first[-1])
    topo = np.zeros((s, 3), np.int32)
    sx = np.zeros(s, np.float32)
    sy = np.zeros(s, np.float32)
    east_nb = np.where(i < nx - 1, grid_id[j, np.minimum(i + 1, nx - 1)], 0)
    north_nb = np.where(j < ny - 1, grid_id[np.minimum(j + 1, ny - 1), i], 0)
    e_ids, n_ids = sid[:, 0], sid[:, 1]
    topo[e_ids] = np.stack([np.full(n, 2), owner, east_nb], axis=1)
    sx[e_ids], sy[e_ids] = (i + 1) * dx, (j + 0.5) * dx
    topo[n_ids] = np.stack([np.full(n, 1), owner, north_nb], axis=1)
    sx[n_ids], sy[n_ids] = (i + 0.5) * dx, (j + 1) * dx
    w = has[:, 2]
    topo[sid[w, 2]] = np.stack([np.full(w.sum(), 2), np.zeros(w.sum(), np.int64), owner[w]], axis=1)
    sx[sid[w, 2]], sy[sid[w, 2]] = 0.0, (j[w] + 0.5) * dx
    so = has[:, 3]
    topo[sid[so, 3]] = np.stack([np.full(so.sum(), 1), np.zeros(so.sum(), np.int64), owner[so]], axis=1)
    sx[sid[so, 3]], sy[sid[so, 3]] = (i[so] + 0.5) * dx, 0.0
    # faces: west side = east side of the west neighbour (or own edge side), etc.
    west_cell = np.where(i > 0, grid_id[j, np.maximum(i - 1, 0)], 0)
    south_cell = np.where(j > 0, grid_id[np.maximum(j - 1, 0), i], 0)
    west_side = np.where(i > 0, sid[np.maximum(west_cell - 1, 0), 0], sid[:, 2])
    south_side = np.where(j > 0, sid[np.maximum(south_cell - 1, 0), 1], sid[:, 3])
    counts = np.zeros((e, 4), np.int32)
    counts[1:] = 1
    face_ptr = np.zeros((e, 4), np.int32)
    face_ptr[1:] = 4 * (owner[:, None] - 1) + np.arange(4)
    isl = np.stack([west_side, e_ids, south_side, n_ids], axis=1).reshape(-1).astype(np.int32)
    length = np.full(s, dx, np.float32)
    length[0] = 0
    return MeshData(x=x, y=y, z=z, land_type=land_type, counts=counts, face_ptr=face_ptr, isl_data=isl,
                    index=np.arange(e, dtype=np.uint32), side_length=length, side_x=sx, side_y=sy,
                    side_z=np.zeros(s, np.float32), side_attr=np.zeros(s, np.uint8),
                    side_index=np.arange(s, dtype=np.uint32), topology=topo)


def fractal_noise(shape, octaves: int, rng, base_cells: int = 4) -> np.ndarray:
    """Sum of bilinearly interpolated random lattices, amplitude halving per
    octave; returns values scaled to [0, 1]."""
    ny, nx = shape
    out = np.zeros(shape, np.float64)
    amp = 1.0
    yy = np.linspace(0.0, 1.0, ny)
    xx = np.linspace(0.0, 1.0, nx)
    for o in range(octaves):
        k = base_cells * (2 ** o) + 1
        lattice = rng.random((k, k))
        fy = yy * (k - 1)
        fx = xx * (k - 1)
        y0 = np.minimum(fy.astype(np.int64), k - 2)
        x0 = np.minimum(fx.astype(np.int64), k - 2)
        ty = (fy - y0)[:, None]
        tx = (fx - x0)[None, :]
        a = lattice[y0][:, x0]
        b = lattice[y0][:, x0 + 1]
        c = lattice[y0 + 1][:, x0]
        d = lattice[y0 + 1][:, x0 + 1]
        out += amp * ((a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty)
        amp *= 0.5
    out -= out.min()
    top = out.max()
    return out / top if top > 0 else out


def _perimeter_lines(width, height):
    return [np.array([[0.0, 0.0], [width, 0.0], [width, height], [0.0, height], [0.0, 0.0]])]


def _uniform_rain(geometry, width, height, starts, ends, millimetres):
    data = np.asarray(millimetres, np.float32).reshape(-1, 1, 1)
    raster = Raster(data.astype(np.float64), from_origin(0, height, width, height), EPSG, None)
    return RainField.from_raster(raster, geometry, starts, ends), raster


def plain_uniform_256(seed: int = 1, n: int = 256, dx: float = 10.0) -> Workload:
    rng = np.random.default_rng(seed)
    width = n * dx
    xc = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(xc, xc)
    bed = 0.001 * Y
    for _ in range(8):
        amp, sigma = rng.uniform(0.5, 2.0), rng.uniform(50.0, 200.0)
        cx, cy = rng.uniform(0, width, size=2)
        bed = bed + amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sigma ** 2))
    px, py = rng.uniform(0, width, size=2)
    theta = rng.uniform(0, 2 * np.pi)
    land = np.where((X - px) * np.cos(theta) + (Y - py) * np.sin(theta) < 0, 1, 2).astype(np.uint8)
    mesh = uniform_grid(n, n, dx, bed.astype(np.float32), land)
    geometry = MeshGeometry.from_mesh(mesh)
    rain, raster = _uniform_rain(geometry, width, width, np.array([0., 1800.]), np.array([1800., 3600.]), [25.0, 0.0])
    outflow = float(mesh.z[1:].min()) - 100.0
    south = [np.array([[0.0, 0.0], [width, 0.0]])]
    claimed = np.zeros(mesh.e_num, bool)
    boundary = select_boundary('south', 'level', south, TimeSeries(np.array([0., 3600.]), np.array([outflow, outflow])),
                               geometry, claimed)
    forcing = Forcing.assemble([boundary], rain, 3600)
    land_parameters = {1: LandParameters(manning_n=0.03, infiltration='none'),
                       2: LandParameters(manning_n=0.06, infiltration='none')}
    return Workload('plain_uniform_256', mesh, geometry, forcing, land_parameters, duration=3600, yield_step=300,
                    rain_raster=raster, meta={'lines': {'south': south}, 'seed': seed})


def dambreak(n: int = 4096, dx: float = 1.0, seed: int = 3, duration: int = 1800) -> Workload:
    rng = np.random.default_rng(seed)
    width = n * dx
    noise = fractal_noise((n, n), 5, rng)
    xc = (np.arange(n) + 0.5) * dx
    bed = (10.0 * noise + 0.002 * (width - xc)[None, :]).astype(np.float32)
    land = np.ones((n, n), np.uint8)
    mesh = uniform_grid(n, n, dx, bed, land)
    geometry = MeshGeometry.from_mesh(mesh)
    rain, raster = _uniform_rain(geometry, width, width, np.array([0.]), np.array([float(duration)]), [0.0])
    outflow = float(mesh.z[1:].min()) - 100.0
    lines = _perimeter_lines(width, width)
    claimed = np.zeros(mesh.e_num, bool)
    boundary = select_boundary('perimeter', 'level', lines,
                               TimeSeries(np.array([0., float(duration)]), np.array([outflow, outflow])),
                               geometry, claimed)
    forcing = Forcing.assemble([boundary], rain, duration)
    depth = np.zeros(mesh.e_num, np.float32)
    depth[1:] = np.where(mesh.x[1:] < 0.1 * width, 2.0, 0.0)
    land_parameters = {1: LandParameters(manning_n=0.03, infiltration='none')}
    return Workload(f'dambreak_{n}', mesh, geometry, forcing, land_parameters, duration=duration, yield_step=300,
                    initial_depth=depth, rain_raster=raster, meta={'lines': {'perimeter': lines}, 'seed': seed})


def simulate(workload: Workload, domain_dir, *, engine_factory=None, end_time=None, batch_size: int = 32):
    """Run a workload through the full time loop (outputs under domain_dir).
    Returns (final budget row, run record)."""
    from .engine import evolve_loaded
    from .input import ForceConfig
    from .run_record import RunRecord
    dc = workload.domain_config(domain_dir)
    fc = ForceConfig.model_construct(boundaries=[], rainfall=None, gate=None)
    with RunRecord(dc, fc) as record:
        record.data['workload'] = workload.name
        row = evolve_loaded(dc, record, workload.duration if end_time is None else end_time, workload.mesh,
                            workload.sbf, workload.geometry, workload.forcing, engine_factory=engine_factory,
                            batch_size=batch_size, state=workload.initial_state())
    return row, record
