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
  multires_quadtree_4m  the same rules over 36.6 km x 36.6 km (about 4M
                      cells, the count the configuration names).
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

from .forcing import Forcing, RainField, TimeSeries, select_boundary
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
    gate: object = None  # input.GateConfig: a gate controller block, or None

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
        """Step inputs; with an enabled gate block, the controller tables too
        (the layout resolved from the mesh bed, control from t = 0)."""
        from .model import build_step_arrays
        arrays = build_step_arrays(self.mesh, self.sbf, self.geometry, self.forcing, self.land_parameters, self.sita)
        if self.gate is not None and self.gate.enabled:
            from .gate import GateController, GateLayout
            layout = GateLayout.load(self.gate, self.geometry.bounds, self.mesh.land_type, self.mesh.topology,
                                     self.forcing.boundaries, arrays.bed)
            arrays.gate = GateController.build(self.gate, layout, arrays.bed, self.mesh.land_type,
                                               self.mesh.topology, 0.).tables
        return arrays

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


def gated_polder(n: int = 1024, dx: float = 5.0, gates: int = 4, seed: int = 6, duration: int = 3600) -> Workload:
    """River land draining south against a dike into a polder pond through
    gates. n x n cells of dx metres: the pond (class 10, bed -2 m) fills the
    southern eighth, a 4-row dike (class 3, 3 m above the land) closes it,
    and `gates` openings of 4 x 16 cells (class 11, closed at the dike top,
    open at -1 m) cut through it, each controlled by the land cell just
    north of its middle. The land (class 1, 1 m fractal relief on a 0.001
    slope towards the dike) starts with 1 m of water in the 40 rows above the
    dike and takes 50 mm/h of rain for the first hour; the pond drains over
    a free-outflow level boundary on the south edge. The trigger (level
    above the highest control bed + 0.5 m) commands every gate at t = 0 and
    they open over 600 s."""
    from .input import GateConfig
    rng = np.random.default_rng(seed)
    width = n * dx
    yc = (np.arange(n) + 0.5) * dx
    noise = fractal_noise((n, n), 5, rng)
    pond_rows, dike_rows = n // 8, 4
    dike0 = pond_rows
    land_bed = 1.0 * noise + 0.001 * (yc[:, None] - dike0 * dx)
    bed = land_bed.copy()
    land = np.ones((n, n), np.uint8)
    bed[:pond_rows] = -2.0
    land[:pond_rows] = 10
    dike_top = float(land_bed[dike0 + dike_rows:dike0 + dike_rows + 8].max()) + 3.0
    bed[dike0:dike0 + dike_rows] = dike_top
    land[dike0:dike0 + dike_rows] = 3
    centres = [int((k + 0.5) * n / gates) for k in range(gates)]
    for c in centres:
        land[dike0:dike0 + dike_rows, c - 8:c + 8] = 11
    mesh = uniform_grid(n, n, dx, bed.astype(np.float32), land)
    geometry = MeshGeometry.from_mesh(mesh)
    rain, raster = _uniform_rain(geometry, width, width, np.array([0., 3600.]), np.array([3600., float(duration) + 3600.]),
                                 [50.0, 0.0])
    outflow = -102.0
    south = [np.array([[0.0, 0.0], [width, 0.0]])]
    claimed = np.zeros(mesh.e_num, bool)
    boundary = select_boundary('south', 'level', south,
                               TimeSeries(np.array([0., float(duration)]), np.array([outflow, outflow])),
                               geometry, claimed)
    forcing = Forcing.assemble([boundary], rain, duration)
    depth = np.zeros(mesh.e_num, np.float32)
    row = np.floor(mesh.y[1:] / dx).astype(np.int64)
    depth[1:] = np.where((row >= dike0 + dike_rows) & (row < dike0 + dike_rows + 40), 1.0, 0.0)
    control_row = dike0 + dike_rows
    controls = [((c + 0.5) * dx, (control_row + 0.5) * dx) for c in centres]
    trigger = float(max(bed[control_row, c] for c in centres)) + 0.5
    gate = GateConfig(land_type=11, pond_land_type=10, enabled=True, trigger_level=trigger, opening_seconds=600.,
                      open_elevation=-1.0,
                      gates=[dict(name=f'G{k}', inside_point=((c + 0.5) * dx, (dike0 + 1.5) * dx),
                                  control_point=controls[k]) for k, c in enumerate(centres)])
    land_parameters = {1: LandParameters(manning_n=0.035, infiltration='none'),
                       3: LandParameters(manning_n=0.05, infiltration='none'),
                       10: LandParameters(manning_n=0.03, infiltration='none'),
                       11: LandParameters(manning_n=0.02, infiltration='none')}
    return Workload(f'gated_polder_{n}', mesh, geometry, forcing, land_parameters, duration=duration, yield_step=300,
                    initial_depth=depth, rain_raster=raster, meta={'lines': {'south': south}, 'seed': seed},
                    gate=gate)


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


# ------------------------------------------------------------ quadtree mesh

def _morton(i: np.ndarray, j: np.ndarray) -> np.ndarray:
    """Interleave the bits of two nonnegative < 2**16 integer arrays."""
    def spread(v):
        v = v.astype(np.uint64) & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v
    return spread(i) | (spread(j) << np.uint64(1))


def quadtree_mesh(leaf_level: np.ndarray, leaf_i: np.ndarray, leaf_j: np.ndarray, base: float, levels: int,
                  nx0: int, ny0: int, bed_at, land_at) -> MeshData:
    """Mesh of the leaves (level, i, j) of a 2:1-balanced quadtree over an
    nx0 x ny0 grid of level-0 cells of size ``base``; a level-L cell has size
    base / 2**L. Leaves are numbered in Morton order of their lower-left
    corner on the finest grid. Each side is created once from its lower
    (west/south) cell; a face with two finer neighbours has two sides,
    ordered along the face."""
    fine = 1 << (levels - 1)
    L = leaf_level.astype(np.int64)
    span = fine >> L                                   # size in finest cells
    fi, fj = leaf_i.astype(np.int64) * span, leaf_j.astype(np.int64) * span
    order = np.argsort(_morton(fi, fj), kind='stable')
    L, span, fi, fj = L[order], span[order], fi[order], fj[order]
    ii, jj = leaf_i.astype(np.int64)[order], leaf_j.astype(np.int64)[order]
    n = len(L)
    ids = np.arange(1, n + 1, dtype=np.int64)
    key = (L << 40) | (ii << 20) | jj
    sort_key = np.argsort(key)
    sorted_keys = key[sort_key]

    def lookup(lv, i, j):
        k = (lv << 40) | (i << 20) | j
        pos = np.searchsorted(sorted_keys, k)
        pos = np.minimum(pos, n - 1)
        hit = (sorted_keys[pos] == k) & (lv >= 0) & (lv < levels) & (i >= 0) & (j >= 0)
        return np.where(hit, ids[sort_key[pos]], 0)

    size = base / (1 << L).astype(np.float64)
    nxl = nx0 << L
    nyl = ny0 << L
    sides = []  # (orient, lo, hi, length, x, y)

    def neighbour_sides(orient):
        # east (orient 2) or north (orient 1) neighbours of every leaf
        di, dj = (1, 0) if orient == 2 else (0, 1)
        ni, nj = ii + di, jj + dj
        inside = (ni < nxl) if orient == 2 else (nj < nyl)
        same = lookup(L, ni, nj)
        coarse = np.where(L > 0, lookup(L - 1, ni >> 1, nj >> 1), 0)
        f1 = lookup(L + 1, 2 * ni, 2 * nj)
        f2 = lookup(L + 1, 2 * ni + (0 if orient == 2 else 1), 2 * nj + (1 if orient == 2 else 0))
        out = []
        # exterior
        m = ~inside
        if orient == 2:
            out.append((ids[m], np.zeros(m.sum(), np.int64), size[m], (ii[m] + 1) * size[m], (jj[m] + .5) * size[m]))
        else:
            out.append((ids[m], np.zeros(m.sum(), np.int64), size[m], (ii[m] + .5) * size[m], (jj[m] + 1) * size[m]))
        m = inside & (same > 0)
        x = (ii + 1) * size if orient == 2 else (ii + .5) * size
        y = (jj + .5) * size if orient == 2 else (jj + 1) * size
        out.append((ids[m], same[m], size[m], x[m], y[m]))
        m = inside & (same == 0) & (coarse > 0)
        out.append((ids[m], coarse[m], size[m], x[m], y[m]))
        m = inside & (same == 0) & (coarse == 0)
        if np.any(m & ((f1 == 0) | (f2 == 0))):
            raise ValueError('quadtree is not 2:1 balanced')
        half = size / 2
        for which, fid in ((0, f1), (1, f2)):
            if orient == 2:
                xs, ys = (ii + 1) * size, jj * size + (which + .5) * half
            else:
                xs, ys = ii * size + (which + .5) * half, (jj + 1) * size
            out.append((ids[m], fid[m], half[m], xs[m], ys[m]))
        lo = np.concatenate([o[0] for o in out]); hi = np.concatenate([o[1] for o in out])
        return (np.full(len(lo), orient), lo, hi, np.concatenate([o[2] for o in out]),
                np.concatenate([o[3] for o in out]), np.concatenate([o[4] for o in out]))

    def edge_sides(orient):
        # west (orient 2) or south (orient 1) exterior sides: lower cell 0
        m = (ii == 0) if orient == 2 else (jj == 0)
        x = np.zeros(m.sum()) if orient == 2 else (ii[m] + .5) * size[m]
        y = (jj[m] + .5) * size[m] if orient == 2 else np.zeros(m.sum())
        return (np.full(m.sum(), orient), np.zeros(m.sum(), np.int64), ids[m], size[m], x, y)

    parts = [neighbour_sides(2), neighbour_sides(1), edge_sides(2), edge_sides(1)]
    so = np.concatenate([p[0] for p in parts]); lo = np.concatenate([p[1] for p in parts])
    hi = np.concatenate([p[2] for p in parts]); ln = np.concatenate([p[3] for p in parts])
    sx = np.concatenate([p[4] for p in parts]); sy = np.concatenate([p[5] for p in parts])
    owner = np.where(lo > 0, lo, hi)
    sord = np.lexsort((sx, sy, so, owner))
    so, lo, hi, ln, sx, sy = so[sord], lo[sord], hi[sord], ln[sord], sx[sord], sy[sord]
    s = len(so) + 1
    sid = np.arange(1, s, dtype=np.int64)
    # faces: a vertical side is the right face of lo and the left face of hi
    cell = np.concatenate([lo, hi])
    direction = np.concatenate([np.where(so == 2, 1, 3), np.where(so == 2, 0, 2)])
    pos = np.concatenate([np.where(so == 2, sy, sx)] * 2)
    side = np.concatenate([sid, sid])
    keep = cell > 0
    cell, direction, pos, side = cell[keep], direction[keep], pos[keep], side[keep]
    fo = np.lexsort((pos, direction, cell))
    cell, direction, side = cell[fo], direction[fo], side[fo]
    e = n + 1
    counts = np.zeros((e, 4), np.int32)
    np.add.at(counts, (cell, direction), 1)
    flat = counts.reshape(-1)
    starts = np.zeros(len(flat), np.int64)
    starts[1:] = np.cumsum(flat)[:-1]
    face_ptr = starts.reshape(e, 4).astype(np.int32)
    face_ptr[0] = 0
    x = np.zeros(e, np.float32); y = np.zeros(e, np.float32)
    x[1:] = (ii + .5) * size; y[1:] = (jj + .5) * size
    z = np.zeros(e, np.float32)
    z[1:] = bed_at(x[1:].astype(np.float64), y[1:].astype(np.float64), L)
    land = np.zeros(e, np.uint8)
    land[1:] = land_at(x[1:].astype(np.float64), y[1:].astype(np.float64), L)
    topo = np.zeros((s, 3), np.int32)
    topo[1:, 0], topo[1:, 1], topo[1:, 2] = so, lo, hi
    length = np.zeros(s, np.float32); length[1:] = ln
    sxa = np.zeros(s, np.float32); sxa[1:] = sx
    sya = np.zeros(s, np.float32); sya[1:] = sy
    mesh = MeshData(x=x, y=y, z=z, land_type=land, counts=counts, face_ptr=face_ptr,
                    isl_data=side.astype(np.int32), index=np.arange(e, dtype=np.uint32), side_length=length,
                    side_x=sxa, side_y=sya, side_z=np.zeros(s, np.float32), side_attr=np.zeros(s, np.uint8),
                    side_index=np.arange(s, dtype=np.uint32), topology=topo)
    mesh.level = np.concatenate([[0], L]).astype(np.int8)
    return mesh


def meander_leaves(seed: int, width: float, base: float, buffer: float, half_channel: float):
    """Leaves of a 3-level quadtree: 5 m cells within the channel, 10 m cells
    within ``buffer`` of its centreline, 20 m elsewhere (base = 20 m)."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.1, 0.2) * width
    wavelength = rng.uniform(0.25, 0.45) * width
    phase = rng.uniform(0, 2 * np.pi)

    def distance(x, y):
        yc = width / 2 + amp * np.sin(2 * np.pi * x / wavelength + phase)
        slope = amp * 2 * np.pi / wavelength * np.cos(2 * np.pi * x / wavelength + phase)
        return np.abs(y - yc) / np.sqrt(1 + slope ** 2)

    n0 = int(round(width / base))
    j0, i0 = np.divmod(np.arange(n0 * n0, dtype=np.int64), n0)
    c0x, c0y = (i0 + .5) * base, (j0 + .5) * base
    refine0 = distance(c0x, c0y) - base * 0.7072 < buffer
    leaves = [(np.zeros((~refine0).sum(), np.int64), i0[~refine0], j0[~refine0])]
    pi, pj = i0[refine0], j0[refine0]
    ci = np.concatenate([2 * pi, 2 * pi + 1, 2 * pi, 2 * pi + 1])
    cj = np.concatenate([2 * pj, 2 * pj, 2 * pj + 1, 2 * pj + 1])
    s1 = base / 2
    refine1 = distance((ci + .5) * s1, (cj + .5) * s1) - s1 * 0.7072 < half_channel
    leaves.append((np.ones((~refine1).sum(), np.int64), ci[~refine1], cj[~refine1]))
    qi, qj = ci[refine1], cj[refine1]
    gi = np.concatenate([2 * qi, 2 * qi + 1, 2 * qi, 2 * qi + 1])
    gj = np.concatenate([2 * qj, 2 * qj, 2 * qj + 1, 2 * qj + 1])
    leaves.append((np.full(len(gi), 2, np.int64), gi, gj))
    lv = np.concatenate([l[0] for l in leaves]); li = np.concatenate([l[1] for l in leaves])
    lj = np.concatenate([l[2] for l in leaves])
    return lv, li, lj, distance, n0


def multires_quadtree(seed: int = 2, width: float = 20000.0, duration: int = 7200, *,
                      hyetograph_peak: float | None = None, n_factors=None, uniform_rain: float | None = None,
                      name: str = 'multires_quadtree') -> Workload:
    """The multi-resolution configuration: 3-level 2:1 quadtree (20/10/5 m)
    around a carved meandering channel (30 m wide, 3 m deep), fractal bed
    (5 octaves, 20 m relief) plus a 0.0005 slope towards the east, 4 land
    classes (channel n = 0.015 without infiltration; 0.035/0.05/0.08 with
    Horton f0 = 60, fc = 10 mm/h, k = 4 /h), a translating Gaussian storm
    (peak 80 mm/h, sigma 3 km, 5 m/s) in 200 m x 300 s raster bands and a
    tidal east level boundary (1.5 m amplitude, 12.42 h period, 300 s knots).

    hyetograph_peak replaces the storm by uniform rain following a triangular
    1 h pulse with that peak (mm/h) in 60 s bands; n_factors multiplies the
    Manning n of the 4 classes (the batched ensemble's perturbations);
    uniform_rain replaces it by constant uniform rain (mm/h) for the whole
    duration (the served requests)."""
    base = 20.0
    lv, li, lj, distance, n0 = meander_leaves(seed, width, base, buffer=500.0, half_channel=15.0)
    rng = np.random.default_rng(seed + 1)
    noise_n = 512
    noise = fractal_noise((noise_n, noise_n), 5, rng)
    classes_noise = fractal_noise((64, 64), 3, rng)

    def sample(field, x, y):
        k = field.shape[0]
        ix = np.clip((x / width * k).astype(np.int64), 0, k - 1)
        iy = np.clip((y / width * k).astype(np.int64), 0, k - 1)
        return field[iy, ix]

    def bed_at(x, y, level):
        z = 20.0 * sample(noise, x, y) + 0.0005 * (width - x)
        return (z - 3.0 * (distance(x, y) < 15.0)).astype(np.float32)

    def land_at(x, y, level):
        cls = 1 + np.minimum((sample(classes_noise, x, y) * 3).astype(np.int64), 2)
        return np.where(distance(x, y) < 15.0, 0, cls).astype(np.uint8)

    mesh = quadtree_mesh(lv, li, lj, base, 3, n0, n0, bed_at, land_at)
    geometry = MeshGeometry.from_mesh(mesh)
    if uniform_rain is not None:
        rain, raster = _uniform_rain(geometry, width, width, [0.0], [float(duration)],
                                     [uniform_rain * duration / 3600.0])
        return _quadtree_workload(name, seed, width, duration, mesh, geometry, rain, raster, n_factors)
    if hyetograph_peak is not None:
        starts = np.arange(0, duration, 60.0)
        ends = starts + 60.0
        mid = 0.5 * (starts + ends)
        rate = hyetograph_peak * np.clip(1.0 - np.abs(mid - 1800.0) / 1800.0, 0.0, None)  # mm/h, exact per band
        rain, raster = _uniform_rain(geometry, width, width, starts, ends, rate * 60.0 / 3600.0)
        return _quadtree_workload(name, seed, width, duration, mesh, geometry, rain, raster, n_factors)
    # translating Gaussian storm, integrated per 300 s band on 200 m pixels
    px = 200.0
    npx = int(width / px)
    starts = np.arange(0, duration, 300.0)
    ends = starts + 300.0
    cx = (np.arange(npx) + .5) * px
    X, Y = np.meshgrid(cx, cx[::-1])
    bands = np.zeros((len(starts), npx, npx))
    for b, (a, e_) in enumerate(zip(starts, ends)):
        t = 0.5 * (a + e_)
        sx, sy = -4000.0 + 5.0 * t, width / 2
        rate = 80.0 * np.exp(-((X - sx) ** 2 + (Y - sy) ** 2) / (2 * 3000.0 ** 2))   # mm/h
        bands[b] = rate * (e_ - a) / 3600.0
    raster = Raster(bands.astype(np.float32).astype(np.float64), from_origin(0, width, px, px), EPSG, None)
    rain = RainField.from_raster(raster, geometry, starts, ends)
    return _quadtree_workload(name, seed, width, duration, mesh, geometry, rain, raster, n_factors)


def multires_quadtree_4m(seed: int = 2, duration: int = 7200) -> Workload:
    """The multi-resolution configuration at the cell count its text names
    (about 4M): the same refinement rules, bed, land classes, storm and tide
    on a 36.6 km x 36.6 km domain. Over 20 km x 20 km the stated rules (5 m
    in the channel, 10 m within 500 m of it, 20 m elsewhere) give 1.36M
    cells; the 20 m cells dominate, so the domain is widened rather than the
    rules changed."""
    return multires_quadtree(seed, width=36600.0, duration=duration, name='multires_quadtree_4m')


def _quadtree_workload(name, seed, width, duration, mesh, geometry, rain, raster, n_factors) -> Workload:
    base = 20.0
    east = mesh.x[1:] > width - base
    datum = float(np.percentile(mesh.z[1:][east], 10)) + 1.0
    knots = np.arange(0, duration + 300, 300.0)
    tide = datum + 1.5 * np.sin(2 * np.pi * knots / 44712.0)
    lines = [np.array([[width, 0.0], [width, width]])]
    claimed = np.zeros(mesh.e_num, bool)
    boundary = select_boundary('tide', 'level', lines, TimeSeries(knots, tide), geometry, claimed)
    forcing = Forcing.assemble([boundary], rain, duration)
    horton = dict(f0_mm_h=60.0, fc_mm_h=10.0, k_per_h=4.0)
    n = np.array([0.015, 0.035, 0.05, 0.08]) * (1.0 if n_factors is None else np.asarray(n_factors, float))
    land_parameters = {0: LandParameters(manning_n=float(n[0]), infiltration='none'),
                       1: LandParameters(manning_n=float(n[1]), infiltration=horton),
                       2: LandParameters(manning_n=float(n[2]), infiltration=horton),
                       3: LandParameters(manning_n=float(n[3]), infiltration=horton)}
    return Workload(name, mesh, geometry, forcing, land_parameters, duration=duration,
                    yield_step=300, rain_raster=raster,
                    meta={'lines': {'tide': lines}, 'seed': seed,
                          'cells_by_level': [int((mesh.level[1:] == k).sum()) for k in range(3)]})


def quadtree_width_for(cells: float) -> float:
    """Domain width whose quadtree has about this many cells (fit of the
    generator: N(w) = 0.0026414 w^2 + 15.28 w, from 2 km and 20 km runs)."""
    a, b = 0.0026414, 15.28
    return float((-b + np.sqrt(b * b + 4 * a * cells)) / (2 * a))


def ensemble_members(seed: int = 4, members: int = 64, low: float = 50e3, high: float = 2e6,
                     duration: int = 3600) -> list[dict]:
    """Parameters of the batched ensemble: per member a seed, a target cell
    count drawn log-uniform in [low, high], a hyetograph peak ~ LogNormal(
    ln 40 mm/h, 0.5) and Manning factors U(0.8, 1.2) per class."""
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(low), np.log(high), members))
    peaks = np.exp(rng.normal(np.log(40.0), 0.5, members))
    factors = rng.uniform(0.8, 1.2, (members, 4))
    return [dict(seed=int(seed * 1000 + i), width=20.0 * max(8, round(quadtree_width_for(c) / 20.0)),
                 duration=duration,
                 hyetograph_peak=float(p), n_factors=[float(f) for f in fa], name=f'ensemble_{i:02d}')
            for i, (c, p, fa) in enumerate(zip(cells, peaks, factors))]


def _member(kw):
    return multires_quadtree(**kw)


def ensemble_scenarios(seed: int = 4, members: int = 64, low: float = 50e3, high: float = 2e6,
                       duration: int = 3600, processes: int | None = None) -> list[Workload]:
    """The batched ensemble (64 seeded quadtree meshes, about 40M cells in
    total), generated in parallel worker processes (spawned, so that no CUDA
    context is inherited)."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    params = ensemble_members(seed, members, low, high, duration)
    workers = min(len(params), processes or os.cpu_count() or 1)
    if workers <= 1:
        return [_member(kw) for kw in params]
    with ProcessPoolExecutor(workers, mp_context=mp.get_context('spawn')) as pool:
        return list(pool.map(_member, params))


def served_requests(seed: int = 5, count: int = 512, rate: float = 2.0, low: float = 16e3, high: float = 4e6,
                    duration_range=(600, 3600), rain_range=(10.0, 100.0)) -> list[dict]:
    """The served request stream: Poisson arrivals (rate per second), per
    request a seeded quadtree with a cell count drawn log-uniform in
    [low, high], uniform rain U(rain_range) mm/h and a duration
    U(duration_range) s. Returns [{'id', 'arrival', 'params'}]."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    cells = np.exp(rng.uniform(np.log(low), np.log(high), count))
    rain = rng.uniform(*rain_range, count)
    durations = rng.integers(duration_range[0], duration_range[1] + 1, count)
    out = []
    for i in range(count):
        params = dict(seed=int(seed * 100000 + i), width=20.0 * max(8, round(quadtree_width_for(cells[i]) / 20.0)),
                      duration=int(durations[i]), uniform_rain=float(rain[i]), name=f'request_{i:03d}')
        out.append(dict(id=i, arrival=float(arrivals[i]), params=params))
    return out
