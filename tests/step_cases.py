"""The cases of the step's golden vectors (tests/golden/step_golden.npz).

Each case runs one solve through this project's host loop on an engine
given by a factory: the reference's own kernels under the Taichi stand-in
when tests/golden/make_step_golden.py writes the fixtures; the CPU
restatement (the oracle) or the CUDA step when tests/test_step_golden.py
checks them. ``Recorder`` wraps the engine and keeps, for every device
batch, the trace rows, the depth and discharge arrays at the batch's end,
and every budget flush.

The cases are the reference tests' own small meshes and seed states
(rebuilt by tests/scenarios.py and tests/test_oracle_physics.py) and three
small synthetic workloads with the shapes of the benchmark configurations:

  two-cell cases         tests/test_solver_forcing.py:64-122 (rain, Horton,
                         warm-up, level and discharge boundaries, sub-second
                         knots, negative discharge)
  grid3 limiter          tests/test_positivity.py:35-113 at theta 1 and 0.7
  pressure strip/plane   tests/test_pressure_gradient.py:23-95 (hanging edges)
  coarse/fine channel    tests/test_face_flux.py:113-242, first 30 s, theta 0.7
  open channel, tide     tests/test_open_boundary.py:135-205, shortened
  uniform_64             a 64 x 64 crop of the plain configuration, 5 cm
                         of water to start, 300 s
  quadtree_small         the multi-resolution generator at 2,662 cells
                         (hanging edges, Horton, moving storm, tide), 60 s
  dambreak_48            the dam-break generator at 48 x 48, 5 s
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

SNAPSHOT = ('depth', 'q')


class Recorder:
    """An engine wrapper that records what the golden vectors compare."""

    def __init__(self, engine):
        self.engine = engine
        self.rows, self.snaps, self.flushes = [], [], []

    def __getattr__(self, name):
        return getattr(self.engine, name)

    def run_batch(self, target_words, origin_words):
        rows = self.engine.run_batch(target_words, origin_words)
        self.rows.append(np.array(rows, np.uint32))
        self.snaps.append({n: self.engine.get(n) for n in SNAPSHOT})
        return rows

    def budget_flush(self):
        out = self.engine.budget_flush()
        self.flushes.append(np.array(out, np.float64))
        return out

    def result(self) -> dict:
        out = {'trace': np.concatenate(self.rows) if self.rows else np.zeros((0, 10), np.uint32),
               'budget': np.array(self.flushes, np.float64)}
        for n in SNAPSHOT:
            out[n] = np.array([s[n] for s in self.snaps])
        return out


def recording(factory):
    made = []

    def make(arrays, params):
        r = Recorder(factory(arrays, params))
        made.append(r)
        return r
    return make, made


# ------------------------------------------------------------------ cases

TWO_CELL = {
    'closed_basin': dict(bands=[[6, 6]], duration=60, q=.1, connected=True),
    'horton': dict(bands=[[100, 0], [0, 100]], duration=120, land_type=1,
                   infiltration=dict(f0_mm_h=76.2, fc_mm_h=2.54, k_per_h=2)),
    'warmup_level_discharge': dict(bands=[[6, 6]], duration=60, q=.01, warmup=20, level=.1,
                                   level_rows=[(0, .1), (60, .2)], q_rows=[(0, .01), (60, .03)], yield_step=10),
    'negative_discharge': dict(bands=[[6, 6]], duration=60, q=-10.),
    'level_knot': dict(bands=[[0, 0]], duration=1, level=0., level_rows=[(0, 0.), (.000002, 1.), (1, 0.)]),
    'cfl_after_level': dict(bands=[[0, 0]], duration=1, connected=True, level=0,
                            level_rows=[(0, 0), (.000002, 100), (1, 100)]),
    'small_rain_high_bed': dict(bands=[[.01, .01]], duration=60, bed=100.),
}


def _two_cell(name):
    def case(path, factory):
        from runner import run
        from scenarios import two_cell_case
        kw = dict(TWO_CELL[name])
        bands, duration = kw.pop('bands'), kw.pop('duration')
        dc, fc = two_cell_case(path, bands, duration, **kw)
        run(dc, fc, factory)
    return case


def _grid3(sita):
    def case(path, factory):
        from nhflood.input import ForceConfig
        from nhflood.raster import from_origin
        from runner import run
        from scenarios import (domain, grid3_mesh, grid_cell, grid_horizontal, grid_vertical, seed_checkpoint,
                               write_rain)
        path.mkdir(parents=True, exist_ok=True)
        grid3_mesh(path)
        rain = write_rain(path, [[[0]]], from_origin(0, 30, 30, 30), [(0, 20)])
        q = np.zeros(25, np.float32)
        for side, value in {grid_vertical(1, 1): -1, grid_vertical(1, 2): 1,
                            grid_horizontal(1, 1): -1, grid_horizontal(2, 1): 1}.items():
            q[side] = value
        depth = np.zeros(10, np.float32)
        depth[grid_cell(1, 1)] = .1
        seed = seed_checkpoint(path / 'seed.fdb', path / 'ne.txt', path / 'ns.txt', depth=depth, q=q)
        dc = domain(path, duration=20, yield_step=5, restart=seed, sita=sita,
                    land={10: dict(manning_n=1e-3, infiltration='none')})
        run(dc, ForceConfig(boundaries=[], rainfall=rain), factory)
    return case


def _corner_extraction(path, factory):
    from scenarios import grid_cell, grid_horizontal, grid_vertical
    from test_oracle_physics import positivity_case
    positivity_case(path, wet_cell=grid_cell(0, 0), face_flows={grid_vertical(0, 1): 1, grid_horizontal(1, 0): 1},
                    extraction=True, engine=factory)


def _pressure(kind):
    def case(path, factory):
        from test_oracle_physics import evolve, strip_cells
        if kind == 'plane':
            cells = [(0, 8, 0, 8), (8, 12, 0, 4), (8, 12, 4, 8), (0, 4, 8, 12), (4, 8, 8, 12), (8, 12, 8, 12)]
            evolve(path, cells, lambda x, y, i: .0013 * x - .0007 * y, lambda x, y, z, i: 1., seconds=30.,
                   engine=factory)
        elif kind == 'dry_tangent':
            evolve(path, strip_cells(), lambda x, y, i: .001 * y, lambda x, y, z, i: 0. if i in (1, 3) else 1.,
                   seconds=30., engine=factory)
        else:  # a rotated strip over a stepped bed with a sloping surface
            evolve(path, strip_cells(True), lambda x, y, i: ((i % 7) - 3) * .125,
                   lambda x, y, z, i: 2. - z + .01 * x, seconds=30., engine=factory)
    return case


def _channel(path, factory):
    """test_face_flux.py's coarse/fine channel, its first 30 s at theta 0.7."""
    from test_oracle_physics import channel_case
    channel_case(path, 0.7, engine=factory, end_time=30.)


def _open(kind, seconds):
    def case(path, factory):
        from test_oracle_physics import open_boundary_case
        open_boundary_case(path, kind, 0.7 if kind == 'channel' else 1.0, .4, engine=factory,
                           end_time=float(seconds))
    return case


def _workload(name):
    def case(path, factory):
        from nhflood.plain import PlainRun
        w = workload(name)
        run = PlainRun(w, factory)
        while not run.done:
            run.advance()
        run.engine.budget_flush()
        run.close()
    return case


def workload(name):
    """The three synthetic workloads, started wet so that water moves from
    the first step."""
    from nhflood import workloads
    if name == 'uniform_64':
        w = workloads.plain_uniform_256(n=64)
        w.duration = 300
        depth = np.full(w.mesh.e_num, 0.05, np.float32)
    elif name == 'quadtree_small':
        w = workloads.multires_quadtree(width=400.0, duration=60)
        w.yield_step = 20
        depth = np.where(w.mesh.land_type == 0, 1.5, 0.3).astype(np.float32)
    elif name == 'dambreak_48':
        w = workloads.dambreak(n=48, dx=1.0, duration=5)
        w.yield_step = 5
        return w
    else:
        raise KeyError(name)
    depth[0] = 0.0
    w.initial_depth = depth
    return w


CASES = {f'two_cell_{n}': _two_cell(n) for n in TWO_CELL}
CASES.update({
    'grid3_limiter_theta1': _grid3(1.0),
    'grid3_limiter_theta07': _grid3(0.7),
    'corner_extraction': _corner_extraction,
    'pressure_plane': _pressure('plane'),
    'pressure_dry_tangent': _pressure('dry_tangent'),
    'pressure_rotated_slope': _pressure('rotated'),
    'channel_theta07_30s': _channel,
    'open_channel_theta07_600s': _open('channel', 600),
    'tidal_basin_3600s': _open('tide', 3600),
    'uniform_64': _workload('uniform_64'),
    'quadtree_small': _workload('quadtree_small'),
    'dambreak_48': _workload('dambreak_48'),
})


def record_case(name: str, path: Path, factory) -> dict:
    """Run one case on engines from ``factory``; the recording of its solve."""
    make, made = recording(factory)
    CASES[name](Path(path), make)
    if len(made) != 1:
        raise RuntimeError(f'{name}: {len(made)} engines were built, expected one')
    return made[0].result()
