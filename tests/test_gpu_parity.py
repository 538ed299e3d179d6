"""CUDA step vs the CPU restatement, through the C ABI, bit for bit.

Both engines run the same time loop on the same inputs. The bar is
bit-exact: every trace row (dt bits, clock words, status, CFL candidate,
event flag, limiter counts, minimum donor scale, wet-cell count), every
state array at the end, the budget and step-statistics CSV files. Float
arithmetic is deterministic on both sides (same F32 operation order, no
contraction, FP64 budget partials in a fixed tree, order-free min/count
reductions), so any difference is a defect.
"""
import filecmp

import numpy as np
import pytest

from runner import run
from scenarios import (all_cells_filtered, domain, grid3_mesh, grid_cell, grid_horizontal, grid_vertical,
                       seed_checkpoint, two_cell_case)

pytestmark = pytest.mark.gpu

STATE = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'first_time_hi', 'first_time_lo')


def assert_runs_identical(a, b):
    assert a.trace.shape == b.trace.shape
    np.testing.assert_array_equal(a.trace, b.trace)
    for name in STATE:
        x, y = getattr(a.state, name), getattr(b.state, name)
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32), err_msg=name)
    for rel in ('mass_balance.csv', 'step_statistics.csv'):
        assert filecmp.cmp(a.path / rel, b.path / rel, shallow=False), rel
    assert a.manifest['dt_sequence_sha256'] == b.manifest['dt_sequence_sha256']


CASES = {
    'closed_basin': dict(bands=[[6, 6]], duration=60, q=.1, connected=True),
    'horton_late': dict(bands=[[100, 0], [0, 100]], duration=120, land_type=1,
                        infiltration=dict(f0_mm_h=76.2, fc_mm_h=2.54, k_per_h=2)),
    'warmup_level_discharge': dict(bands=[[6, 6]], duration=60, q=.01, warmup=20, level=.1,
                                   level_rows=[(0, .1), (60, .2)], q_rows=[(0, .01), (60, .03)], yield_step=10),
    'negative_discharge': dict(bands=[[6, 6]], duration=60, q=-10.),
    'level_knot': dict(bands=[[0, 0]], duration=1, level=0., level_rows=[(0, 0.), (.000002, 1.), (1, 0.)]),
    'cfl_after_level': dict(bands=[[0, 0]], duration=1, connected=True, level=0,
                            level_rows=[(0, 0), (.000002, 100), (1, 100)]),
    'small_rain_high_bed': dict(bands=[[.01, .01]], duration=60, bed=100.),
}


def cuda_engine(path):
    """'auto': the form chosen for the mesh (the lattice form on uniform
    grids of at least 2^20 cells, else the fused tiled step, which keeps the
    CFL in the step on these small meshes); 'pass': the fused tiled step with
    the separate CFL pass; 'multipass': the reference's pass structure."""
    def factory(arrays, params):
        from nhflood.native import CudaEngine
        params.path = {'multipass': 'multipass', 'pass': 'tiled'}.get(path, 'auto')
        params.cfl = 'pass' if path == 'pass' else 'auto'
        engine = CudaEngine(arrays, params)
        want = ('multipass',) if path == 'multipass' else ('tiled',) if path == 'pass' else ('tiled', 'lattice')
        assert engine.path.startswith(want), engine.path
        if path == 'pass':
            assert 'cfl=pass' in engine.path, engine.path
        return engine
    return factory


PATHS = ['auto', 'pass', 'multipass']


@pytest.mark.parametrize('path', PATHS)
@pytest.mark.parametrize('name', sorted(CASES))
def test_two_cell_cases_bit_exact(tmp_path, cuda_available, name, path):
    kw = dict(CASES[name])
    bands, duration = kw.pop('bands'), kw.pop('duration')
    dc, fc = two_cell_case(tmp_path / 'oracle', bands, duration, **kw)
    a = run(dc, fc, 'oracle')
    dc, fc = two_cell_case(tmp_path / 'cuda', bands, duration, **kw)
    b = run(dc, fc, cuda_engine(path))
    assert b.manifest['backend'] == 'cuda'
    assert_runs_identical(a, b)


@pytest.mark.parametrize('path', PATHS)
@pytest.mark.parametrize('sita', [1.0, 0.7])
def test_grid_with_limiter_and_theta_bit_exact(tmp_path, cuda_available, sita, path):
    results = []
    for engine in ('oracle', cuda_engine(path)):
        name = 'oracle' if engine == 'oracle' else 'cuda'
        path_dir = tmp_path / name
        path_dir.mkdir()
        grid3_mesh(path_dir)
        from scenarios import write_rain
        from nhflood.raster import from_origin
        from nhflood.input import ForceConfig
        rain = write_rain(path_dir, [[[0]]], from_origin(0, 30, 30, 30), [(0, 20)])
        q = np.zeros(25, np.float32)
        for side, value in {grid_vertical(1, 1): -1, grid_vertical(1, 2): 1,
                            grid_horizontal(1, 1): -1, grid_horizontal(2, 1): 1}.items():
            q[side] = value
        depth = np.zeros(10, np.float32)
        depth[grid_cell(1, 1)] = .1
        seed = seed_checkpoint(path_dir / 'seed.fdb', path_dir / 'ne.txt', path_dir / 'ns.txt', depth=depth, q=q)
        dc = domain(path_dir, duration=20, yield_step=5, restart=seed, sita=sita,
                    land={10: dict(manning_n=1e-3, infiltration='none')})
        fc = ForceConfig(boundaries=[], rainfall=rain)
        results.append(run(dc, fc, engine))
    assert_runs_identical(*results)
    assert results[1].manifest['limiter_activity']['limited_cell_steps'] > 0


@pytest.mark.parametrize('path', PATHS)
def test_plain_uniform_256_full_run_bit_exact(tmp_path, cuda_available, path):
    """The 65,536-cell plain configuration for its whole 3600 s: identical
    dt sequences and per-step wet counts; every 300 s frame identical."""
    from nhflood.output import list_depth_frames, read_depth_frame
    from nhflood.workloads import plain_uniform_256, simulate
    from runner import oracle_factory
    w = plain_uniform_256()
    row_a, rec_a = simulate(w, tmp_path / 'oracle', engine_factory=oracle_factory)
    row_b, rec_b = simulate(w, tmp_path / 'cuda', engine_factory=cuda_engine(path))
    assert rec_b.data['backend'] == 'cuda'
    np.testing.assert_array_equal(rec_a.trace, rec_b.trace)
    assert rec_a.trace[:, 9].max() > 1000  # the run does flood
    fa = list_depth_frames(tmp_path / 'oracle' / 'output')
    fb = list_depth_frames(tmp_path / 'cuda' / 'output')
    assert [s for s, _ in fa] == [s for s, _ in fb]
    for (_, pa), (_, pb) in zip(fa, fb):
        np.testing.assert_array_equal(read_depth_frame(pa).view(np.uint32), read_depth_frame(pb).view(np.uint32))
    assert row_a == row_b


@pytest.mark.parametrize('path', PATHS)
def test_multires_quadtree_bit_exact(tmp_path, cuda_available, path):
    """2:1 quadtree (20/10/5 m) with hanging-edge pressure reconstruction,
    Horton infiltration, moving rain and a tidal level boundary, started wet
    so that water crosses the resolution interfaces from the first step."""
    from nhflood.output import list_depth_frames, read_depth_frame
    from nhflood.workloads import multires_quadtree, simulate
    from runner import oracle_factory
    w = multires_quadtree(width=2000.0, duration=600)
    depth = np.where(w.mesh.land_type == 0, 1.5, 0.3).astype(np.float32)
    depth[0] = 0.0
    w.initial_depth = depth
    assert w.step_arrays().hang_cells > 1000
    row_a, rec_a = simulate(w, tmp_path / 'oracle', engine_factory=oracle_factory)
    row_b, rec_b = simulate(w, tmp_path / 'cuda', engine_factory=cuda_engine(path))
    np.testing.assert_array_equal(rec_a.trace, rec_b.trace)
    assert rec_a.trace[:, 6].sum() >= 0 and rec_a.trace[:, 9].min() > 1000
    for (_, pa), (_, pb) in zip(list_depth_frames(tmp_path / 'oracle' / 'output'),
                                list_depth_frames(tmp_path / 'cuda' / 'output')):
        np.testing.assert_array_equal(read_depth_frame(pa).view(np.uint32), read_depth_frame(pb).view(np.uint32))
    assert row_a == row_b


@pytest.mark.parametrize('path', PATHS)
def test_six_boundaries_use_the_wide_budget_bit_exact(tmp_path, cuda_available, path):
    """4 + 6 x 6 = 40 budget terms (more than the 32-term mask of the fused
    step): three level and three discharge boundaries on a 24 x 4 strip."""
    from nhflood.input import ForceConfig
    from nhflood.raster import from_origin
    from scenarios import strip_grid_mesh, write_line, write_rain, write_series
    results = []
    for engine in ('oracle', cuda_engine(path)):
        d = tmp_path / ('oracle' if engine == 'oracle' else 'cuda')
        d.mkdir()
        strip_grid_mesh(d, 24, 4, 10)
        rain = write_rain(d, [[[20.]], [[0.]]], from_origin(0, 40, 240, 40), [(0, 150), (150, 300)])
        boundaries = []
        for k in range(3):
            boundaries.append(dict(name=f'q{k}', kind='discharge',
                                   line=write_line(d / f'q{k}.geojson', [[80 * k + 5, 0], [80 * k + 35, 0]]),
                                   series=write_series(d / f'q{k}.csv', [(0, .5 + k), (300, .2)])))
            boundaries.append(dict(name=f'h{k}', kind='level',
                                   line=write_line(d / f'h{k}.geojson', [[80 * k + 5, 40], [80 * k + 35, 40]]),
                                   series=write_series(d / f'h{k}.csv', [(0, .3 * k), (300, .1)])))
        dc = domain(d, duration=300, yield_step=60)
        results.append(run(dc, ForceConfig(boundaries=boundaries, rainfall=rain), engine))
    assert_runs_identical(*results)
    assert results[0].manifest["steps"] > 100 and sum(k.startswith("level:") for k in results[0].budget) == 3


@pytest.mark.parametrize('cfl', ['fused', 'pass'])
def test_tile_1024_both_cfl_forms_bit_exact(cuda_available, cfl):
    """The 1024-cell tiles (512 threads, two cells per thread) in both CFL
    forms on the 65,536-cell configuration: 40 batches from t = 0, traces and
    every state array identical to the oracle after each batch."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / 'oracle'))
    from engine import OracleEngine
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    from nhflood.workloads import plain_uniform_256

    def cuda(arrays, params):
        params.path, params.cfl = 'tile1024', cfl
        engine = CudaEngine(arrays, params)
        assert engine.path.startswith('tiled(tile=1024') and f'cfl={cfl}' in engine.path, engine.path
        return engine

    w = plain_uniform_256()
    runs = [PlainRun(w, lambda a, p: OracleEngine(a, p)), PlainRun(w, cuda)]
    for _ in range(40):
        rows = []
        for r in runs:
            tw, ow = r.begin()
            rows.append(r.engine.run_batch(tw, ow))
            r.finish(rows[-1])
        np.testing.assert_array_equal(rows[0], rows[1])
        for name in STATE_F32 + STATE_U32:
            assert runs[0].engine.get(name).tobytes() == runs[1].engine.get(name).tobytes(), name
    assert runs[1].elapsed > 0
    for r in runs:
        r.close()


@pytest.mark.parametrize('rows,blocks', [(None, None), ('4', '2'), ('7', '4'), ('16', '3')])
def test_lattice_march_with_horton_rain_and_level_bit_exact(cuda_available, monkeypatch, rows, blocks):
    """The lattice form on a 90 x 90 grid (strips of 28 columns and chunks
    that do not divide it) with Horton infiltration on one land class, rain,
    a level boundary and a 1 m wet start (donor limiting, flows
    across strip and chunk edges): rows per chunk and resident blocks per
    SM forced through the planner's knobs, so that strip and chunk edges
    (whose CFL sides the close pass takes) cut through the wet area. Traces
    and every state array equal the oracle's after each of 30 batches."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / 'oracle'))
    from engine import OracleEngine
    from nhflood.input import HortonInfiltration, LandParameters
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    from nhflood.workloads import plain_uniform_256
    for key, value in (('NHF_LATTICE_ROWS', rows), ('NHF_LATTICE_BLOCKS', blocks)):
        if value is None:
            monkeypatch.delenv(key, raising=False)
        else:
            monkeypatch.setenv(key, value)

    def cuda(arrays, params):
        params.path = 'lattice'
        engine = CudaEngine(arrays, params)
        assert engine.path.startswith('lattice(90x90'), engine.path
        if rows:
            assert f'rows={rows},' in engine.path and f'blocks={blocks})' in engine.path, engine.path
        return engine

    w = plain_uniform_256(n=90)
    w.land_parameters[1] = LandParameters(manning_n=0.03, infiltration=HortonInfiltration(
        f0_mm_h=60.0, fc_mm_h=10.0, k_per_h=4.0))
    depth = np.full(w.mesh.e_num, 1.0, np.float32)
    depth[0] = 0.0
    w.initial_depth = depth
    runs = [PlainRun(w, lambda a, p: OracleEngine(a, p)), PlainRun(w, cuda)]
    try:
        for _ in range(30):
            out = []
            for r in runs:
                tw, ow = r.begin()
                out.append(r.engine.run_batch(tw, ow))
                r.finish(out[-1])
            np.testing.assert_array_equal(out[0], out[1])
            for name in STATE_F32 + STATE_U32:
                assert runs[0].engine.get(name).tobytes() == runs[1].engine.get(name).tobytes(), name
        np.testing.assert_array_equal(runs[0].engine.budget_flush(), runs[1].engine.budget_flush())
        assert (runs[1].engine.get('infiltration') > 0).any()
    finally:
        for r in runs:
            r.close()


@pytest.mark.parametrize('name,batches,path', [('multires_quadtree', 2, 'auto'), ('multires_quadtree_4m', 1, 'auto'),
                                               ('dambreak_4096', 1, 'pass'), ('dambreak_4096', 2, 'auto')])
def test_full_size_configurations_bit_exact(cuda_available, name, batches, path):
    """The bench's full-size meshes, 1,362,175 quadtree cells (20 km, 2:1,
    hanging edges), the 4.0 M-cell quadtree (36.6 km) and 16,777,216
    dam-break cells (33.5 M sides, 1024-cell tiles, the separate CFL pass):
    the first 32-step batches on the fused step as planned for the mesh and
    on the CPU restatement give identical trace rows, state arrays and
    budget totals."""
    from lockstep import FIELDS
    from nhflood.plain import PlainRun
    from nhflood.workloads import dambreak, multires_quadtree, multires_quadtree_4m
    from runner import oracle_factory
    workload = {'multires_quadtree': multires_quadtree, 'multires_quadtree_4m': multires_quadtree_4m,
                'dambreak_4096': dambreak}[name]()
    runs = [PlainRun(workload, factory, batch_size=32) for factory in (oracle_factory, cuda_engine(path))]
    try:
        form = runs[1].engine.path
        assert form.startswith('lattice') if name.startswith('dambreak') and path == 'auto' else 'cfl=pass' in form, form
        for _ in range(batches):
            rows = []
            for run in runs:
                target, origin = run.begin()
                rows.append(run.engine.run_batch(target, origin))
                run.finish(rows[-1])
            np.testing.assert_array_equal(rows[0], rows[1])
            assert (rows[0][:, 3] == 1).all()  # every step completed
        for field in FIELDS:
            a, b = (run.engine.get(field) for run in runs)
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32), err_msg=field)
        np.testing.assert_array_equal(runs[0].engine.budget_flush(), runs[1].engine.budget_flush())
    finally:
        for run in runs:
            run.close()


def test_mesh_without_cells_runs_like_the_oracle(tmp_path, cuda_available):
    """Every cell filtered out: the engine takes the multi-pass step (no
    tiles to plan) and runs the same ten empty steps as the oracle."""
    from nhflood.native import CudaEngine
    paths = []

    def factory(arrays, params):
        engine = CudaEngine(arrays, params)
        paths.append(engine.path)
        return engine
    results = [run(*all_cells_filtered(tmp_path / name), engine)
               for name, engine in (('oracle', 'oracle'), ('cuda', factory))]
    assert paths == ['multipass (mesh has no cells)']
    assert_runs_identical(*results)
    assert results[0].manifest['steps'] == 10 and len(results[0].state.depth) == 1
