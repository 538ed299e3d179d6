"""Known answers of the reference's physics tests, restated on the CPU
restatement of the step (the oracle): donor-factor positivity
(tests/test_positivity.py:116-160), hanging-interface pressure
reconstruction (tests/test_pressure_gradient.py:98-151), the coarse/fine
channel's steady uniform flow (tests/test_face_flux.py:245-271), and the
open boundaries' steady channel outflow and tidal basin
(tests/test_open_boundary.py:208-262). The meshes
and seed states are rebuilt here from the reference tests' descriptions; the
tolerances are the reference's."""
import csv
from pathlib import Path

import numpy as np
import pytest

from nhflood.geometry import hanging_geometry
from nhflood.input import ForceConfig
from nhflood.raster import from_origin
from runner import run
from scenarios import (channel_cells, domain, grid3_mesh, grid_cell, grid_horizontal, grid_vertical,
                       rectangles_mesh, seed_checkpoint, write_line, write_rain, write_series)


# ---------------------------------------------------------------- positivity

def positivity_case(path: Path, *, wet_cell, face_flows, extraction=False, engine='oracle'):
    path.mkdir(parents=True)
    grid3_mesh(path)
    rain = write_rain(path, [[[0]]], from_origin(0, 30, 30, 30), [(0, 1)])
    depth = np.zeros(10, np.float32)
    depth[wet_cell] = np.float32(.1)  # 100 m2 x 0.1 m = 10 m3
    q = np.zeros(25, np.float32)
    for side, value in face_flows.items():
        q[side] = value
    seed = seed_checkpoint(path / 'seed.fdb', path / 'ne.txt', path / 'ns.txt', depth=depth, q=q)
    boundaries = []
    if extraction:
        boundaries.append(dict(name='river', kind='discharge', line=write_line(path / 'river.geojson', [[0, 0], [0, 10]]),
                               series=write_series(path / 'river.csv', [(0, -100), (1, -100)])))
    dc = domain(path, duration=1, yield_step=1, restart=seed, sita=1,
                land={10: dict(manning_n=1e-6, infiltration='none')})
    return run(dc, ForceConfig(boundaries=boundaries, rainfall=rain), engine)


def test_four_outgoing_faces_share_one_cell_inventory(tmp_path):
    first_cfl = .5 * 10 / (np.sqrt(9.81 * .1) + 1 / .1)
    assert 4 * 10 * first_cfl > 10  # unscaled faces would carry more than the cell holds
    r = positivity_case(tmp_path / 'center', wet_cell=grid_cell(1, 1), face_flows={
        grid_vertical(1, 1): -1, grid_vertical(1, 2): 1, grid_horizontal(1, 1): -1, grid_horizontal(2, 1): 1})
    depth = r.state.depth
    neighbours = depth[[grid_cell(1, 0), grid_cell(1, 2), grid_cell(0, 1), grid_cell(2, 1)]]
    assert np.all(depth >= 0) and np.all(neighbours > 0)
    np.testing.assert_allclose(neighbours, neighbours[0], rtol=0, atol=2e-7)
    b = r.budget
    assert b['initial_storage_m3'] == pytest.approx(10)
    assert b['storage_m3'] == pytest.approx(10, abs=1e-5)
    assert b['rainfall_m3'] == b['infiltration_m3'] == 0
    assert b['bed_clamp_nonlevel_m3'] <= 1e-5
    assert abs(b['residual_m3']) <= 1e-5
    assert r.manifest['steps'] >= 2
    activity = r.manifest['limiter_activity']
    assert activity['limited_cell_steps'] > 0 and activity['limited_face_steps'] >= 4
    assert 0 <= activity['minimum_donor_scale'] < 1
    rows = list(csv.DictReader((r.path / 'step_statistics.csv').open()))
    assert sum(int(x['limited_cell_steps']) for x in rows) == activity['limited_cell_steps']
    assert sum(int(x['limited_face_steps']) for x in rows) == activity['limited_face_steps']
    assert min(float(x['minimum_donor_scale']) for x in rows) == activity['minimum_donor_scale']


def test_negative_discharge_and_faces_share_corner_inventory(tmp_path):
    r = positivity_case(tmp_path / 'corner', wet_cell=grid_cell(0, 0),
                        face_flows={grid_vertical(0, 1): 1, grid_horizontal(1, 0): 1}, extraction=True)
    depth = r.state.depth
    assert np.all(depth >= 0)
    assert depth[grid_cell(0, 1)] > 0 and depth[grid_cell(1, 0)] > 0
    b = r.budget
    assert b['requested_discharge:river_m3'] == pytest.approx(-100)
    assert -10 < b['discharge:river_m3'] < 0
    assert b['storage_m3'] > 0
    assert b['bed_clamp_nonlevel_m3'] <= 1e-5
    assert abs(b['residual_m3']) <= 1e-5


# ---------------------------------------------------- pressure reconstruction

def strip_cells(rotated=False):
    """Three 8 m cells beside six 4 m cells (a 2:1 interface along one axis)."""
    cells = [(0, 8, y, y + 8) for y in range(0, 24, 8)] + [(8, 12, y, y + 4) for y in range(0, 24, 4)]
    return [(c, d, a, b) for a, b, c, d in cells] if rotated else cells


def evolve(path: Path, cells, bed_at, depth_at, seconds=.125, engine='oracle'):
    path.mkdir(parents=True, exist_ok=True)
    xy = np.array([(0, 0)] + [((a + b) / 2, (c + d) / 2) for a, b, c, d in cells], np.float32)
    bed = np.r_[0, [bed_at(x, y, i) for i, (x, y) in enumerate(xy[1:], 1)]].astype(np.float32)
    topo, side_xy = rectangles_mesh(path, cells, bed)
    depth = np.r_[0, [depth_at(x, y, bed[i], i) for i, (x, y) in enumerate(xy[1:], 1)]].astype(np.float32)
    seed = seed_checkpoint(path / 'seed.fdb', path / 'ne.txt', path / 'ns.txt', depth=depth, bed=bed)
    x1, y1 = max(c[1] for c in cells), max(c[3] for c in cells)
    rain = write_rain(path, [[[0]]], from_origin(0, y1, x1, y1), [(0, 3600)])
    dc = domain(path, duration=max(1, int(seconds)), restart=seed)
    r = run(dc, ForceConfig(boundaries=[], rainfall=rain), engine, end_time=seconds)
    return r.state, depth, xy, topo.astype(np.int32), side_xy.astype(np.float32)


@pytest.mark.parametrize('rotated', [False, True])
def test_linear_tangential_surface_has_only_roundoff_crossflow(tmp_path, rotated):
    axis = 0 if rotated else 1
    state, _, xy, topo, side_xy = evolve(tmp_path, strip_cells(rotated), lambda x, y, i: .001 * (x if rotated else y),
                                         lambda x, y, z, i: 1.)
    interface = (topo[:, 0] == (1 if rotated else 2)) & (topo[:, 1] != 0) & (topo[:, 2] != 0)
    assert np.max(np.abs(state.q[interface])) < 3e-7
    assert .001 / 3 * 9.81 * .125 > 1000 * np.max(np.abs(state.q[interface]))
    layout = hanging_geometry(xy[:, 0], xy[:, 1], side_xy[:, 0], side_xy[:, 1], topo)
    np.testing.assert_array_equal(layout.cells, [1, 2, 3])
    assert len(layout.offsets) == 6
    np.testing.assert_array_equal(layout.axes[:, axis], 1)
    np.testing.assert_array_equal(layout.axes[:, 1 - axis], 0)


@pytest.mark.parametrize('rotated', [False, True])
def test_variable_bed_still_water_is_bitwise_unchanged(tmp_path, rotated):
    state, initial, *_ = evolve(tmp_path, strip_cells(rotated), lambda x, y, i: ((i % 7) - 3) * .125,
                                lambda x, y, z, i: 2. - z, seconds=60.)
    np.testing.assert_array_equal(state.depth.view(np.uint32), initial.view(np.uint32))
    assert np.all(state.q == 0.)


@pytest.mark.parametrize('dry_cells', [(1,), (3,), (3, .02), (1, 3)])
def test_dry_tangent_neighbours_use_one_side_or_zero(tmp_path, dry_cells):
    threshold = dry_cells == (3, .02)
    unavailable = (3,) if threshold else dry_cells
    state, _, _, topo, _ = evolve(tmp_path, strip_cells(), lambda x, y, i: .001 * y,
                                  lambda x, y, z, i: (.02 if threshold else 0.) if i in unavailable else 1.)
    middle = (topo[:, 0] == 2) & (topo[:, 1] == 2)
    if len(unavailable) == 1:
        assert np.max(np.abs(state.q[middle])) < 3e-7
    else:
        np.testing.assert_allclose(np.sort(state.q[middle]), [-.00040875, .00040875], atol=3e-7, rtol=0)


def test_one_cell_caches_both_axes_and_reconstructs_linear_plane(tmp_path):
    cells = [(0, 8, 0, 8), (8, 12, 0, 4), (8, 12, 4, 8), (0, 4, 8, 12), (4, 8, 8, 12), (8, 12, 8, 12)]
    a, b = .0013, -.0007
    state, _, xy, topo, side_xy = evolve(tmp_path, cells, lambda x, y, i: a * x + b * y, lambda x, y, z, i: 1.)
    layout = hanging_geometry(xy[:, 0], xy[:, 1], side_xy[:, 0], side_xy[:, 1], topo)
    np.testing.assert_array_equal(layout.cells, [1])
    np.testing.assert_array_equal(layout.axes, [[1, 1]])
    edges = layout.edge_index >= 0
    expected = -9.81 * .125 * np.where(topo[edges, 0] == 2, a, b)
    np.testing.assert_allclose(state.q[edges], expected, atol=3e-7, rtol=0)


# ------------------------------------------------- coarse/fine channel flow

def channel_case(path: Path, theta: float, engine='oracle', end_time=None):
    path.mkdir(parents=True)
    cells = channel_cells()
    bed = np.r_[0, [10 - .002 * (x0 + x1) / 2 for x0, x1, _, _ in cells]].astype(np.float32)
    rectangles_mesh(path, cells, bed)
    duration = 4000
    expected_q = np.sqrt(.002) / .03
    rain = write_rain(path, [[[0]]], from_origin(0, 2, 1024, 2), [(0, duration)])
    boundaries = []
    for name, x, value, kind in (('upstream', 0, 2 * expected_q, 'discharge'),
                                 ('downstream', 1024, float(bed[-1] + 1), 'level')):
        boundaries.append(dict(name=name, kind=kind, line=write_line(path / f'{name}.geojson', [[x, .1], [x, 1.9]]),
                               series=write_series(path / f'{name}.csv', [(0, value), (duration, value)])))
    depth = np.ones(len(cells) + 1, np.float32)
    depth[0] = 0
    seed = seed_checkpoint(path / 'seed.fdb', path / 'ne.txt', path / 'ns.txt', depth=depth, bed=bed)
    sampled = [(i, c) for i, c in enumerate(cells, 1) if c == (510, 512, 0, 2) or c[:2] == (512, 513)]
    stations = {str(i): ((x0 + x1) / 2, (y0 + y1) / 2) for i, (x0, x1, y0, y1) in sampled}
    dc = domain(path, duration=duration, yield_step=300, restart=seed, stations=stations, sita=theta)
    r = run(dc, ForceConfig(boundaries=boundaries, rainfall=rain), engine, end_time=end_time)
    samples = list(csv.DictReader((Path(dc.output_dir) / 'stations.csv').open(newline='')))
    return cells, r, samples


@pytest.mark.parametrize('theta', [0.7, 1.0])
def test_coarse_fine_channel_reaches_continuous_steady_flow(tmp_path, theta):
    cells, r, samples = channel_case(tmp_path / f'theta_{theta}', theta)
    coarse = next(i for i, c in enumerate(cells, 1) if c == (510, 512, 0, 2))
    fine = [i for i, c in enumerate(cells, 1) if c[:2] == (512, 513)]
    predicted = np.sqrt(.002) / .03  # H^(5/3) sqrt(S) / n with H = 1 m
    times = sorted({float(s['elapsed_seconds']) for s in samples})[-4:-1]
    history = []
    depth_at = {}
    for t in times:
        row = {int(s['cell_id']): s for s in samples if float(s['elapsed_seconds']) == t}
        q_coarse = float(row[coarse]['depth']) * float(row[coarse]['u'])
        q_fine = sum(float(row[i]['depth']) * float(row[i]['u']) for i in fine) / 2
        history.append((q_coarse, q_fine))
        depth_at[t] = (float(row[coarse]['depth']), [float(row[i]['depth']) for i in fine])
    q_coarse, q_fine = history[-1]
    dc, dfine = depth_at[times[-1]]
    interface = (dc + sum(dfine) / 2) / 2
    assert q_coarse == pytest.approx(predicted, rel=2e-3)
    assert q_fine == pytest.approx(predicted, rel=2e-3)
    assert q_coarse == pytest.approx(q_fine, rel=1e-4)
    assert max(np.ptp([h[j] for h in history]) for j in (0, 1)) < 1e-4
    assert interface == pytest.approx(1, abs=.02)
    b = r.budget
    assert abs(b['residual_m3']) / (b['initial_storage_m3'] + b['discharge:upstream_m3']) < 1e-4


# ----------------------------------------------------------- open boundaries

PERIOD = 86_400


def open_boundary_case(path: Path, kind: str, theta: float, afa: float, engine='oracle', end_time=None):
    """A flat 40 x 2 strip: a channel between a 10 m3/s inflow and a 1 m level
    (10 m cells, 6000 s), or a basin driven by a daily 1 m tide at its west
    edge (100 m cells, two days); tests/test_open_boundary.py:135-205."""
    from scenarios import strip_grid_mesh
    path.mkdir(parents=True)
    nx, ny = 40, 2
    dx = 10 if kind == 'channel' else 100
    duration = 6_000 if kind == 'channel' else 2 * PERIOD
    strip_grid_mesh(path, nx, ny, dx)
    rain = write_rain(path, [[[0]]], from_origin(0, ny * dx, nx * dx, ny * dx), [(0, duration)])
    definitions = ([('upstream', 'discharge', 0, 10.), ('downstream', 'level', nx * dx, 1.)]
                   if kind == 'channel' else [('sea', 'level', 0, None)])
    boundaries = []
    for name, bkind, x, constant in definitions:
        if constant is not None:
            rows = [(0, constant), (duration, constant)]
        else:
            rows = [(s, 3 + np.sin(2 * np.pi * s / PERIOD)) for s in range(0, duration + 300, 300)]
        boundaries.append(dict(name=name, kind=bkind, line=write_line(path / f'{name}.geojson', [[x, .1], [x, ny * dx - .1]]),
                               series=write_series(path / f'{name}.csv', rows)))
    depth = np.r_[0., np.full(nx * ny, 1. if kind == 'channel' else 3.)].astype(np.float32)
    seed = seed_checkpoint(path / 'seed.fdb', path / 'ne.txt', path / 'ns.txt', depth=depth)
    dc = domain(path, duration=duration, yield_step=500 if kind == 'channel' else 600, restart=seed,
                sita=theta, afa=afa)
    r = run(dc, ForceConfig(boundaries=boundaries, rainfall=rain), engine, end_time=end_time)
    from nhflood.output import list_depth_frames
    return r, list_depth_frames(dc.output_dir), nx, ny, Path(dc.output_dir)


def test_open_channel_steady_profile_is_stable_across_theta_and_time_step(tmp_path):
    from nhflood.output import read_bed_at, read_depth_frame
    profiles = []
    for theta in (1., .7):
        for afa in (.4, .1):
            r, frames, nx, ny, out = open_boundary_case(tmp_path / f'ch_{theta}_{afa}', 'channel', theta, afa)
            eta = [(read_bed_at(out, s) + read_depth_frame(f))[1:].reshape(ny, nx) for s, f in frames[-3:]]
            profile = eta[-1].mean(axis=0)
            profiles.append(profile)
            assert abs(profile[0] - profile[1]) < .005
            assert abs(profile[-2] - profile[-1]) < .005
            assert np.max(np.abs(eta[-1] - eta[-2])) < 2e-4
            rows = list(csv.DictReader((r.path / 'mass_balance.csv').open()))
            outflow = [-(float(b['level:downstream_m3']) - float(a['level:downstream_m3']))
                       / (float(b['elapsed_seconds']) - float(a['elapsed_seconds']))
                       for a, b in zip(rows[-3:-1], rows[-2:])]
            assert all(abs(q - 10.) < .01 for q in outflow), (theta, afa, outflow)
            b = r.budget
            assert abs(b['residual_m3']) / (b['initial_storage_m3'] + b['discharge:upstream_m3']) < 1e-4
    assert np.ptp(np.stack(profiles), axis=0).max() < 2e-4


def test_tidal_basin_keeps_amplitude_and_phase_across_time_steps(tmp_path):
    from nhflood.output import read_depth_frame
    metrics = []
    omega = 2 * np.pi / PERIOD
    for afa in (.04, .015):
        _, frames, nx, _, _ = open_boundary_case(tmp_path / f'tide_{afa}', 'tide', .7, afa)
        t = np.array([s for s, _ in frames], float)
        y = np.array([float(read_depth_frame(f)[nx]) for _, f in frames])
        last = t >= PERIOD
        t, y = t[last], y[last]
        basis = np.column_stack([np.sin(omega * t), np.cos(omega * t), np.ones(len(t)), (t - t.mean()) / PERIOD])
        sine, cosine, _, _ = np.linalg.lstsq(basis, y, rcond=None)[0]
        amplitude = float(np.hypot(sine, cosine))
        phase_minutes = float(np.arctan2(-cosine, sine) / omega / 60)
        metrics.append((amplitude, phase_minutes))
        assert abs(amplitude - 1.) < .01
        assert abs(phase_minutes) < 2.
    assert abs(metrics[0][0] - metrics[1][0]) < .002
    assert abs(metrics[0][1] - metrics[1][1]) < .1


# ------------------------------------------------------ inventory rounding

def test_transport_and_small_rain_have_one_inventory_rounding(tmp_path):
    """Rain and the face transport join before the one F32 rounding of the
    depth (tests/test_inventory_rounding.py:19-54)."""
    from scenarios import two_cell_mesh
    two_cell_mesh(tmp_path, connected=True)
    mm = np.float32(1.4911491234670393e-5)
    rain = write_rain(tmp_path, [[[mm, 0]]], from_origin(0, 10, 10, 10), [(0, 1)])
    depth = np.array([0, .5, .4], np.float32)
    seed = seed_checkpoint(tmp_path / 'seed.fdb', tmp_path / 'ne.txt', tmp_path / 'ns.txt', depth=depth)
    r = run(domain(tmp_path, duration=1, restart=seed), ForceConfig(boundaries=[], rainfall=rain), 'oracle')
    assert r.manifest['steps'] == 1
    rain_rate = float(np.float32(float(mm) * .001))
    ideal = float(depth[1]) - float(r.state.q[2]) * 10 / 100 + rain_rate
    assert abs(float(r.state.depth[1]) - ideal) < .55 * float(np.spacing(np.float32(ideal)))
