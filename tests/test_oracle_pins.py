"""Pin the CPU restatement to the reference tests' known answers.

Each case rebuilds a fixture of the reference test it names
(tests/test_solver_forcing.py, test_positivity.py, test_inventory_rounding.py)
and runs the full time loop on the oracle engine; the assertions and
tolerances are the reference's own.
"""
import csv

import numpy as np
import pytest

from runner import run
from scenarios import all_cells_filtered, two_cell_case

ORACLE = 'oracle'


def test_next_cfl_uses_depth_after_the_level_update(tmp_path):
    # test_solver_forcing.py:23-46
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 1, connected=True, level=0,
                           level_rows=[(0, 0), (.000002, 100), (1, 100)])
    res = run(dc, fc, ORACLE)
    rows = res.trace[res.trace[:, 3] == 1]
    candidates = rows[:, 4].copy().view(np.float32)
    assert candidates[1] == pytest.approx(.5 * 10 / np.sqrt(9.81 * 100), rel=2e-7)
    assert candidates[1] < 1
    stats = list(csv.DictReader((tmp_path / 'out/step_statistics.csv').open()))
    last = stats[-1]
    assert float(last['face_depth_m']) == max(float(last['lower_depth_m']), float(last['higher_depth_m']))
    expected = .5 * 10 / (np.sqrt(9.81 * float(last['face_depth_m'])) + abs(float(last['face_velocity_m_s'])))
    assert float(last['cfl_min_s']) == pytest.approx(expected, rel=2e-7)


def test_all_event_steps_have_explicit_standard_statistics(tmp_path):
    # test_solver_forcing.py:49-61
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 1, q=.1, q_rows=[(0, .1), (.000002, .1), (1, .1)])
    run(dc, fc, ORACLE)
    last = list(csv.DictReader((tmp_path / 'out/step_statistics.csv').open()))[-1]
    assert last['steps'] == last['event_short_steps'] == '2'
    assert last['standard_steps'] == '0'
    for name in ['standard_dt_min_s', 'standard_dt_max_s', 'standard_dt_mean_s']:
        assert last[name] == ''
    assert float(last['event_dt_min_s']) == pytest.approx(.000002)
    assert float(last['event_dt_sum_s']) == pytest.approx(1., abs=1e-7)


def test_closed_basin_rain_and_discharge_balance(tmp_path):
    # test_solver_forcing.py:125-134
    dc, fc = two_cell_case(tmp_path, [[6, 6]], 60, q=.1, connected=True)
    res = run(dc, fc, ORACLE)
    r = res.budget
    assert r['rainfall_m3'] == pytest.approx(1.2, abs=1e-8)
    assert r['discharge:river_m3'] == pytest.approx(6., abs=1e-7)
    assert abs(r['residual_m3']) / 7.2 < 1e-4
    assert r['storage_m3'] == pytest.approx(7.2, rel=1e-4)
    assert np.all(np.isfinite(res.h))
    assert res.manifest['status'] == 'completed' and res.manifest['steps'] >= 60
    assert len(res.manifest['input_sha256']) == 6


def test_horton_clocks_are_local(tmp_path):
    # test_solver_forcing.py:137-144
    horton = dict(f0_mm_h=76.2, fc_mm_h=2.54, k_per_h=2)
    dc, fc = two_cell_case(tmp_path / 'late', [[100, 0], [0, 100]], 120, land_type=1, infiltration=horton)
    late = run(dc, fc, ORACLE)
    dc, fc = two_cell_case(tmp_path / 'reference', [[0, 100]], 60, land_type=1, infiltration=horton)
    ref = run(dc, fc, ORACLE)
    assert late.h[2] == pytest.approx(ref.h[2], abs=1e-6)


def test_actual_infiltration_is_bounded_by_water(tmp_path):
    # test_solver_forcing.py:147-153
    dc, fc = two_cell_case(tmp_path, [[.001, .001]], 60, land_type=6,
                           infiltration=dict(f0_mm_h=101.6, fc_mm_h=7.62, k_per_h=2))
    res = run(dc, fc, ORACLE)
    assert res.budget['infiltration_m3'] == pytest.approx(res.budget['rainfall_m3'], rel=2e-6)
    assert res.budget['bed_clamp_nonlevel_m3'] == 0
    assert res.budget['bed_clamp_level_m3'] == 0
    assert np.max(res.h) == 0


def test_configured_constant_horton_capacity_changes_actual_infiltration(tmp_path):
    # test_solver_forcing.py:156-164
    out = {}
    for name, inf in (('high', dict(f0_mm_h=36, fc_mm_h=36, k_per_h=0)),
                      ('low', dict(f0_mm_h=18, fc_mm_h=18, k_per_h=0)), ('none', 'none')):
        dc, fc = two_cell_case(tmp_path / name, [[100, 100]], 60, infiltration=inf)
        out[name] = run(dc, fc, ORACLE).budget
    assert out['high']['infiltration_m3'] == pytest.approx(.12, rel=1e-4)
    assert out['low']['infiltration_m3'] == pytest.approx(.06, rel=1e-4)
    assert out['none']['infiltration_m3'] == 0.


def test_warmup_holds_boundaries_and_has_no_rain(tmp_path):
    # test_solver_forcing.py:167-179
    dc, fc = two_cell_case(tmp_path, [[6, 6]], 60, q=.01, warmup=20, level=.1,
                           level_rows=[(0, .1), (60, .2)], q_rows=[(0, .01), (60, .03)], yield_step=10)
    res = run(dc, fc, ORACLE)
    rows = list(csv.DictReader((tmp_path / 'out/mass_balance.csv').open()))
    at_start = next(r for r in rows if float(r['elapsed_seconds']) == 0)
    assert float(at_start['rainfall_m3']) == 0
    assert float(at_start['discharge:river_m3']) == pytest.approx(.2)
    assert res.budget['rainfall_m3'] == pytest.approx(1.2)
    assert res.budget['discharge:river_m3'] == pytest.approx(1.4)
    assert [float(r['elapsed_seconds']) for r in rows if r['phase'] == 'warmup'] == [-20., -10.]
    from nhflood.output import read_checkpoint
    state = read_checkpoint(tmp_path / 'out/output/state_start.fdb')
    assert state.depth[2] == pytest.approx(.1)
    assert abs(res.budget['relative_residual']) < 1e-4


@pytest.mark.parametrize('bed,land_type', [(-5., 10), (1., 8)])
def test_cold_start_is_dry_without_boundaries(tmp_path, bed, land_type):
    # test_solver_forcing.py:182-187
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 2, bed=bed, land_type=land_type)
    res = run(dc, fc, ORACLE)
    assert res.budget['initial_storage_m3'] == 0.
    assert res.budget['storage_m3'] == 0.
    np.testing.assert_array_equal(res.h[1:], [bed, bed])


def test_warmup_only_stops_at_start_and_outputs_each_interval(tmp_path):
    # test_solver_forcing.py:190-202
    dc, fc = two_cell_case(tmp_path, [[6, 6]], 60, q=.01, warmup=20, level=.1, yield_step=10)
    res = run(dc, fc, ORACLE, warmup_only=True)
    rows = list(csv.DictReader((tmp_path / 'out/mass_balance.csv').open()))
    assert [float(r['elapsed_seconds']) for r in rows] == [-20., -10., 0.]
    assert all(r['phase'] == 'warmup' for r in rows)
    assert res.budget['rainfall_m3'] == 0.
    assert res.budget['discharge:river_m3'] == pytest.approx(.2)
    assert res.manifest['run_kind'] == 'warmup'
    assert res.manifest['dt_seconds']['sum'] == pytest.approx(20.)
    assert res.manifest['simulation_end'] == dc.start.isoformat()
    assert sorted(p.stem for p in (tmp_path / 'out/output/frames').glob('*.fdb')) == ['depth_-20', 'depth_0']
    assert (tmp_path / 'out/output/state_final.fdb').exists()


def test_small_rain_is_retained_above_large_bed(tmp_path):
    # test_solver_forcing.py:205-209
    dc, fc = two_cell_case(tmp_path, [[.01, .01]], 60, bed=100.)
    res = run(dc, fc, ORACLE)
    assert res.budget['storage_m3'] == pytest.approx(.002, rel=2e-6)
    assert abs(res.budget['residual_m3']) < 4e-9


def test_level_accounts_for_small_rain_at_high_bed(tmp_path):
    # test_solver_forcing.py:252-255
    dc, fc = two_cell_case(tmp_path, [[0, .01]], 60, bed=99., level=100.)
    res = run(dc, fc, ORACLE)
    assert abs(res.budget['residual_m3']) < 1e-8
    assert res.budget['level:sea_m3'] == pytest.approx(100. - .001, abs=1e-8)


def test_level_below_bed_is_zero_depth_and_closes_budget(tmp_path):
    # test_solver_forcing.py:258-264
    dc, fc = two_cell_case(tmp_path, [[0, .01]], 60, bed=100., level=50.)
    res = run(dc, fc, ORACLE)
    assert res.budget['storage_m3'] == 0.
    assert res.budget['bed_clamp_nonlevel_m3'] == 0.
    assert res.budget['bed_clamp_level_m3'] == 0.
    assert res.budget['rainfall_m3'] == pytest.approx(.001, abs=1e-10)
    assert abs(res.budget['residual_m3']) < 1e-7


def test_negative_discharge_shares_available_water_without_creating_water(tmp_path):
    # test_solver_forcing.py:354-360
    dc, fc = two_cell_case(tmp_path, [[6, 6]], 60, q=-10.)
    r = run(dc, fc, ORACLE).budget
    assert r['discharge:river_m3'] == pytest.approx(-.6, abs=2e-6)
    assert r['requested_discharge:river_m3'] == pytest.approx(-600.)
    assert r['storage_m3'] == pytest.approx(.6, abs=2e-6)
    assert r['bed_clamp_nonlevel_m3'] < 1e-6
    assert abs(r['residual_m3']) < 2e-6


def test_horton_uses_f0_on_wet_cell_before_any_rain(tmp_path):
    # test_solver_forcing.py:363-366
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 60, level=.1, infiltration=dict(f0_mm_h=76.2, fc_mm_h=2.54, k_per_h=2))
    r = run(dc, fc, ORACLE).budget
    assert r['infiltration_m3'] == pytest.approx(76.2 / 1000 / 3600 * 100 * 60, rel=2e-6)


def test_true_small_cfl_stops_with_limiting_edge_diagnostics(tmp_path):
    # test_solver_forcing.py:369-371
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 1, level=1e9, connected=True)
    with pytest.raises(RuntimeError, match=r'CFL.*edge=2, cells=\[1, 2\].*depth_m=.*velocity_m_s='):
        run(dc, fc, ORACLE)


def test_subsecond_rain_knot_selects_the_next_band(tmp_path):
    # test_solver_forcing.py:374-389
    from datetime import timedelta
    from scenarios import START, domain
    from nhflood.input import ForceConfig
    path = tmp_path / 'rain_knot'
    two_cell_case(path, [[1, 0], [0, 2]], 2)
    (path / 'intervals.csv').write_text(
        'interval_start,interval_end\n'
        f'{START.isoformat()},{(START + timedelta(microseconds=2)).isoformat()}\n'
        f'{(START + timedelta(microseconds=2)).isoformat()},{(START + timedelta(seconds=1)).isoformat()}\n')
    dc = domain(path, duration=1, yield_step=1, out='knot_out')
    fc = ForceConfig(boundaries=[], rainfall=dict(raster=str(path / 'rain.tif'), intervals=str(path / 'intervals.csv')))
    res = run(dc, fc, ORACLE)
    np.testing.assert_allclose(res.state.depth[1:], [.001, .002], rtol=2e-6, atol=0)
    assert res.budget['storage_m3'] == pytest.approx(.3, rel=2e-6)


def test_subsecond_level_knot_and_between_frame_peak(tmp_path):
    # test_solver_forcing.py:392-402
    from nhflood.output import list_depth_frames, read_depth_frame, read_extrema
    dc, fc = two_cell_case(tmp_path, [[0, 0]], 1, level=0., level_rows=[(0, 0.), (.000002, 1.), (1, 0.)])
    res = run(dc, fc, ORACLE)
    assert abs(res.h[2]) < 2e-6
    root = tmp_path / 'out/output'
    extrema = read_extrema(root / 'extrema.fdb')
    assert extrema.max_depth[2] == pytest.approx(1., abs=2e-6)
    assert all(read_depth_frame(p)[2] < 2e-6 for _, p in list_depth_frames(root))
    peak = (int(extrema.first_time_hi[2]) * 2 ** 32 + int(extrema.first_time_lo[2])) / 2 ** 40
    assert peak == pytest.approx(.000002, abs=5e-13)


def test_mesh_without_cells_runs_with_zero_storage(tmp_path):
    """Every cell filtered out (z = -9999): the reference's loops run over
    empty ranges, so the run completes at dt = 1 s with nothing stored."""
    r = run(*all_cells_filtered(tmp_path), 'oracle')
    assert r.manifest['steps'] == 10 and r.manifest['status'] == 'completed'
    assert len(r.state.depth) == 1
    assert r.budget['storage_m3'] == 0 and r.budget['residual_m3'] == 0
