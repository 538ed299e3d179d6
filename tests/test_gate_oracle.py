"""Gate controller mechanism cases on the CPU restatement through the real
time loop: the known answers of the reference's tests/test_gate_solver.py
(bed motion, strict trigger, latching, independent gates, warmup, still
water, bitwise restart, exchange and source accounting, hanging faces,
limiter, replayed beds) and tests/test_gate_extended.py (large components,
paired uniform/hanging sections, the refined dry-channel transient, the
30,000 s command clock)."""
import csv
import functools

import numpy as np
import pytest

import nhflood.solver_compact as solver_compact
from gate_cases import event_steps, level_boundary, run, setup
from nhflood.engine import evolve
from nhflood.input import DomainConfig
from nhflood.output import read_bed_at, read_checkpoint, write_checkpoint


def gate_of(result):
    return result.manifest['gate_control']['gates'][0]


def pond_of(result):
    return result.manifest['gate_control']['pond_budget']


def test_local_bed_motion_preserves_water_and_drives_expected_exchange(tmp_path):
    """test_gate_solver.py:78-90: the first step moves the bed after its
    hydraulic substep; the next step feels the 0.1 m head."""
    dc, force, topo, depth, bed = setup(tmp_path, gate=dict(opening_seconds=.1))
    run(dc, force, .1)
    r = run(dc, force, .2, output=tmp_path / 'next', restart=tmp_path / 'out/output/state_final.fdb')
    internal = np.flatnonzero((topo[:, 1] > 0) & (topo[:, 2] > 0))
    assert r.state.q[internal[0]] * 10 == pytest.approx(.1962, rel=2e-5)
    assert np.sum(r.state.depth) * 100 == pytest.approx(600, abs=3e-5)
    assert r.state.depth[2] > r.state.depth[1]
    assert gate_of(r)['command_seconds'] == 0
    assert r.manifest['bed_events'] == []


@pytest.mark.parametrize('control_depth,threshold,expected', [(2, 1, 0), (2, 2, None), (0, -1, None),
                                                               (.001, -1, None), (2, 3, None)])
def test_strict_threshold_and_dry_control(tmp_path, control_depth, threshold, expected):
    dc, force, *_ = setup(tmp_path, depth=[control_depth, 0, 0], bed=[0, 10, 0], gate=dict(trigger_level=threshold))
    r = run(dc, force, .1)
    assert gate_of(r)['command_seconds'] == expected


def test_end_bed_and_pond_exchange_accounting(tmp_path):
    dc, force, topo, initial, bed = setup(tmp_path, depth=[2, 2, 1])
    r = run(dc, force, 3)
    gate, pond = gate_of(r), pond_of(r)
    assert r.state.bed[2] == pytest.approx(-.1)
    assert gate['pond_in_m3'] > 0
    assert gate['first_effective_flow_seconds'] is not None
    assert gate['fully_open_seconds'] == 1
    assert abs(pond['residual_m3']) < 3e-5
    assert pond['storage_m3'] - pond['initial_storage_m3'] == pytest.approx(
        gate['pond_net_m3'] + pond['rounding_m3'], abs=3e-5)
    np.testing.assert_array_equal(read_bed_at(tmp_path / 'out/output', 3), r.state.bed)


@pytest.mark.parametrize('batch_size,yield_step', [(1, 1), (32, 1), (32, 2)])
def test_short_pulse_latches_each_step_and_never_recloses(tmp_path, monkeypatch, batch_size, yield_step):
    monkeypatch.setattr(solver_compact, 'evolve', functools.partial(evolve, batch_size=batch_size))
    boundaries = level_boundary(tmp_path, [(0, 1), (.125, 2), (.25, 1), (3600, 1)])
    dc, force, *_ = setup(tmp_path, bed=[0, 10, 0], depth=[1, 0, 0],
                          gate=dict(trigger_level=1.5, opening_seconds=1.875, open_elevation=0),
                          boundaries=boundaries, yield_step=yield_step)
    r = run(dc, force, 2)
    gate = gate_of(r)
    assert gate['command_seconds'] == .125
    assert gate['fully_open_seconds'] == 2
    assert gate['first_fully_open_sample_seconds'] == 2
    assert r.state.bed[2] == 0
    assert abs(pond_of(r)['residual_m3']) < 1e-5


def test_gates_trigger_independently(tmp_path):
    dc, force, *_ = setup(tmp_path, cells=[(i * 10, (i + 1) * 10, 0, 10) for i in range(6)],
                          types=[1, 11, 10, 1, 11, 10], depth=[2, 0, 0, 0, 0, 0], bed=[0, 10, 0, 0, 10, 0],
                          gate=dict(gates=[dict(name='A', inside_point=(15, 5), control_point=(5, 5)),
                                           dict(name='B', inside_point=(45, 5), control_point=(35, 5))]))
    r = run(dc, force, 1)
    assert [g['command_seconds'] for g in r.manifest['gate_control']['gates']] == [0, None]
    assert r.state.bed[2] < 10 and r.state.bed[5] == 10


def test_warmup_disables_control_until_formal_zero(tmp_path):
    dc, force, *_ = setup(tmp_path, warmup=2, depth=[2, 0, 0], bed=[0, 10, 0])
    warming = run(dc, force, 0)
    assert gate_of(warming)['command_seconds'] is None
    formal = run(dc, force, 1, output=tmp_path / 'formal', restart=tmp_path / 'out/output/state_final.fdb')
    assert gate_of(formal)['command_seconds'] == 0
    assert formal.state.bed[2] == np.float32(-.1)


@pytest.mark.parametrize('moving', [False, True])
def test_fixed_still_water_and_uniform_motion_have_zero_flux(tmp_path, moving):
    dc, force, _, depth, bed = setup(
        tmp_path, cells=[(100, 110, 0, 10), (10, 20, 0, 10), (20, 30, 0, 10), (30, 40, 0, 10), (0, 10, 0, 10)],
        types=[1, 11, 11, 10, 1], bed=[0, 0, 0, 10, 10], depth=[2, 2, 2, 0, 0],
        gate=dict(trigger_level=1 if moving else 3))
    r = run(dc, force, 2)
    np.testing.assert_array_equal(r.state.depth, depth)
    assert np.all(r.state.q == 0)
    np.testing.assert_array_equal(r.state.bed[2:4], np.full(2, -.1 if moving else 0, dtype=np.float32))


@pytest.mark.parametrize('split_at', [1, 3, 5])
def test_restart_before_during_after_opening_is_bitwise(tmp_path, split_at):
    boundaries = level_boundary(tmp_path, [(0, 1), (1, 1), (2, 2), (3600, 2)])
    dc, force, *_ = setup(tmp_path, boundaries=boundaries, depth=[1, 0, 0], bed=[0, 3, 0],
                          gate=dict(trigger_level=1.5, opening_seconds=2))
    full = run(dc, force, 6)
    partial = run(dc, force, split_at, output=tmp_path / 'part')
    resumed = run(dc, force, 6, output=tmp_path / 'resumed', restart=tmp_path / 'part/output/state_final.fdb')
    for name in ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'first_time_hi',
                 'first_time_lo'):
        assert getattr(full.state, name).tobytes() == getattr(resumed.state, name).tobytes(), name
    assert full.state.metadata_json == resumed.state.metadata_json
    assert full.manifest['gate_control'] == resumed.manifest['gate_control']
    for t in (split_at, 6):
        np.testing.assert_array_equal(read_bed_at(tmp_path / 'out/output', t),
                                      read_bed_at(tmp_path / 'resumed/output', t))
    np.testing.assert_array_equal(read_bed_at(tmp_path / 'out/output', split_at), partial.state.bed)

    def rows(path):
        with path.open() as stream:
            return [r for r in csv.DictReader(stream) if float(r['elapsed_seconds']) > split_at]
    assert rows(tmp_path / 'out/gate_balance.csv') == rows(tmp_path / 'resumed/gate_balance.csv')


@pytest.mark.parametrize('pond_depth,gate_depth', [(0, 2), (2, .021), (1, 1.00001), (2, 1)])
def test_dry_near_dry_small_and_reverse_heads(tmp_path, pond_depth, gate_depth):
    dc, force, *_ = setup(tmp_path, depth=[gate_depth, gate_depth, pond_depth],
                          gate=dict(trigger_level=-1, open_elevation=0))
    r = run(dc, force, 2)
    gate = gate_of(r)
    assert np.all(r.state.depth >= 0)
    assert abs(pond_of(r)['residual_m3']) < 4e-5
    if gate_depth > pond_depth:
        assert gate['pond_in_m3'] > 0
    else:
        assert gate['pond_out_m3'] > 0


@pytest.mark.parametrize('pond_depth', [0, 2])
def test_hanging_subedges_have_one_shared_flux_and_new_bed_pressure(tmp_path, pond_depth):
    cells = [(100, 110, 0, 10), (0, 10, 0, 10), (10, 15, 0, 5), (10, 15, 5, 10), (15, 25, 0, 10)]
    dc, force, topo, depth, bed = setup(
        tmp_path, cells=cells, types=[1, 10, 11, 11, 1], depth=[2, pond_depth, 2, 2, 2],
        gate=dict(gates=[dict(name='A', inside_point=(12, 2), control_point=(105, 5))]))
    r = run(dc, force, 2)
    shared = (topo[:, 1] == 2) & np.isin(topo[:, 2], [3, 4])
    assert np.count_nonzero(shared) == 2
    assert np.all(r.state.q[shared] != 0)
    gate, pond = gate_of(r), pond_of(r)
    assert pond['storage_m3'] - pond['initial_storage_m3'] == pytest.approx(
        gate['pond_net_m3'] + pond['rounding_m3'], abs=2e-5)
    assert abs(pond['residual_m3']) < 2e-5
    assert r.state.bed[3] == np.float32(-.1)


def test_local_movement_response_converges_with_step_refinement(tmp_path):
    results = []
    for i, step in enumerate((.125, .0625, .03125)):
        path = tmp_path / str(i)
        dc, force, *_ = setup(path, gate=dict(opening_seconds=.5))
        force = force.model_copy(update={'rainfall': type(force.rainfall)(**event_steps(path, step, 1))})
        r = run(dc, force, 1)
        results.append(r.state.depth)
        assert np.sum(r.state.depth) * 100 == pytest.approx(600, abs=8e-5)
        assert abs(pond_of(r)['residual_m3']) < 2e-5
    assert np.linalg.norm(results[2] - results[1]) < np.linalg.norm(results[1] - results[0])


def test_multicell_dry_channel_wets_and_can_reverse(tmp_path):
    cells = [(i * 10, (i + 1) * 10, 0, 10) for i in range(5)]
    boundaries = level_boundary(tmp_path, [(0, 4), (30, 4), (31, 0), (3600, 0)])
    dc, force, *_ = setup(tmp_path, cells=cells, types=[1, 11, 11, 11, 10], bed=[0, 4, 4, 4, 0],
                          depth=[4, 0, 0, 0, 0], boundaries=boundaries,
                          gate=dict(open_elevation=0, opening_seconds=1))
    r = run(dc, force, 90)
    gate = gate_of(r)
    assert gate['pond_in_m3'] > 0 and gate['pond_out_m3'] > 0
    assert gate['river_in_m3'] > 0 and gate['river_out_m3'] > 0
    assert gate['first_effective_flow_seconds'] > gate['command_seconds']
    assert np.all(r.state.depth >= 0)
    assert abs(pond_of(r)['residual_m3']) < .002


def horton(dc, land_type):
    data = dc.model_dump()
    data['land_parameters'][land_type]['infiltration'] = dict(f0_mm_h=36, fc_mm_h=18, k_per_h=2)
    return DomainConfig.model_validate(data)


def test_pond_rain_infiltration_overtopping_and_roundoff_close(tmp_path):
    cells = [(i * 10, (i + 1) * 10, 0, 10) for i in range(4)]
    dc, force, *_ = setup(tmp_path, cells=cells, types=[1, 11, 10, 1], depth=[2, 2, 1, .5], rain=100,
                          gate=dict(open_elevation=0))
    r = run(horton(dc, 10), force, 4)
    pond = pond_of(r)
    assert pond['rain_m3'] > 0 and pond['infiltration_m3'] > 0
    assert pond['overtopping_out_m3'] > 0
    assert abs(pond['residual_m3']) < 2e-5


def test_limiter_records_actual_shared_flux_not_requested_flux(tmp_path):
    dc, force, topo, *_ = setup(tmp_path, depth=[.021, .021, 0], gate=dict(trigger_level=-1, open_elevation=0))
    seed = read_checkpoint(dc.restart_state)
    seed.q[:] = 0
    seed.q[np.flatnonzero((topo[:, 1] == 2) & (topo[:, 2] == 3))[0]] = 100
    seed.q[np.flatnonzero((topo[:, 1] == 1) & (topo[:, 2] == 2))[0]] = -100
    write_checkpoint(dc.restart_state, **vars(seed))
    r = run(dc.model_copy(update={'afa': 1.}), force, 1)
    gate, pond = gate_of(r), pond_of(r)
    assert r.manifest['limiter_activity']['limited_face_steps'] > 0
    assert gate['pond_in_m3'] <= .021 * 100 + 1e-6
    assert r.state.depth[3] * 100 == pytest.approx(gate['pond_net_m3'], abs=1e-6)
    assert abs(pond['residual_m3']) < 1e-6


def test_fractional_opening_replays_online_bed_bitwise(tmp_path):
    dc, force, *_ = setup(tmp_path, bed=[0, 10, 0], depth=[2, 0, 0], gate=dict(opening_seconds=7, open_elevation=1.3))
    r = run(dc, force, 1.25)
    assert read_bed_at(tmp_path / 'out/output', 1.25).tobytes() == r.state.bed.tobytes()


def test_pond_level_reservoir_accounts_for_overwritten_negative_depth(tmp_path):
    boundaries = level_boundary(tmp_path, [(0, .01), (3600, .01)], line=((30, 0), (30, 10)))
    dc, force, topo, *_ = setup(tmp_path, boundaries=boundaries, depth=[2, 2, .01])
    seed = read_checkpoint(dc.restart_state)
    seed.q[np.flatnonzero((topo[:, 1] == 2) & (topo[:, 2] == 3))[0]] = -100
    write_checkpoint(dc.restart_state, **vars(seed))
    r = run(dc, force, .125)
    pond = pond_of(r)
    assert r.state.depth[3] == np.float32(.01)
    assert gate_of(r)['pond_out_m3'] > 1
    assert pond['boundary_m3'] > 1
    assert pond['positivity_m3'] == 0
    assert abs(pond['residual_m3']) < 3e-5


def test_cold_warmup_initialization_preserves_closed_gate_barrier(tmp_path):
    boundaries = level_boundary(tmp_path, [(0, 2), (3600, 2)])
    dc, force, *_ = setup(tmp_path, boundaries=boundaries, warmup=2, bed=[0, 10, 0], depth=[0, 0, 0])
    r = run(dc.model_copy(update={'restart_state': ''}), force, 0)
    assert r.manifest['initialization']['method'] == 'connected_still_water'
    assert gate_of(r)['command_seconds'] is None
    assert r.state.bed[2] == 10
    assert r.state.depth[1] == 2 and np.all(r.state.depth[2:] == 0)


@pytest.mark.parametrize('pond_type', [10, 7])
def test_configurable_pond_and_channel_source_budgets_close(tmp_path, pond_type):
    boundaries = level_boundary(tmp_path, [(0, .01), (3600, .01)], line=((10, 10), (20, 10)),
                                name='gate_supply', kind='discharge')
    dc, force, *_ = setup(tmp_path, boundaries=boundaries, types=[1, 11, pond_type], depth=[2, 2, 1], rain=100,
                          gate=dict(pond_land_type=pond_type, open_elevation=0))
    r = run(horton(dc, 11), force, 4)
    control = r.manifest['gate_control']
    channel = control['gates'][0]['channel_budget']
    assert control['pond_land_type'] == pond_type
    assert channel['rain_m3'] > 0 and channel['infiltration_m3'] > 0
    assert channel['boundary_m3'] == pytest.approx(.04, abs=3e-8)
    assert channel['initial_storage_m3'] == 200
    assert channel['storage_m3'] == float(r.state.depth[2]) * 100
    assert abs(channel['residual_m3']) < 3e-5
    assert abs(control['pond_budget']['residual_m3']) < 3e-5
    rows = list(csv.DictReader((tmp_path / 'out/gate_balance.csv').open()))
    final = next(row for row in reversed(rows) if row['region'] == 'A')
    assert float(final['residual_m3']) == channel['residual_m3']
    assert float(final['river_net_m3']) == channel['river_net_m3']


def assert_control_volume(budget, *, scale=1.):
    terms = ('initial_storage_m3', 'storage_m3', 'rain_m3', 'infiltration_m3', 'positivity_m3', 'pipe_m3',
             'boundary_m3', 'rounding_m3', 'residual_m3')
    assert all(np.isfinite(budget[key]) for key in terms)
    assert abs(budget['residual_m3']) <= max(2e-4, 2e-6 * scale)


def large_components(path):
    """Seven separate 25 x 20 gate channels of 4 m cells between a river row
    and a pond row (tests/test_gate_extended.py:45-60)."""
    cells, types, bed, depth, gates = [], [], [], [], []
    for group in range(7):
        y = group * 100
        for row in range(22):
            for col in range(25):
                x, bottom = 4 * col, y + 4 * row
                cells.append((x, x + 4, bottom, bottom + 4))
                types.append(1 if row == 0 else 10 if row == 21 else 11)
                bed.append(0. if row in (0, 21) else 1.)
                depth.append(2. if row == 0 else .3 if row == 21 else .2)
        gates.append(dict(name=f'G{group}', inside_point=(2, y + 6), control_point=(2, y + 2)))
    return setup(path, cells=cells, types=types, bed=bed, depth=depth,
                 gate=dict(gates=gates, opening_seconds=.25, trigger_level=1., open_elevation=0., pond_land_type=10))


def test_seven_large_components_open_and_close_each_control_volume(tmp_path):
    dc, force, topo, initial, _ = large_components(tmp_path)
    r = run(dc, force, .5)
    report = r.manifest['gate_control']
    gates = report['gates']
    assert len(gates) == 7
    assert sum(len(g['cell_ids']) for g in gates) == 3500
    assert len(topo) // 256 >= 7
    assert [g['command_seconds'] for g in gates] == [0.] * 7
    assert [g['fully_open_seconds'] for g in gates] == [.25] * 7
    assert all(g['pond_in_m3'] > 0 and g['river_in_m3'] > 0 for g in gates)
    assert np.all(r.state.depth >= 0)
    assert all(r.state.bed[np.asarray(g['cell_ids'], dtype=int)].max() == 0 for g in gates)
    area = np.r_[0., np.full(7 * 550, 16.)]
    initial_storage = float(np.dot(initial.astype(float), area))
    final_storage = float(np.dot(r.state.depth.astype(float), area))
    global_budget = r.manifest['mass_balance_final']
    assert final_storage - initial_storage == pytest.approx(
        global_budget['storage_m3'] - global_budget['initial_storage_m3'], abs=.02)
    assert abs(global_budget['residual_m3']) < .05
    assert_control_volume(report['pond_budget'], scale=initial_storage)
    for gate in gates:
        channel = gate['channel_budget']
        assert_control_volume(channel, scale=channel['initial_storage_m3'])
        expected = (channel['river_net_m3'] - channel['pond_net_m3'] + channel['rain_m3']
                    - channel['infiltration_m3'] + channel['positivity_m3'] + channel['pipe_m3']
                    + channel['boundary_m3'] + channel['rounding_m3'])
        assert channel['storage_m3'] - channel['initial_storage_m3'] == pytest.approx(
            expected + channel['residual_m3'], abs=.003)
        assert channel['pond_net_m3'] == pytest.approx(gate['pond_net_m3'], abs=1e-5)


def test_disabled_gate_runs_without_controller_and_keeps_identity(tmp_path):
    dc, force, *_ = setup(tmp_path, depth=[2, 0, 0], bed=[0, 10, 0], gate=dict(enabled=False))
    r = run(dc, force, 1)
    assert 'gate_control' not in r.manifest
    assert r.manifest['gate_cell_count'] == 1
    assert r.state.bed[2] == 10
    assert not r.state.gate_open


def paired_section(path, *, hanging, regime):
    """The same 8 m river-to-pond section with one whole pond face or two
    split ones (tests/test_gate_extended.py:63-83)."""
    cells, types = [(0, 8, 0, 8), (8, 16, 0, 8)], [1, 11]
    if hanging:
        cells += [(x, x + 4, y, y + 4) for x in (16, 20) for y in (0, 4)]
        types += [10] * 4
    else:
        cells.append((16, 24, 0, 8))
        types.append(10)
    rest = len(cells) - 2
    beds = [0., .1] + [0.] * rest
    depths = [1.0001, .9] + [1.] * rest if regime == 'near_balance' else [2., .05] + [0.] * rest
    return setup(path, cells=cells, types=types, bed=beds, depth=depths,
                 gate=dict(gates=[dict(name='A', inside_point=(12, 2), control_point=(4, 2))], opening_seconds=.25,
                           trigger_level=.5, open_elevation=0., pond_land_type=10))


@pytest.mark.parametrize('regime', ['near_balance', 'dry_wet'])
def test_uniform_and_hanging_section_agree_on_width_and_cumulative_flow(tmp_path, regime):
    """tests/test_gate_extended.py:132-193: one shared 8 m face, whole or
    split; the first step's exchange follows the head jump over the centre
    distance (8 m, or 6 m to the split cells' centres), the second step
    continues from the half-open bed."""
    observations = []
    for hanging in (False, True):
        path = tmp_path / ('hanging' if hanging else 'uniform')
        dc, force, topo, *_ = paired_section(path, hanging=hanging, regime=regime)
        r = run(dc, force, .125)
        gate, pond = gate_of(r), pond_of(r)
        assert_control_volume(pond, scale=100.)
        assert_control_volume(gate['channel_budget'], scale=100.)
        interface = (topo[:, 1] == 2) & (topo[:, 2] > 2)
        assert np.count_nonzero(interface) == (2 if hanging else 1)
        lengths = np.full(np.count_nonzero(interface), 4. if hanging else 8.)
        width_flow = float(np.dot(r.state.q[interface], lengths))
        first_net = gate['pond_net_m3']
        pond_cells = topo[interface, 2]
        left_eta = float(r.state.bed[2]) + float(r.state.depth[2])
        right_eta = r.state.bed[pond_cells].astype(float) + r.state.depth[pond_cells].astype(float)
        face_depth = np.maximum(left_eta, right_eta) - np.maximum(float(r.state.bed[2]),
                                                                  r.state.bed[pond_cells].astype(float))
        distance = 6. if hanging else 8.
        expected_q = r.state.q[interface].astype(float) - 9.81 * face_depth * (right_eta - left_eta) / distance * .125
        nxt = run(dc, force, .25, output=path / 'next', restart=path / 'out/output/state_final.fdb')
        np.testing.assert_allclose(nxt.state.q[interface], expected_q, rtol=3e-5, atol=2e-8)
        second = gate_of(nxt)['pond_net_m3'] - first_net
        assert second == pytest.approx(float(np.dot(expected_q, lengths)) * .125, rel=3e-5, abs=2e-8)
        assert nxt.state.bed[2] == 0.
        observations.append(dict(width_flow=width_flow, pond_net=gate['pond_net_m3'],
                                 river_net=gate['channel_budget']['river_net_m3'], pond_storage=pond['storage_m3'],
                                 channel_storage=gate['channel_budget']['storage_m3'], distance=distance))
    uniform, hanging = observations
    if regime == 'dry_wet':
        for o in observations:
            expected = 9.81 * .05 * .15 / o['distance'] * .125 * 8.
            assert o['width_flow'] == pytest.approx(expected, rel=2e-5)
            assert o['pond_net'] == pytest.approx(expected * .125, rel=2e-5)
            assert o['pond_storage'] == pytest.approx(o['pond_net'], abs=2e-5)
        assert hanging['width_flow'] / uniform['width_flow'] == pytest.approx(4 / 3, rel=2e-5)
        assert hanging['river_net'] == pytest.approx(uniform['river_net'], rel=2e-5)
    else:
        keys = ('width_flow', 'pond_net', 'river_net', 'pond_storage', 'channel_storage')
        np.testing.assert_allclose([uniform[k] for k in keys], [hanging[k] for k in keys], rtol=2e-3, atol=2e-4)


@pytest.mark.parametrize('opening_seconds', [1800., 3600.])
def test_formal_30000s_command_and_f32_opening_age(tmp_path, opening_seconds):
    """tests/test_gate_extended.py:227-274: the trigger check and the F32
    opening age at clock words 30,000 s in, by setting the clock directly."""
    from engine import OracleEngine
    from nhflood.forcing import Forcing
    from nhflood.gate import GateController, GateLayout
    from nhflood.geometry import MeshGeometry
    from nhflood.model import StepParams, build_step_arrays
    from nhflood.preprocess import load_mesh, preprocess
    from nhflood.clock import seconds_to_ticks, words
    cells = [(4, 8, 0, 4), (0, 4, 0, 4), (8, 12, 0, 4)]  # gate, control (river), pond
    dc, force, *_ = setup(tmp_path, cells=cells, types=[11, 1, 10], bed=[8, 0, 0], depth=[0, 0, 0],
                          gate=dict(trigger_level=1., opening_seconds=opening_seconds, open_elevation=0.,
                                    gates=[dict(name='A', inside_point=(6., 2.), control_point=(2., 2.))]))
    preprocess(dc, force)
    mesh, flags = load_mesh(dc)
    geometry = MeshGeometry.from_mesh(mesh)
    forcing = Forcing.load(dc, force, geometry)
    arrays = build_step_arrays(mesh, flags, geometry, forcing, dc.land_parameters, dc.sita)
    layout = GateLayout.load(force.gate, geometry.bounds, mesh.land_type, mesh.topology, forcing.boundaries,
                             arrays.bed)
    assert layout.cell_gate.tolist() == [-1, 0, -1, -1] and layout.controls.tolist() == [2]
    controller = GateController.build(force.gate, layout, arrays.bed, mesh.land_type, mesh.topology, 0.)
    arrays.gate = controller.tables
    eng = OracleEngine(arrays, StepParams(min_h=1e-5))
    eng.initialize()
    eng.set('bed', np.array([0, 8, 0, 0], np.float32))
    fractional_age = np.float32(1.234567)
    fractional_bed = np.float32(8. - 8. * np.float32(fractional_age / np.float32(opening_seconds)))
    for seconds, expected in ((29999., None), (30000., 8.), (30001.234567, fractional_bed),
                              (30000. + opening_seconds / 4, 6.), (30000. + opening_seconds / 2, 4.),
                              (30000. + opening_seconds, 0.)):
        if seconds == 30000.:
            eng.set('depth', np.array([0, 0, 2, 0], np.float32))
        eng.set_clock(words(seconds_to_ticks(seconds)))
        eng.set_active(1)
        eng.gate_check()
        state = eng.gate_state()
        assert state['commanded'][0] == int(expected is not None)
        if expected is not None:
            assert eng.get('bed')[1] == pytest.approx(expected, abs=2e-6)
    controller.state = eng.gate_state()
    controller.initialize_inventory(eng.get('depth'), np.array([0., 16., 16., 16.]))
    report = controller.report(eng.get('depth'), np.array([0., 16., 16., 16.]), 30000. + opening_seconds)['gates'][0]
    assert report['command_seconds'] == 30000.
    assert report['scheduled_fully_open_seconds'] == 30000. + opening_seconds
    assert report['fully_open_seconds'] == 30000. + opening_seconds
    assert report['first_fully_open_sample_seconds'] == 30000. + opening_seconds
    assert report['command_clock_ticks'] == words(seconds_to_ticks(30000.)).tolist()
    eng.close()


def test_disabled_and_never_triggered_gates_leave_the_step_bitwise_unchanged(tmp_path):
    """tests/test_gate_compatibility.py's invariant: the controller changes
    nothing of the hydraulics until a gate is commanded; a disabled block, an
    enabled block whose trigger is never reached, and no gate block give
    identical states and traces."""
    import json as _json
    from nhflood.input import ForceConfig
    results = {}
    for name, gate in (('none', None), ('disabled', dict(enabled=False)), ('idle', dict(trigger_level=1000.))):
        dc, force, *_ = setup(tmp_path / name, depth=[2, 2, 1], rain=50, gate=gate or {})
        if gate is None:
            force = ForceConfig(boundaries=force.boundaries, rainfall=force.rainfall, gate=None)
            seed = read_checkpoint(dc.restart_state)
            meta = _json.loads(seed.metadata_json)
            meta['gate_config'] = 'null'
            seed.metadata_json = _json.dumps(meta)
            write_checkpoint(dc.restart_state, **vars(seed))
        results[name] = run(dc, force, 3)
    base = results['none']
    for name in ('disabled', 'idle'):
        r = results[name]
        np.testing.assert_array_equal(base.trace, r.trace)
        for field in ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed'):
            assert getattr(base.state, field).tobytes() == getattr(r.state, field).tobytes(), (name, field)
    assert gate_of(results['idle'])['command_seconds'] is None


def test_dry_multicell_transient_refines_first_water_volume_and_oscillation(tmp_path):
    """A river cell 4 m deep beside a dry four-cell gate channel (bed 2 m,
    opening to 0 m in 0.5 s) and a dry pond cell, for 16 s at step limits of
    1/8, 1/16 and 1/32 s (tests/test_gate_extended.py:86-94,197-225): both
    control volumes close, water first reaches the pond no later at the
    finest step, and the pond volumes and the oscillation of the per-second
    pond exchange converge."""
    cells = [(4 * i, 4 * (i + 1), 0, 4) for i in range(6)]
    measurements = []
    for step in (.125, .0625, .03125):
        path = tmp_path / str(step)
        dc, force, *_ = setup(path, cells=cells, types=[1, 11, 11, 11, 11, 10], bed=[0., 2., 2., 2., 2., 0.],
                              depth=[4., 0., 0., 0., 0., 0.],
                              gate=dict(gates=[dict(name='A', inside_point=(6, 2), control_point=(2, 2))],
                                        opening_seconds=.5, trigger_level=1., open_elevation=0.,
                                        pond_land_type=10))
        force = force.model_copy(update={'rainfall': type(force.rainfall)(**event_steps(path, step, 16., 24, 4))})
        r = run(dc, force, 16.)
        gate, pond = gate_of(r), pond_of(r)
        assert_control_volume(pond, scale=100.)
        assert_control_volume(gate['channel_budget'], scale=100.)
        assert np.all(r.state.depth >= 0)
        assert gate['first_effective_flow_seconds'] is not None
        rows = [row for row in csv.DictReader((path / 'out/gate_balance.csv').open()) if row['region'] == 'A']
        cumulative = np.array([float(row['pond_net_m3']) for row in rows])
        measurements.append(dict(first_water_s=gate['first_effective_flow_seconds'], pond_in_m3=gate['pond_in_m3'],
                                 pond_out_m3=gate['pond_out_m3'],
                                 oscillation_m3=float(np.sum(np.abs(np.diff(np.diff(cumulative)))))))
    coarse, middle, fine = measurements
    assert fine['first_water_s'] <= coarse['first_water_s'] + .5
    for key in ('pond_in_m3', 'pond_out_m3', 'oscillation_m3'):
        assert np.isfinite([m[key] for m in measurements]).all()
        assert abs(fine[key] - middle[key]) <= abs(middle[key] - coarse[key]) + .02
    assert fine['pond_in_m3'] > 0
