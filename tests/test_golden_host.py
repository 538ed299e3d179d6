"""Golden vectors from the reference's own code. tests/golden/make_golden.py
ran nh-flood-2d's preprocess/hydraulics.py, preprocess/gate.py and
input/*.py, and the plain-Python definitions of core/clock.py (tick
conversion, batch begin and trace read-back), core/pressure.py (hanging_geometry), preprocess/domain.py
(_filter_ne_ns), preprocess/force.py (TimeSeries, RainField),
core/run_record.py (WaterBudget), core/gate.py (GateController.report,
append_gate_balance) and core/output.py (array rules, station rows) on
seeded meshes, configs and controller states. Every case is replayed
through nhflood: arrays must match bit for bit, errors by message, configs
by acceptance, error locations and the validated dump, CSV files byte for
byte."""
import json
from datetime import datetime, timedelta, timezone
from pathlib import Path
from types import SimpleNamespace as NS

import numpy as np
import pytest
from pydantic import ValidationError

from nhflood.clock import seconds_to_ticks, words
from nhflood.forcing import RainField, TimeSeries
from nhflood.gate import GateController, GateLayout, append_gate_balance
from nhflood.geometry import (connected_still_water, hanging_geometry, map_land_parameters,
                              open_boundary_face_fractions)
from nhflood.input import DomainConfig, ForceConfig, LandParameters, absolute_time
from nhflood.preprocess import filter_ne_ns
from nhflood.run_record import WaterBudget

GOLDEN = Path(__file__).parent / 'golden'
CASES = json.loads((GOLDEN / 'host_golden.json').read_text())
ARRAYS = np.load(GOLDEN / 'host_golden.npz')
MESH = {key[5:]: ARRAYS[key] for key in ARRAYS.files if key.startswith('mesh_')}
ORIGIN = datetime(2023, 9, 7, 8, tzinfo=timezone.utc)


def same_bits(actual, expected):
    actual, expected = np.asarray(actual), np.asarray(expected)
    assert actual.dtype == expected.dtype and actual.shape == expected.shape
    np.testing.assert_array_equal(actual.view(np.uint8), expected.view(np.uint8))


@pytest.mark.parametrize('case', range(len(CASES['land'])))
def test_land_parameters_match_the_reference(case):
    spec = CASES['land'][case]
    table = {int(k): LandParameters.model_validate(v) for k, v in spec['table'].items()}
    types_ = ARRAYS[f'land{case}_types']
    if spec['error'] is not None:
        with pytest.raises(ValueError) as error:
            map_land_parameters(table, types_, MESH['topology'])
        assert str(error.value) == spec['error']
        return
    for name, value in zip(('side_n', 'f0', 'fc', 'k'), map_land_parameters(table, types_, MESH['topology'])):
        same_bits(value, ARRAYS[f'land{case}_{name}'])


@pytest.mark.parametrize('case', CASES['faces'])
def test_open_face_fractions_match_the_reference(case):
    result = open_boundary_face_fractions(ARRAYS[f'faces{case}_selected'], MESH['length'], MESH['topology'],
                                          MESH['face_ptr'], MESH['face_count'], MESH['flat'])
    same_bits(result, ARRAYS[f'faces{case}_result'])


def boundary(spec):
    return NS(name=spec['name'], kind=spec['kind'], cells=np.asarray(spec['cells'], dtype=np.int64),
              series=NS(at=lambda t, v=spec['level']: v))


@pytest.mark.parametrize('case', range(len(CASES['still'])))
def test_still_water_fill_matches_the_reference(case):
    spec = CASES['still'][case]
    args = (ARRAYS[f'still{case}_bed'], ARRAYS[f'still{case}_crest'], ARRAYS[f'still{case}_closed'],
            MESH['topology'], [boundary(b) for b in spec['boundaries']], MESH['area'])
    if spec['error'] is not None:
        with pytest.raises(ValueError) as error:
            connected_still_water(*args)
        assert str(error.value) == spec['error']
        return
    depth, meta = connected_still_water(*args)
    same_bits(depth, ARRAYS[f'still{case}_depth'])
    assert meta == spec['meta']


def check_gate_layout(spec, prefix):
    types_ = ARRAYS[f'{prefix}_types'].copy()
    if spec['overlap']:
        types_[types_ == spec['land_type']] = spec['pond_land_type']
    config = NS(land_type=spec['land_type'], pond_land_type=spec['pond_land_type'],
                open_elevation=spec['open_elevation'],
                gates=[NS(name=g['name'], inside_point=tuple(g['inside_point']),
                          control_point=tuple(g['control_point'])) for g in spec['gates']])
    boundaries = [NS(kind='level', cells=np.asarray(cells, dtype=np.int64)) for cells in spec['level_cells']]
    args = (config, ARRAYS[f'{prefix}_bounds'], types_, ARRAYS[f'{prefix}_topology'], boundaries,
            ARRAYS[f'{prefix}_bed'])
    if spec['error'] is not None:
        with pytest.raises(ValueError) as error:
            GateLayout.load(*args)
        assert str(error.value) == spec['error']
        return
    layout = GateLayout.load(*args)
    assert layout.cell_gate.tolist() == spec['cell_gate']
    assert layout.controls.tolist() == spec['controls']
    assert [c.tolist() for c in layout.cells] == spec['cells']


@pytest.mark.parametrize('case', range(len(CASES['gate'])))
def test_gate_layout_matches_the_reference(case):
    check_gate_layout(CASES['gate'][case], 'gate')


@pytest.mark.parametrize('case', range(len(CASES['hanging_gate'])))
def test_gate_layout_through_hanging_subedges_matches_the_reference(case):
    check_gate_layout(CASES['hanging_gate'][case], 'hgate')


@pytest.mark.parametrize('case', range(len(CASES['configs'])))
def test_config_schema_matches_the_reference(tmp_path, case):
    spec = CASES['configs'][case]
    config = dict(spec['config'])
    if spec['kind'] == 'domain':
        (tmp_path / 'NE').write_text('mesh\n')
        (tmp_path / 'NS').write_text('mesh\n')
        for key in ('ne', 'ns', 'domain_dir'):
            config[key] = str(tmp_path / config[key])
    model = DomainConfig if spec['kind'] == 'domain' else ForceConfig
    try:
        value = model.model_validate_json(json.dumps(config))
    except ValidationError as error:
        assert not spec['accepted'], error
        assert sorted([[str(p) for p in e['loc']] for e in error.errors()]) == spec['errors']
        return
    assert spec['accepted'], f'the reference rejects {spec["config"]}: {spec["errors"]}'
    dump = value.model_dump(mode='json')
    if spec['kind'] == 'domain':
        for key in ('ne', 'ns', 'domain_dir'):
            dump[key] = Path(dump[key]).name
    assert dump == spec['dump']


@pytest.mark.parametrize('case', CASES['times'], ids=lambda c: c['text'])
def test_absolute_time_matches_the_reference(case):
    if 'error' in case:
        with pytest.raises(ValueError) as error:
            absolute_time(case['text'])
        assert str(error.value) == case['error']
    else:
        assert absolute_time(case['text']).isoformat() == case['value']


@pytest.mark.parametrize('case', CASES['ticks'], ids=lambda c: c['seconds'])
def test_clock_ticks_match_the_reference(case):
    seconds = float(case['seconds'])
    if 'error' in case:
        with pytest.raises(ValueError) as error:
            seconds_to_ticks(seconds)
        assert str(error.value) == case['error']
        return
    ticks = seconds_to_ticks(seconds)
    assert ticks == int(case['ticks'])
    assert words(ticks).tolist() == case['words']


@pytest.mark.parametrize('case', range(len(CASES['series'])))
def test_time_series_match_the_reference(tmp_path, case):
    spec = CASES['series'][case]
    path = tmp_path / 'series.csv'
    path.write_text(spec['csv'])
    if spec['error'] is not None:
        with pytest.raises(ValueError) as error:
            TimeSeries.load(path, ORIGIN, spec['begin'], spec['end'])
        assert str(error.value) == spec['error'].replace('{path}', str(path))
        return
    series = TimeSeries.load(path, ORIGIN, spec['begin'], spec['end'])
    assert series.times.tolist() == spec['times'] and series.values.tolist() == spec['values']
    assert [series.at(q) for q in spec['queries']] == spec['at']


@pytest.mark.parametrize('case', range(len(CASES['rain'])))
def test_rain_intervals_match_the_reference(case):
    spec = CASES['rain'][case]
    field = RainField(np.array(spec['starts']), np.array(spec['ends']), np.array(spec['millimetres']),
                      np.array(spec['pixel_index'], dtype=np.int32))
    assert [field.index_at(q) for q in spec['queries']] == spec['index']
    assert [field.rates(i).tolist() for i in range(len(spec['starts']))] == spec['rates']


@pytest.mark.parametrize('case', range(len(CASES['budget'])))
def test_mass_balance_rows_match_the_reference(tmp_path, case):
    spec = CASES['budget'][case]
    path = tmp_path / 'mass_balance.csv'
    budget = WaterBudget(path, [NS(kind=kind, name=name) for kind, name in spec['boundaries']], spec['initial'])
    for call in spec['calls']:
        if call[0] == 'forcing':
            budget.add_forcing(call[1], call[2], np.array(call[3]))
        elif call[0] == 'terms':
            budget.set_device_terms(np.array(call[1]))
        else:
            budget.output(datetime.fromisoformat(call[1]), call[2], call[3], call[4])
    budget.close()
    assert path.read_text() == spec['csv']


def gate_controller(spec, case):
    """nhflood's GateController in the state the reference's report was given."""
    layout_spec = CASES['gate'][spec['gate_case']]
    config = NS(gates=[NS(name=g['name']) for g in layout_spec['gates']], opening_seconds=case['opening_seconds'],
                trigger_level=case['trigger_level'], pond_land_type=layout_spec['pond_land_type'],
                open_elevation=layout_spec['open_elevation'])
    layout = GateLayout(np.array(layout_spec['cell_gate'], dtype=np.int32),
                        np.array(layout_spec['controls'], dtype=np.int32),
                        [np.array(c, dtype=np.int32) for c in layout_spec['cells']])
    controller = GateController.build(config, layout, ARRAYS['gate_bed'], ARRAYS['gate_types'],
                                      ARRAYS['gate_topology'], case['origin_seconds'])
    controller.totals = np.array(case['totals'])
    controller.initial_storage = case['initial_storage']
    controller.initial_channel_storage = np.array(case['initial_channel'])
    controller.state.update(commanded=np.array(case['commanded'], dtype=np.int32),
                            command=np.array(case['command'], dtype=np.uint32),
                            flow_seen=np.array(case['flow_seen'], dtype=np.int32),
                            first_flow=np.array(case['first_flow'], dtype=np.uint32),
                            opened=np.array(case['opened'], dtype=np.int32),
                            opened_at=np.array(case['opened_at'], dtype=np.uint32))
    return controller


def test_gate_report_and_balance_rows_match_the_reference(tmp_path):
    spec = CASES['report']
    area = np.full(len(ARRAYS['gate_types']), spec['area'])
    path = tmp_path / 'gate_balance.csv'
    for case in spec['cases']:
        report = gate_controller(spec, case).report(np.array(case['depth'], dtype=np.float32), area,
                                                     case['clock_seconds'])
        assert json.loads(json.dumps(report)) == case['report']
        append_gate_balance(path, ORIGIN + timedelta(seconds=case['clock_seconds']), case['clock_seconds'], report)
    assert path.read_text() == spec['balance_csv']


@pytest.mark.parametrize('case', range(len(CASES['hanging'])))
def test_hanging_geometry_matches_the_reference(case):
    arrays = {key: ARRAYS[f'hang{case}_{key}'] for key in ('x', 'y', 'sx', 'sy', 'topology')}
    result = hanging_geometry(arrays['x'], arrays['y'], arrays['sx'], arrays['sy'], arrays['topology'])
    if CASES['hanging'][case]['none']:
        assert result is None
        return
    for key in ('edge_index', 'offsets', 'gradient_slots', 'cells', 'axes'):
        same_bits(getattr(result, key), ARRAYS[f'hang{case}_{key}'])


@pytest.mark.parametrize('case', range(len(CASES['filter'])))
def test_ne_ns_filter_matches_the_reference(case):
    spec = CASES['filter'][case]
    ne, ns = filter_ne_ns(spec['ne'].splitlines(keepends=True), spec['ns'].splitlines(keepends=True))
    assert ''.join(line + '\n' for line in ne) == spec['ne_out']
    assert ''.join(line + '\n' for line in ns) == spec['ns_out']


@pytest.mark.parametrize('case', range(len(CASES['filter'])))
def test_native_preprocessing_builds_the_tables_of_the_reference_filter(case):
    """libnhfprep.so filters in C++; its tables equal the tables built from
    the reference filter's output text."""
    from nhflood import preprocess
    from nhflood.build import build_host
    build_host()
    spec = CASES['filter'][case]
    ne, ns = preprocess.native_tables(spec['ne'].encode(), spec['ns'].encode())
    expected_ne = preprocess.build_ne_tables(spec['ne_out'].splitlines(keepends=True))
    expected_ns = preprocess.build_ns_tables(spec['ns_out'].splitlines(keepends=True))
    for actual, expected in ((ne, expected_ne), (ns, expected_ns)):
        assert actual.keys() == expected.keys()
        for key in actual:
            same_bits(actual[key], np.asarray(expected[key]))


def golden_value(value):
    if isinstance(value, list):
        return np.array([golden_value(v) for v in value])
    return float(value) if isinstance(value, str) else value


@pytest.mark.filterwarnings('ignore:overflow encountered in cast:RuntimeWarning')  # 1e39 rounds to inf in F32
@pytest.mark.parametrize('case', [c for c in CASES['output']['cases'] if 'value' in c], ids=lambda c: str(c['value']))
def test_output_array_rules_match_the_reference(case):
    """The F32 and U32 array rules of the checkpoint, frame and extrema
    writers accept and reject what the reference's do, with its messages."""
    from nhflood.output import _float_array, _uint_array
    for kind, check in (('float', _float_array), ('uint', _uint_array)):
        expected = case[kind]
        if 'error' in expected:
            with pytest.raises(ValueError) as error:
                check(golden_value(case['value']), 'field')
            assert str(error.value) == expected['error']
        else:
            result = check(golden_value(case['value']), 'field')
            assert str(result.dtype) == expected['dtype'] and result.tolist() == expected['values']


def test_station_rows_match_the_reference(tmp_path):
    from nhflood.output import append_station_samples
    path = tmp_path / 'stations.csv'
    for case in CASES['output']['cases']:
        if 'stations_call' in case:
            append_station_samples(path, **case['stations_call'])
    assert path.read_text() == CASES['output']['stations_csv']


@pytest.mark.parametrize('case', range(len(CASES['clock_protocol'])))
def test_batch_clock_protocol_matches_the_reference(case):
    """HostClock.begin / read_trace against StepClock.begin / read_trace:
    the uploaded target and origin words, the host tick mirror, the pending
    flag and every refusal, step by step."""
    from nhflood.clock import HostClock
    spec = CASES['clock_protocol'][case]
    clock = HostClock(spec['initial'])
    for step in spec['steps']:
        try:
            if step['op'] == 'begin':
                target_words, origin_words = clock.begin(step['target'], float(step['origin']))
            else:
                clock.read_trace(np.array(step['rows'], dtype=np.uint32))
        except (ValueError, RuntimeError) as error:
            assert (type(error).__name__, str(error)) == (step.get('error'), step.get('message')), step
        else:
            assert 'error' not in step, step
            if step['op'] == 'begin':
                assert target_words.tolist() == step['next'] and origin_words.tolist() == step['origin_words']
        assert (clock.now_ticks, clock.pending) == (int(step['now']), step['pending']), step


@pytest.mark.parametrize('case', CASES['output']['frames'], ids=lambda c: ','.join(c['names']) or 'none')
def test_depth_frame_listing_matches_the_reference(tmp_path, case):
    from nhflood.output import list_depth_frames
    (tmp_path / 'frames').mkdir()
    for name in case['names']:
        (tmp_path / 'frames' / name).write_bytes(b'')
    if 'error' in case:
        with pytest.raises(ValueError) as error:
            list_depth_frames(tmp_path)
        assert str(error.value) == case['error'].replace('{root}', str(tmp_path))
    else:
        assert [[seconds, path.name] for seconds, path in list_depth_frames(tmp_path)] == case['listed']


@pytest.mark.parametrize('case', range(len(CASES['output']['timelines'])))
def test_bed_timeline_matches_the_reference(tmp_path, case):
    """Frame-time beds: recorded bed events, then the gate beds re-derived
    with the F32 opening arithmetic, bit for bit at every frame time."""
    from nhflood.output import BedTimeline, write_bed
    spec = CASES['output']['timelines'][case]
    write_bed(tmp_path / 'output' / 'bed.fdb', np.array(spec['bed'], dtype=np.float32))
    timeline = BedTimeline(tmp_path / 'output', spec['manifest'])
    for seconds, expected in zip(spec['times'], spec['beds']):
        same_bits(timeline.at(seconds).astype(np.float32), np.array(expected, dtype=np.float32))
