"""Golden vectors from the reference's own code (tests/golden/make_golden.py
ran preprocess/hydraulics.py, preprocess/gate.py and input/*.py of
nh-flood-2d on seeded quadtree meshes and configs). Every case is replayed
through nhflood: arrays must match bit for bit, errors by message, configs
by acceptance, error locations and the validated dump."""
import json
from pathlib import Path
from types import SimpleNamespace as NS

import numpy as np
import pytest
from pydantic import ValidationError

from nhflood.gate import GateLayout
from nhflood.geometry import connected_still_water, map_land_parameters, open_boundary_face_fractions
from nhflood.input import DomainConfig, ForceConfig, LandParameters, absolute_time

GOLDEN = Path(__file__).parent / 'golden'
CASES = json.loads((GOLDEN / 'host_golden.json').read_text())
ARRAYS = np.load(GOLDEN / 'host_golden.npz')
MESH = {key[5:]: ARRAYS[key] for key in ARRAYS.files if key.startswith('mesh_')}


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


@pytest.mark.parametrize('case', range(len(CASES['gate'])))
def test_gate_layout_matches_the_reference(case):
    spec = CASES['gate'][case]
    types_ = ARRAYS['gate_types'].copy()
    if spec['overlap']:
        types_[types_ == spec['land_type']] = spec['pond_land_type']
    config = NS(land_type=spec['land_type'], pond_land_type=spec['pond_land_type'],
                open_elevation=spec['open_elevation'],
                gates=[NS(name=g['name'], inside_point=tuple(g['inside_point']),
                          control_point=tuple(g['control_point'])) for g in spec['gates']])
    boundaries = [NS(kind='level', cells=np.asarray(cells, dtype=np.int64)) for cells in spec['level_cells']]
    args = (config, ARRAYS['gate_bounds'], types_, ARRAYS['gate_topology'], boundaries, ARRAYS['gate_bed'])
    if spec['error'] is not None:
        with pytest.raises(ValueError) as error:
            GateLayout.load(*args)
        assert str(error.value) == spec['error']
        return
    layout = GateLayout.load(*args)
    assert layout.cell_gate.tolist() == spec['cell_gate']
    assert layout.controls.tolist() == spec['controls']
    assert [c.tolist() for c in layout.cells] == spec['cells']


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
