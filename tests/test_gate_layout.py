"""Gate configuration and layout resolution (the reference's
tests/test_gate_config.py): schema validation, component partition by
shared subedges, inside/control point location and every rejection the
layout makes (overlap, empty pond, unclaimed or shared components, missing
pond or river interface, open elevation above a closed bed, level boundary
overlap), including with the controller disabled."""
from types import SimpleNamespace

import numpy as np
import pytest
from pydantic import ValidationError

from nhflood.gate import GateController, GateLayout, flux_sides
from nhflood.input import GateConfig


def config(**changes):
    return GateConfig(**(dict(land_type=11, pond_land_type=10, enabled=True, trigger_level=3.07,
                              opening_seconds=1800, open_elevation=1.3,
                              gates=[dict(name='A', inside_point=(1.5, .5), control_point=(.5, .5))]) | changes))


@pytest.mark.parametrize('changes', [dict(threshold=3), dict(level_boundary='sea'), dict(opening_seconds=0),
                                     dict(opening_seconds=float('inf')), dict(pond_land_type=-1),
                                     dict(pond_land_type=256), dict(pond_land_type=11),
                                     dict(gates=[dict(name='A', inside_point=(float('nan'), 0),
                                                      control_point=(0, 0))])])
def test_invalid_config(changes):
    with pytest.raises(ValidationError):
        config(**changes)


def test_pond_land_type_is_required():
    raw = config().model_dump()
    del raw['pond_land_type']
    with pytest.raises(ValidationError, match='pond_land_type'):
        GateConfig(**raw)


def layout(cfg, types=(0, 1, 11, 11, 10, 11, 1), boundaries=(), bed=None, topology=None):
    bounds = np.array([[0, 0, 0, 0]] + [[i, 0, i + 1, 1] for i in range(len(types) - 1)], dtype=float)
    if topology is None:
        topology = np.array([[0, 0, 0]] + [[2, i, i + 1] for i in range(1, len(types) - 1)])
    if bed is None:
        bed = np.full(len(types), 2.0)
    return GateLayout.load(cfg, bounds, np.array(types), topology, boundaries, np.array(bed))


def two_gates(**changes):
    return config(gates=[dict(name='A', inside_point=(1.5, .5), control_point=(.5, .5)),
                         dict(name='B', inside_point=(4.5, .5), control_point=(5.5, .5))], **changes)


def test_component_partition():
    resolved = layout(two_gates())
    assert resolved.cell_gate.tolist() == [-1, -1, 0, 0, -1, 1, -1]
    assert resolved.controls.tolist() == [1, 6]
    assert [a.tolist() for a in resolved.cells] == [[2, 3], [5]]


def test_configurable_pond_land_type():
    resolved = layout(two_gates(pond_land_type=7), types=(0, 1, 11, 11, 7, 11, 1))
    assert [a.tolist() for a in resolved.cells] == [[2, 3], [5]]


def test_mesh_loader_rejects_overlapping_regions_after_model_mutation():
    cfg = two_gates()
    cfg.pond_land_type = cfg.land_type
    with pytest.raises(ValueError, match='must not overlap'):
        layout(cfg)


def test_equal_f32_closed_target_is_allowed_but_next_higher_target_is_not():
    beds = np.full(7, np.float32(1.3), dtype=np.float32)
    layout(two_gates(open_elevation=1.3), bed=beds)
    with pytest.raises(ValueError, match='open_elevation'):
        layout(two_gates(open_elevation=float(np.nextafter(np.float32(1.3), np.float32(2.)))), bed=beds)


@pytest.mark.parametrize('enabled', [True, False])
def test_unclaimed_component_rejected_even_when_disabled(enabled):
    with pytest.raises(ValueError, match='exactly one'):
        layout(config(enabled=enabled))


@pytest.mark.parametrize('field,point,error', [('inside_point', (3.5, .5), 'not on'),
                                               ('inside_point', (10, 10), 'outside'),
                                               ('control_point', (1.5, .5), 'on a gate'),
                                               ('control_point', (10, 10), 'outside')])
def test_invalid_point(field, point, error):
    cfg = two_gates()
    setattr(cfg.gates[0], field, point)
    with pytest.raises(ValueError, match=error):
        layout(cfg)


def test_duplicate_component_and_name_rejected():
    cfg = two_gates()
    cfg.gates[1].inside_point = (2.5, .5)
    with pytest.raises(ValueError, match='exactly one'):
        layout(cfg)
    with pytest.raises(ValidationError, match='unique'):
        config(gates=[cfg.gates[0], cfg.gates[0]])


@pytest.mark.parametrize('enabled', [True, False])
def test_level_overlap_rejected(enabled):
    with pytest.raises(ValueError, match='overlap'):
        layout(two_gates(enabled=enabled), boundaries=[SimpleNamespace(kind='level', cells=np.array([3]))])


@pytest.mark.parametrize('enabled', [True, False])
def test_empty_pond_rejected_even_when_disabled(enabled):
    with pytest.raises(ValueError, match='selects no pond cells'):
        layout(two_gates(enabled=enabled), types=(0, 1, 11, 11, 1, 11, 1))
    with pytest.raises(ValueError, match='selects no pond cells'):
        layout(two_gates(enabled=enabled, pond_land_type=0))


@pytest.mark.parametrize('enabled', [True, False])
def test_missing_gate_interface_rejected_even_when_disabled(enabled):
    cfg = two_gates(enabled=enabled)
    no_pond_edge = np.array([[0, 0, 0], [2, 1, 2], [2, 2, 3], [2, 5, 6]])
    with pytest.raises(ValueError, match='edges to pond'):
        layout(cfg, topology=no_pond_edge)
    no_river_edge = np.array([[0, 0, 0], [2, 2, 3], [2, 3, 4], [2, 4, 5], [2, 5, 6]])
    with pytest.raises(ValueError, match='non-pond'):
        layout(cfg, topology=no_river_edge)


@pytest.mark.parametrize('enabled', [True, False])
def test_open_elevation_above_any_closed_cell_rejected_even_when_disabled(enabled):
    with pytest.raises(ValueError, match='open_elevation'):
        layout(two_gates(enabled=enabled), bed=(0, 2, 2, 1.2, 2, 2, 2))
    assert layout(two_gates(enabled=enabled), bed=(0, 2, 2, 1.3, 2, 2, 2)).cell_gate[3] == 0


def test_components_are_numbered_by_their_lowest_cell():
    """A component whose cells come later in id order but touch a lower cell
    through a long chain still takes the rank of its lowest cell."""
    types = [0] + [11] * 9
    topology = np.array([[0, 0, 0], [2, 9, 8], [2, 8, 7], [2, 7, 1], [2, 2, 3], [2, 3, 4], [2, 5, 6]])
    from nhflood.gate import _components
    comp = _components(np.array(types) == 11, topology)
    assert comp.tolist() == [-1, 0, 1, 1, 1, 2, 2, 0, 0, 0]


def test_recorded_sides_and_device_tables():
    """Sides recorded by the controller: gate/non-gate and pond/non-pond
    sides outside the gates; the tables carry the closed bed and formal tick."""
    cfg = two_gates()
    types = np.array([0, 1, 11, 11, 10, 11, 1])
    topology = np.array([[0, 0, 0]] + [[2, i, i + 1] for i in range(1, 6)] + [[2, 0, 1], [2, 4, 0]])
    lay = layout(cfg, topology=topology)
    bed = np.full(7, 2.0, np.float32)
    controller = GateController.build(cfg, lay, bed, types, topology, 2.0)
    t = controller.tables
    assert t.terms == 28 and t.count == 2
    assert t.pond.tolist() == [0, 0, 0, 0, 1, 0, 0]
    assert t.targets.tolist() == [2, 3, 5]
    assert t.formal_tick == 2 * 2 ** 40
    # 1-2 gate/river, 3-4 gate/pond, 4-5 pond/gate, 5-6 gate/river, 4-0 pond/exterior
    assert flux_sides(t.cell_gate, t.pond, topology).tolist() == [1, 3, 4, 5, 7]
