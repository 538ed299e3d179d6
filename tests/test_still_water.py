"""Warm-up still-water fill (hydraulic connectivity of level boundaries):
the reference's tests/test_still_water.py:24-56,102-105 cases on
nhflood.geometry.connected_still_water."""
from types import SimpleNamespace as NS

import numpy as np
import pytest

from nhflood.geometry import connected_still_water


def boundary(name, cell, level):
    return NS(name=name, kind='level', cells=np.array([cell]), series=NS(at=lambda t: level))


def fill(bed, levels, *, crest=None, closed=None):
    """A chain of four cells beside the exterior cell 0 (no route through it)."""
    sides = np.array([[0, 0, 0], [2, 0, 1], [2, 1, 2], [2, 2, 3], [2, 3, 4], [2, 4, 0]])
    return connected_still_water(np.array([0, *bed], np.float32),
                                 np.full(6, -999.) if crest is None else np.array(crest),
                                 np.zeros(6, np.uint8) if closed is None else np.array(closed),
                                 sides, levels, np.array([0, 1, 1, 1, 1]))


def test_bed_barrier_is_strict_and_isolated_low_pool_stays_empty():
    depth, meta = fill([-2, -1, 1, -3], [boundary('sea', 1, 1)])
    np.testing.assert_array_equal(depth, [0, 3, 2, 0, 0])
    assert meta['storage_m3'] == 5


@pytest.mark.parametrize('obstacle', ['crest', 'closed'])
def test_edge_crest_and_closed_side_block_filling(obstacle):
    kw = {'crest': [-999, -999, -999, 1, -999, -999]} if obstacle == 'crest' else {'closed': [0, 0, 0, 1, 0, 0]}
    depth, _ = fill([-2, -1, -2, -3], [boundary('sea', 1, 1)], **kw)
    np.testing.assert_array_equal(depth, [0, 3, 2, 0, 0])


@pytest.mark.parametrize('reverse', [False, True])
def test_connected_different_levels_reject_in_either_order(reverse):
    levels = [boundary('sea_A', 1, 1), boundary('sea_B', 4, .5)]
    with pytest.raises(ValueError, match='Conflicting initial levels'):
        fill([-2, -1, -2, -3], levels[::-1] if reverse else levels)


def test_disconnected_levels_fill_separately_and_equal_levels_share_body():
    depth, _ = fill([-2, 2, -2, -3], [boundary('A', 1, 1), boundary('B', 4, .5)])
    np.testing.assert_array_equal(depth, [0, 3, 0, 2.5, 3.5])
    depth, meta = fill([-2, -1, -2, -3], [boundary('A', 1, 1), boundary('B', 4, 1)])
    np.testing.assert_array_equal(depth, [0, 3, 2, 3, 4])
    assert len(meta['levels']) == 1 and meta['levels'][0]['connected_components'] == 1


def test_connectivity_compares_input_level_without_rounding_it_to_f32():
    depth, _ = fill([1, 1, 1, 1], [boundary('sea', 1, 1 + 1e-8)])
    np.testing.assert_allclose(depth[1:], 1e-8, rtol=1e-7)
