"""Output and restart file contracts (the reference's tests/test_output_io.py):
single-array F32 depth frames and their ordering, the bed timeline rebuilt
from bed.fdb plus bed events, checkpoints that keep every F32 bit, the clock
words and the metadata text, extrema, station resolution (smallest cell id
on a shared edge) and one CSV row per station."""
import csv

import numpy as np
import pytest

from nhflood.geometry import ExteriorEdges, MeshGeometry
from nhflood.output import (append_station_samples, list_depth_frames, read_bed_at, read_checkpoint,
                            read_depth_frame, read_extrema, resolve_station_cells, write_bed, write_checkpoint,
                            write_depth_frame, write_extrema, write_manifest)


def test_depth_frames_are_single_f32_arrays_and_bed_events_rebuild_the_bed(tmp_path):
    root = tmp_path / 'output'
    write_bed(root / 'bed.fdb', [0, 10, 20])
    write_depth_frame(root / 'frames/depth_900.fdb', [0, .25, .5])
    write_depth_frame(root / 'frames/depth_0.fdb', [0, 1, 2])
    write_manifest(root.parent / 'manifest.json',
                   {'bed_events': [{'elapsed_seconds': 450, 'cell_ids': [1], 'new_bed': [0]}]})
    assert [seconds for seconds, _ in list_depth_frames(root)] == [0, 900]
    np.testing.assert_array_equal(read_bed_at(root, 0), [0, 10, 20])
    np.testing.assert_array_equal(read_bed_at(root, 900), [0, 0, 20])
    depth = read_depth_frame(root / 'frames/depth_900.fdb', expected_count=3)
    assert depth.dtype == np.float32
    np.testing.assert_array_equal(depth, [0, .25, .5])
    with pytest.raises(ValueError, match='expected 4'):
        read_depth_frame(root / 'frames/depth_900.fdb', expected_count=4)


def test_checkpoint_preserves_exact_f32_and_metadata_and_extrema(tmp_path):
    path = tmp_path / 'checkpoint.fdb'
    depth = np.array([0, np.nextafter(np.float32(0), np.float32(1))], dtype=np.float32)
    metadata_json = '{ "budget_units": ["12345678901234567890"], "phase": "simulation" }'
    write_checkpoint(path, depth=depth, bed=[0, 10000], q=[0, -0.25, 0.5], rain_time=[0, 12],
                     infiltration=[0, .0001], max_depth=[0, .5], first_time_hi=[0, 2], first_time_lo=[0, 3],
                     max_speed=[0, 1.25], clock_hi=2, clock_lo=4294967295, gate_open=True,
                     metadata_json=metadata_json)
    state = read_checkpoint(path, expected_cells=2, expected_sides=3)
    np.testing.assert_array_equal(state.depth.view(np.uint32), depth.view(np.uint32))
    np.testing.assert_array_equal(state.bed, [0, 10000])
    np.testing.assert_array_equal(state.q, [0, -.25, .5])
    np.testing.assert_array_equal(state.max_depth, [0, .5])
    np.testing.assert_array_equal(state.first_time_hi, [0, 2])
    np.testing.assert_array_equal(state.first_time_lo, [0, 3])
    np.testing.assert_array_equal(state.max_speed, [0, 1.25])
    assert (state.clock_hi, state.clock_lo, state.gate_open) == (2, 4294967295, True)
    assert state.metadata_json == metadata_json
    with pytest.raises(ValueError, match='side count'):
        read_checkpoint(path, expected_sides=4)
    with pytest.raises(ValueError, match='depth'):
        write_checkpoint(path, depth=[0, np.nan], bed=[0, 10000], q=[0, 0, 0], rain_time=[0, 0],
                         infiltration=[0, 0], max_depth=depth, first_time_hi=[0, 0], first_time_lo=[0, 0],
                         max_speed=[0, 0], clock_hi=0, clock_lo=0, gate_open=False, metadata_json='{}')
    maxima_path = tmp_path / 'extrema.fdb'
    write_extrema(maxima_path, [0, .5], [0, 2], [0, 4294967295], [0, 1.25])
    maxima = read_extrema(maxima_path, expected_count=2)
    np.testing.assert_array_equal(maxima.max_depth, [0, .5])
    np.testing.assert_array_equal(maxima.first_time_hi, [0, 2])
    np.testing.assert_array_equal(maxima.first_time_lo, [0, 4294967295])
    np.testing.assert_array_equal(maxima.max_speed, [0, 1.25])


def two_cells():
    """Two 10 m cells centred at x = 5 and 15 sharing the edge x = 10."""
    edges = ExteriorEdges(np.zeros(0, int), np.zeros(0, int), np.zeros(0, int), np.zeros(0), np.zeros((0, 2, 2)))
    return MeshGeometry(np.array([0., 5., 15.]), np.array([0., 5., 5.]),
                        np.array([[0, 0, 0, 0], [0, 0, 10, 10], [10, 0, 20, 10]], float),
                        np.array([0., 100., 100.]), edges)


def test_station_boundary_chooses_smallest_cell_and_csv_has_one_row_per_station(tmp_path):
    cells = resolve_station_cells({'joint': (10, 5), 'right': (15, 5)}, two_cells())
    assert cells == {'joint': 1, 'right': 2}
    with pytest.raises(ValueError, match='outside the mesh'):
        resolve_station_cells({'missing': (25, 5)}, two_cells())
    csv_path = tmp_path / 'stations.csv'
    append_station_samples(csv_path, elapsed_seconds=300, time='2024-01-01T00:05:00+00:00',
                           samples={'right': {'cell_id': 2, 'depth': .5, 'level': 20.5, 'u': 1, 'v': 2},
                                    'joint': {'cell_id': 1, 'depth': .25, 'level': 10.25, 'u': 3, 'v': 4}})
    with csv_path.open(newline='') as stream:
        rows = list(csv.DictReader(stream))
    assert [row['station'] for row in rows] == ['joint', 'right']
    assert rows[0]['cell_id'] == '1'
    assert rows[0]['level'] == '10.25'
