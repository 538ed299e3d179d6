"""The reference's physics cases (positivity, hanging-interface pressure,
coarse/fine channel at theta 0.7 and 1) on the CUDA step, bit for bit
against the oracle, for both step forms; the oracle side of each case is
pinned to the reference's known answers in test_oracle_physics.py."""
import numpy as np
import pytest

from test_gpu_parity import PATHS, assert_runs_identical, cuda_engine
from test_oracle_physics import channel_case, evolve, positivity_case, strip_cells
from scenarios import grid_cell, grid_horizontal, grid_vertical

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('path', PATHS)
def test_positivity_cases_bit_exact(tmp_path, cuda_available, path):
    flows = {grid_vertical(1, 1): -1, grid_vertical(1, 2): 1, grid_horizontal(1, 1): -1, grid_horizontal(2, 1): 1}
    a = positivity_case(tmp_path / 'oracle', wet_cell=grid_cell(1, 1), face_flows=flows)
    b = positivity_case(tmp_path / 'cuda', wet_cell=grid_cell(1, 1), face_flows=flows, engine=cuda_engine(path))
    assert_runs_identical(a, b)
    flows = {grid_vertical(0, 1): 1, grid_horizontal(1, 0): 1}
    a = positivity_case(tmp_path / 'oracle2', wet_cell=grid_cell(0, 0), face_flows=flows, extraction=True)
    b = positivity_case(tmp_path / 'cuda2', wet_cell=grid_cell(0, 0), face_flows=flows, extraction=True,
                        engine=cuda_engine(path))
    assert_runs_identical(a, b)


@pytest.mark.parametrize('path', PATHS)
def test_pressure_reconstruction_cases_bit_exact(tmp_path, cuda_available, path):
    cases = [(strip_cells(False), lambda x, y, i: .001 * y, lambda x, y, z, i: 1., .125),
             (strip_cells(True), lambda x, y, i: ((i % 7) - 3) * .125, lambda x, y, z, i: 2. - z, 60.),
             ([(0, 8, 0, 8), (8, 12, 0, 4), (8, 12, 4, 8), (0, 4, 8, 12), (4, 8, 8, 12), (8, 12, 8, 12)],
              lambda x, y, i: .0013 * x - .0007 * y, lambda x, y, z, i: 1., .125)]
    for k, (cells, bed_at, depth_at, seconds) in enumerate(cases):
        sa = evolve(tmp_path / f'o{k}', cells, bed_at, depth_at, seconds)[0]
        sb = evolve(tmp_path / f'c{k}', cells, bed_at, depth_at, seconds, engine=cuda_engine(path))[0]
        for name in ('depth', 'q', 'max_depth', 'max_speed'):
            np.testing.assert_array_equal(getattr(sa, name).view(np.uint32), getattr(sb, name).view(np.uint32),
                                          err_msg=f'case {k} {name}')


@pytest.mark.parametrize('path', PATHS)
@pytest.mark.parametrize('theta', [0.7, 1.0])
def test_coarse_fine_channel_bit_exact(tmp_path, cuda_available, theta, path):
    _, a, _ = channel_case(tmp_path / 'oracle', theta)
    _, b, _ = channel_case(tmp_path / 'cuda', theta, engine=cuda_engine(path))
    assert_runs_identical(a, b)


@pytest.mark.parametrize('path', PATHS)
@pytest.mark.parametrize('theta', [0.7, 1.0])
def test_open_channel_bit_exact(tmp_path, cuda_available, theta, path):
    from test_oracle_physics import open_boundary_case
    a = open_boundary_case(tmp_path / 'oracle', 'channel', theta, .1)[0]
    b = open_boundary_case(tmp_path / 'cuda', 'channel', theta, .1, engine=cuda_engine(path))[0]
    assert_runs_identical(a, b)


@pytest.mark.parametrize('path', PATHS)
def test_restart_continues_bitwise_on_the_gpu(tmp_path, cuda_available, path):
    from test_oracle_restart import restart_continues_bitwise
    full_o, resumed_o = restart_continues_bitwise(tmp_path / 'oracle', 'oracle')
    full_c, resumed_c = restart_continues_bitwise(tmp_path / 'cuda', cuda_engine(path))
    np.testing.assert_array_equal(full_o.trace, full_c.trace)
    np.testing.assert_array_equal(resumed_o.trace, resumed_c.trace)
    assert full_o.budget == full_c.budget
