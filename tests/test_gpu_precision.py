"""The FP64 build of the CUDA step (libnhflood_f64.so: the multi-pass
kernels compiled with nhf_real = double, the clock unchanged) against the
CPU restatement's FP64 build (oracle/step_ref.c with -DORA_REAL_DOUBLE),
bit for bit, on cases of the step's golden set; and the F32 step's depth
gap to it on a flowing case, the quantity the precision form reports."""
import numpy as np
import pytest

import step_cases

pytestmark = pytest.mark.gpu

CASES = ['two_cell_horton', 'two_cell_warmup_level_discharge', 'grid3_limiter_theta07', 'pressure_plane',
         'channel_theta07_30s', 'open_channel_theta07_600s', 'quadtree_small', 'dambreak_48']


@pytest.mark.parametrize('name', CASES)
def test_fp64_cuda_step_matches_the_fp64_restatement(tmp_path, cuda_available, name):
    from engine import OracleEngine
    from nhflood.native import CudaEngine
    a = step_cases.record_case(name, tmp_path / 'oracle', lambda ar, p: OracleEngine(ar, p, precision='f64'))
    b = step_cases.record_case(name, tmp_path / 'cuda', lambda ar, p: CudaEngine(ar, p, precision='f64'))
    np.testing.assert_array_equal(a['trace'], b['trace'])
    for key in ('depth', 'q'):
        assert a[key].dtype == np.float64 and b[key].dtype == np.float64
        np.testing.assert_array_equal(a[key].view(np.uint64), b[key].view(np.uint64), err_msg=key)
    np.testing.assert_array_equal(a['budget'], b['budget'])


def test_f32_step_against_its_fp64_build(cuda_available):
    """The 64 x 64 crop for 300 s: the F32 depths stay within 1 mm of the
    FP64 build's at every yield time (a gentle case; the configurations'
    own figures come from ``python -m nhflood.precision``)."""
    from nhflood.precision import compare
    worst = compare(step_cases.workload('uniform_64'))
    assert worst['steps_f32'] > 100 and worst['max_depth_m'] > 0.04
    assert worst['max_abs_m'] < 1e-3, worst
