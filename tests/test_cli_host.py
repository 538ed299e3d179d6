"""``python -m nhflood``, the reference's main.py command line
(nh-flood-2d main.py:8-17): its arguments, the refused pipe config, and the
product path failing loudly where there is no GPU."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

PACKAGE = Path(__file__).resolve().parents[1] / 'nh-flood-2d_b200'


def nhflood(*args, cwd=PACKAGE):
    return subprocess.run([sys.executable, '-m', 'nhflood', *map(str, args)], cwd=cwd, capture_output=True, text=True)


def test_help_names_the_reference_arguments():
    result = nhflood('--help')
    assert result.returncode == 0
    for flag in ('--domain', '--force', '--pipe'):
        assert flag in result.stdout


def test_domain_and_force_are_required():
    result = nhflood('--domain', 'domain.json')
    assert result.returncode == 2 and '--force' in result.stderr


def test_pipe_config_is_refused_before_any_work(tmp_path):
    result = nhflood('--domain', tmp_path / 'missing.json', '--force', tmp_path / 'missing.json',
                     '--pipe', tmp_path / 'pipe.json')
    assert result.returncode == 2 and 'SWMM pipe coupling is not part of this engine' in result.stderr


def test_without_a_gpu_the_run_fails_loudly_and_records_it(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present: the full run is covered by the GPU tests')
    from scenarios import two_cell_case
    dc, fc = two_cell_case(tmp_path / 'case', [[6, 6]], 10)
    (tmp_path / 'domain.json').write_text(dc.model_dump_json())
    (tmp_path / 'force.json').write_text(fc.model_dump_json())
    result = nhflood('--domain', tmp_path / 'domain.json', '--force', tmp_path / 'force.json')
    assert result.returncode == 1
    assert 'the step has no CPU fallback' in result.stderr
    manifest = json.loads((Path(dc.domain_dir) / 'manifest.json').read_text())
    assert manifest['status'] == 'failed' and 'no CPU fallback' in manifest['error']
