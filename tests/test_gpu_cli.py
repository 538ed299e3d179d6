"""A complete run through ``python -m nhflood`` from a copy of the package
without Git metadata (the reference's tests/test_run_record.py:28-46): the
manifest records completion, no commit, and the copy's source hash."""
import json
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

PACKAGE = Path(__file__).resolve().parents[1] / 'nh-flood-2d_b200'


def test_complete_simulation_in_copy_without_git(tmp_path, cuda_available):
    from nhflood.run_record import source_tree_sha256
    from scenarios import two_cell_case
    copied = tmp_path / 'distribution' / 'nh-flood-2d_b200'
    shutil.copytree(PACKAGE, copied, ignore=shutil.ignore_patterns('__pycache__'))
    dc, fc = two_cell_case(tmp_path / 'inputs', [[6, 6]], 10)
    (tmp_path / 'domain.json').write_text(dc.model_dump_json())
    (tmp_path / 'force.json').write_text(fc.model_dump_json())
    result = subprocess.run([sys.executable, '-m', 'nhflood', '--domain', str(tmp_path / 'domain.json'),
                             '--force', str(tmp_path / 'force.json')], cwd=copied, capture_output=True, text=True)
    assert result.returncode == 0, result.stdout + result.stderr
    manifest = json.loads((Path(dc.domain_dir) / 'manifest.json').read_text())
    assert manifest['status'] == 'completed' and manifest['steps'] > 0
    assert manifest['backend'] == 'cuda'
    assert manifest['git_commit'] is None and manifest['git_dirty'] is None
    assert manifest['source_sha256'] == source_tree_sha256(copied) == source_tree_sha256(PACKAGE)
