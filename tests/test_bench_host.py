"""bench.py's host-side bookkeeping: the kernels a batch graph launches for
each step form (the ``gpu_launches`` claim) and the algorithmic bytes per
cell-update of each workload kind (the roofline's numerator)."""
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def fake_run(path, *, hang=0, sita=1.0, gate_flux=None, batch=32):
    gate = None if gate_flux is None else SimpleNamespace(flux_sides=np.zeros(gate_flux, np.int32))
    return SimpleNamespace(engine=SimpleNamespace(path=path), arrays=SimpleNamespace(hang_cells=hang, gate=gate),
                           w=SimpleNamespace(sita=sita), params=SimpleNamespace(batch_size=batch))


@pytest.mark.parametrize('path,hang,sita,gate,expected', [
    ('tiled(tile=256,patterns=52,smem=35104,cfl=fused)', 0, 1.0, None, 4 + 32 * 1),
    ('tiled(tile=256,patterns=4159,smem=32852,cfl=pass)', 11000, 1.0, None, 4 + 32 * (2 + 1)),
    ('tiled(tile=256,patterns=4159,smem=32852,cfl=pass)', 0, 0.7, None, 4 + 32 * (2 + 1)),
    ('multipass', 0, 1.0, None, 1 + 32 * 6),
    ('multipass', 5, 0.7, None, 1 + 32 * (6 + 2)),
    # gate runs: exchange volumes with the end motion, the start motion in the
    # CFL pass and once at the batch start (fused) ...
    ('tiled(tile=256,patterns=124,smem=28168,cfl=pass)', 0, 1.0, 2400, 4 + 1 + 32 * (2 + 1)),
    # ... or bed motion, exchange volumes, bed motion (multi-pass)
    ('multipass', 0, 1.0, 2400, 1 + 32 * (6 + 3)),
    ('multipass', 0, 1.0, 0, 1 + 32 * (6 + 2)),
])
def test_launches_per_batch(path, hang, sita, gate, expected):
    import bench
    assert bench.launches_per_batch(fake_run(path, hang=hang, sita=sita, gate_flux=gate)) == expected


def test_algorithmic_bytes_by_workload_kind():
    import bench
    from nhflood import workloads
    assert bench.algorithmic_bytes(workloads.dambreak(n=64)) == 52.0
    assert bench.algorithmic_bytes(workloads.plain_uniform_256(n=64)) == 56.0
    assert bench.algorithmic_bytes(workloads.gated_polder(n=128, dx=40.0)) == 64.0
    q = workloads.multires_quadtree(width=2000.0)
    s_over_n = (q.mesh.s_num - 1) / q.cells
    assert bench.algorithmic_bytes(q) == pytest.approx(52 + 4 + 28 + 12 * s_over_n + 20)


def test_source_hash_is_relocatable_and_ignores_non_sources(tmp_path):
    """The run record's source identity (the reference's test_run_record.py
    property): sorted relative paths, lengths and bytes of the sources only,
    the same after a copy, changed by a rename or an edit."""
    import shutil
    from nhflood.run_record import source_tree_sha256
    src = tmp_path / 'src'
    (src / 'pkg').mkdir(parents=True)
    (src / 'pkg' / 'z.py').write_bytes(b'z=1\n')
    (src / 'a.cu').write_bytes(b'// a\n')
    (src / 'notes.txt').write_text('irrelevant')
    first = source_tree_sha256(src)
    copied = tmp_path / 'copy'
    shutil.copytree(src, copied)
    assert source_tree_sha256(copied) == first
    (copied / 'notes.txt').write_text('changed')
    assert source_tree_sha256(copied) == first
    (copied / 'a.cu').rename(copied / 'b.cu')
    assert source_tree_sha256(copied) != first
    (src / 'pkg' / 'z.py').write_bytes(b'z=2\n')
    assert source_tree_sha256(src) != first
