"""Gate controller on the B200: the CUDA step with the controller attached,
on the fused step (256-cell tiles, separate CFL pass) and on the multi-pass
step, is bit-identical to the CPU restatement through the whole time loop (state,
trace, controller words and every exchange and source total of the
``gate_control`` report), on the reference's gate mechanism cases: bed
motion and pond exchange, a short level pulse latching the command, seven
large gate components, split (hanging) gate faces, pond rain, Horton
infiltration and overtopping, a limited first step, and a restart in the
middle of the opening."""
import numpy as np
import pytest

from gate_cases import level_boundary, run, setup
from nhflood.input import DomainConfig
from nhflood.output import read_checkpoint, write_checkpoint

pytestmark = pytest.mark.gpu

STATE = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'first_time_hi',
         'first_time_lo')


CUDA = ('cuda', 'cuda_multipass')


def same(tmp_path, make, seconds, **kw):
    results = {}
    for engine in ('oracle',) + CUDA:
        dc, force = make(tmp_path / engine)
        results[engine] = run(dc, force, seconds, engine=engine, **kw)
    a = results['oracle']
    for engine in CUDA:
        b = results[engine]
        assert b.manifest['backend'] == 'cuda'
        for name in STATE:
            assert getattr(a.state, name).tobytes() == getattr(b.state, name).tobytes(), (engine, name)
        np.testing.assert_array_equal(a.trace, b.trace)
        assert a.manifest['gate_control'] == b.manifest['gate_control'], engine
        assert a.state.gate_open == b.state.gate_open
        assert a.manifest['mass_balance_final'] == b.manifest['mass_balance_final'], engine
    return a, results['cuda']


def test_bed_motion_and_pond_exchange(tmp_path):
    def make(path):
        dc, force, *_ = setup(path, depth=[2, 2, 1])
        return dc, force
    a, _ = same(tmp_path, make, 3)
    gate = a.manifest['gate_control']['gates'][0]
    assert gate['pond_in_m3'] > 0 and gate['fully_open_seconds'] == 1


def test_short_level_pulse_latches_the_command(tmp_path):
    def make(path):
        boundaries = level_boundary(path, [(0, 1), (.125, 2), (.25, 1), (3600, 1)])
        dc, force, *_ = setup(path, bed=[0, 10, 0], depth=[1, 0, 0], boundaries=boundaries,
                              gate=dict(trigger_level=1.5, opening_seconds=1.875, open_elevation=0))
        return dc, force
    a, _ = same(tmp_path, make, 2)
    assert a.manifest['gate_control']['gates'][0]['command_seconds'] == .125


def test_seven_large_components(tmp_path):
    def make(path):
        cells, types, bed, depth, gates = [], [], [], [], []
        for group in range(7):
            y = group * 100
            for row in range(22):
                for col in range(25):
                    x, bottom = 4 * col, y + 4 * row
                    cells.append((x, x + 4, bottom, bottom + 4))
                    types.append(1 if row == 0 else 10 if row == 21 else 11)
                    bed.append(0. if row in (0, 21) else 1.)
                    depth.append(2. if row == 0 else .3 if row == 21 else .2)
            gates.append(dict(name=f'G{group}', inside_point=(2, y + 6), control_point=(2, y + 2)))
        dc, force, *_ = setup(path, cells=cells, types=types, bed=bed, depth=depth,
                              gate=dict(gates=gates, opening_seconds=.25, trigger_level=1., open_elevation=0.))
        return dc, force
    a, _ = same(tmp_path, make, .5)
    assert len(a.manifest['gate_control']['gates']) == 7


def test_split_gate_faces(tmp_path):
    def make(path):
        cells = [(100, 110, 0, 10), (0, 10, 0, 10), (10, 15, 0, 5), (10, 15, 5, 10), (15, 25, 0, 10)]
        dc, force, *_ = setup(path, cells=cells, types=[1, 10, 11, 11, 1], depth=[2, 2, 2, 2, 2],
                              gate=dict(gates=[dict(name='A', inside_point=(12, 2), control_point=(105, 5))]))
        return dc, force
    same(tmp_path, make, 2)


def test_pond_rain_infiltration_and_overtopping(tmp_path):
    def make(path):
        cells = [(i * 10, (i + 1) * 10, 0, 10) for i in range(4)]
        dc, force, *_ = setup(path, cells=cells, types=[1, 11, 10, 1], depth=[2, 2, 1, .5], rain=100,
                              gate=dict(open_elevation=0))
        data = dc.model_dump()
        data['land_parameters'][10]['infiltration'] = dict(f0_mm_h=36, fc_mm_h=18, k_per_h=2)
        return DomainConfig.model_validate(data), force
    a, _ = same(tmp_path, make, 4)
    pond = a.manifest['gate_control']['pond_budget']
    assert pond['rain_m3'] > 0 and pond['infiltration_m3'] > 0 and pond['overtopping_out_m3'] > 0


def test_limited_first_step(tmp_path):
    def make(path):
        dc, force, topo, *_ = setup(path, depth=[.021, .021, 0], gate=dict(trigger_level=-1, open_elevation=0))
        seed = read_checkpoint(dc.restart_state)
        seed.q[np.flatnonzero((topo[:, 1] == 2) & (topo[:, 2] == 3))[0]] = 100
        seed.q[np.flatnonzero((topo[:, 1] == 1) & (topo[:, 2] == 2))[0]] = -100
        write_checkpoint(dc.restart_state, **vars(seed))
        return dc.model_copy(update={'afa': 1.}), force
    a, _ = same(tmp_path, make, 1)
    assert a.manifest['limiter_activity']['limited_face_steps'] > 0


def test_restart_during_opening_matches_the_oracle(tmp_path):
    def make(path):
        boundaries = level_boundary(path, [(0, 1), (1, 1), (2, 2), (3600, 2)])
        dc, force, *_ = setup(path, boundaries=boundaries, depth=[1, 0, 0], bed=[0, 3, 0],
                              gate=dict(trigger_level=1.5, opening_seconds=2))
        return dc, force
    for engine in ('oracle',) + CUDA:
        dc, force = make(tmp_path / engine)
        run(dc, force, 3, output=tmp_path / engine / 'part', engine=engine)
    results = {}
    for engine in ('oracle',) + CUDA:
        dc, force = make(tmp_path / engine)
        results[engine] = run(dc, force, 6, output=tmp_path / engine / 'resumed', engine=engine,
                              restart=tmp_path / engine / 'part/output/state_final.fdb')
    a = results['oracle']
    for engine in CUDA:
        b = results[engine]
        for name in STATE:
            assert getattr(a.state, name).tobytes() == getattr(b.state, name).tobytes(), (engine, name)
        assert a.manifest['gate_control'] == b.manifest['gate_control'], engine


@pytest.mark.parametrize('path', ['auto', 'multipass'])
def test_gated_polder_matches_the_oracle_batch_by_batch(path):
    """The polder workload at 128 x 128 (four gates, 256 gate cells, 384
    recorded sides), on the fused and the multi-pass step: 10 batches on
    both engines, state, controller words and gate totals identical after
    every batch."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / 'oracle'))
    from engine import OracleEngine
    from nhflood import workloads
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    w = workloads.gated_polder(n=128, dx=40.0)
    def cuda(a, p):
        p.path = path
        return CudaEngine(a, p)

    runs = [PlainRun(w, lambda a, p: OracleEngine(a, p)), PlainRun(w, cuda)]
    if path == 'auto':
        assert runs[1].engine.path.startswith('tiled(tile=256') and 'cfl=pass' in runs[1].engine.path
    else:
        assert runs[1].engine.path.startswith('multipass')
    for _ in range(10):
        steps = [r.advance() for r in runs]
        assert steps[0] == steps[1]
        for name in STATE_F32 + STATE_U32:
            assert runs[0].engine.get(name).tobytes() == runs[1].engine.get(name).tobytes(), name
        a, b = (r.engine.gate_state() for r in runs)
        for name in a:
            np.testing.assert_array_equal(a[name], b[name], err_msg=name)
        np.testing.assert_array_equal(runs[0].engine.gate_flush(), runs[1].engine.gate_flush())
    assert all(runs[1].engine.gate_state()['commanded'] == 1)
    for r in runs:
        r.close()


def test_gated_polder_full_size_matches_the_oracle_batch_by_batch():
    """The bench's polder at its full size, 1024 x 1024 cells of 5 m (four
    gates of 64 cells commanded at t = 0 and opening over 600 s), on the
    fused step: state, controller words and gate totals identical to the CPU
    restatement after each of the first three 32-step batches."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / 'oracle'))
    from engine import OracleEngine
    from nhflood import workloads
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    w = workloads.gated_polder()
    runs = [PlainRun(w, lambda a, p: OracleEngine(a, p)), PlainRun(w, CudaEngine)]
    try:
        assert runs[1].engine.path.startswith('tiled(tile=256') and 'cfl=pass' in runs[1].engine.path
        bed0 = runs[1].engine.get('bed').copy()
        for _ in range(3):
            steps = [r.advance() for r in runs]
            assert steps[0] == steps[1] == 32
            for name in STATE_F32 + STATE_U32:
                assert runs[0].engine.get(name).tobytes() == runs[1].engine.get(name).tobytes(), name
            a, b = (r.engine.gate_state() for r in runs)
            for name in a:
                np.testing.assert_array_equal(a[name], b[name], err_msg=name)
            np.testing.assert_array_equal(runs[0].engine.gate_flush(), runs[1].engine.gate_flush())
        assert all(runs[1].engine.gate_state()['commanded'] == 1)
        assert (runs[1].engine.get('bed') < bed0).sum() == 4 * 64  # every gate cell has moved down
    finally:
        for r in runs:
            r.close()


def test_gated_members_run_in_the_member_graph_schedule_only():
    """A gated polder in an ensemble: the one-launch schedule, which has no
    gate passes, refuses it; in the member-graph schedule, beside an ungated
    member, it matches its own single run bit for bit, gate words and totals
    included."""
    from nhflood import workloads
    from nhflood.ensemble import EnsembleRun
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.native import CudaEngine
    from nhflood.plain import PlainRun
    gated, plain = workloads.gated_polder(n=128, dx=40.0), workloads.plain_uniform_256(n=64)
    with pytest.raises(RuntimeError, match='gate controller'):
        EnsembleRun([plain, gated], tile=256, grid_blocks=-1)
    ens, single = EnsembleRun([plain, gated]), PlainRun(gated, CudaEngine)
    try:
        assert ens.schedule == 'member graphs'
        for _ in range(4):
            completed = ens.advance()
            assert completed[1] == single.advance() > 0
            member = ens.runs[1].engine
            for name in STATE_F32 + STATE_U32:
                assert member.get(name).tobytes() == single.engine.get(name).tobytes(), name
            a, b = member.gate_state(), single.engine.gate_state()
            for name in a:
                np.testing.assert_array_equal(a[name], b[name], err_msg=name)
            np.testing.assert_array_equal(member.gate_flush(), single.engine.gate_flush())
        assert all(member.gate_state()['commanded'] == 1)
    finally:
        ens.close()
        single.close()
