"""Restart from a run's final checkpoint continues the uninterrupted run bit
for bit (trace rows after the split, every state array, the budget, step
counts), as the reference's tests/test_restart.py:71-243 require; a changed
theta or a checkpoint past the requested end is rejected, and a checkpoint at
the end completes without steps. The case: two connected 10 m cells, rain
moving from one to the other at 5 s, Horton infiltration."""
import json
from pathlib import Path

import numpy as np
import pytest

from nhflood.input import ForceConfig
from nhflood.raster import from_origin
from runner import run
from scenarios import domain, two_cell_mesh, write_rain

STATE = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'first_time_hi',
         'first_time_lo')


def inputs(path: Path):
    path.mkdir(parents=True)
    two_cell_mesh(path, connected=True)
    return write_rain(path, [[[100, 0]], [[0, 100]]], from_origin(0, 10, 10, 10), [(0, 5), (5, 10)])


def solve(src: Path, rain, out: Path, duration, restart='', *, afa=.5, sita=1., engine='oracle'):
    dc = domain(src, duration=duration, yield_step=1, restart=str(restart) if restart else '', afa=afa, sita=sita,
                out=str(out), land={10: dict(manning_n=.03, infiltration=dict(f0_mm_h=36, fc_mm_h=18, k_per_h=2))})
    return run(dc, ForceConfig(boundaries=[], rainfall=rain), engine)


def restart_continues_bitwise(tmp_path, engine):
    src = tmp_path / 'inputs'
    rain = inputs(src)
    full = solve(src, rain, tmp_path / 'full', 10, engine=engine)
    first = solve(src, rain, tmp_path / 'first', 5, engine=engine)
    split = tmp_path / 'first' / 'output' / 'state_final.fdb'
    resumed = solve(src, rain, tmp_path / 'resumed', 10, restart=split, engine=engine)
    ticks = (full.trace[:, 1].astype(np.uint64) << np.uint64(32)) | full.trace[:, 2].astype(np.uint64)
    np.testing.assert_array_equal(full.trace[ticks > np.uint64(5 * 2 ** 40)], resumed.trace)
    assert first.budget['rainfall_m3'] > 0 and first.budget['infiltration_m3'] > 0
    assert np.any(first.state.rain_time[1:] > 0) and np.any(first.state.q[1:] != 0)
    for name in STATE:
        np.testing.assert_array_equal(getattr(full.state, name), getattr(resumed.state, name), err_msg=name)
    assert (full.state.clock_hi, full.state.clock_lo) == (resumed.state.clock_hi, resumed.state.clock_lo)
    assert full.budget == resumed.budget
    assert full.manifest['steps'] == first.manifest['steps'] + resumed.manifest['steps']
    assert json.loads(resumed.state.metadata_json)['total_steps'] == full.manifest['steps']
    assert json.loads(first.state.metadata_json)['elapsed_seconds'] == 5
    return full, resumed


def test_restart_matches_uninterrupted_rain_and_horton_evolution(tmp_path):
    restart_continues_bitwise(tmp_path, 'oracle')


def test_restart_allows_changed_afa_but_rejects_changed_sita(tmp_path):
    src = tmp_path / 'inputs'
    rain = inputs(src)
    first = solve(src, rain, tmp_path / 'first', 5, afa=.25)
    checkpoint = tmp_path / 'first' / 'output' / 'state_final.fdb'
    physics = json.loads(first.state.metadata_json)['physics_config']
    assert physics['afa'] == .25
    final = solve(src, rain, tmp_path / 'resumed', 10, restart=checkpoint, afa=.0625)
    meta = json.loads(final.state.metadata_json)
    assert final.manifest['steps'] > 0 and meta['elapsed_seconds'] == 10
    assert final.budget['rainfall_m3'] > first.budget['rainfall_m3']
    assert meta['physics_config'] == {**physics, 'afa': .0625}
    with pytest.raises(ValueError, match='Checkpoint clock or physical parameters'):
        solve(src, rain, tmp_path / 'changed', 10, restart=checkpoint, afa=.0625, sita=.7)


def test_restart_after_requested_end_is_rejected_and_at_end_takes_no_steps(tmp_path):
    src = tmp_path / 'inputs'
    rain = inputs(src)
    done = solve(src, rain, tmp_path / 'first', 10)
    checkpoint = tmp_path / 'first' / 'output' / 'state_final.fdb'
    with pytest.raises(ValueError, match='Checkpoint time.*simulation end'):
        solve(src, rain, tmp_path / 'invalid', 5, restart=checkpoint)
    same = solve(src, rain, tmp_path / 'same', 10, restart=checkpoint)
    assert same.manifest['steps'] == 0
    assert same.manifest['completion_reason'] == 'checkpoint_at_end'
    assert same.budget == done.budget
    np.testing.assert_array_equal(same.state.depth, done.state.depth)


def test_adopted_state_continues_like_the_original_run():
    """PlainRun.adopt: a second engine that takes over a run's state, clock
    and bookkeeping produces the original run's next batches bit for bit."""
    from engine import OracleEngine
    from nhflood.plain import PlainRun
    from nhflood.workloads import plain_uniform_256
    w = plain_uniform_256(n=32)
    a = PlainRun(w, lambda x, p: OracleEngine(x, p))
    while a.elapsed < 1300:
        a.advance()
    b = PlainRun(w, lambda x, p: OracleEngine(x, p))
    b.adopt(a)
    for _ in range(5):
        ta, oa = a.begin()
        tb, ob = b.begin()
        np.testing.assert_array_equal(ta, tb)
        ra, rb = a.engine.run_batch(ta, oa), b.engine.run_batch(tb, ob)
        np.testing.assert_array_equal(ra, rb)
        a.finish(ra)
        b.finish(rb)
    for name in ('depth', 'q', 'max_depth', 'peak_hi', 'peak_lo'):
        np.testing.assert_array_equal(a.engine.get(name), b.engine.get(name))


def test_nonfinite_budget_term_stops_the_run(tmp_path):
    """device_budget.py:71-73: a non-finite F32 budget term raises at the next
    output's flush (here an engine whose flush reports NaN)."""
    from runner import oracle_factory

    def poisoned(arrays, params):
        engine = oracle_factory(arrays, params)
        clean = engine.budget_flush

        def flush():
            totals = clean()
            totals[0] = float('nan')
            return totals
        engine.budget_flush = flush
        return engine

    src = tmp_path / 'inputs'
    rain = inputs(src)
    with pytest.raises(FloatingPointError, match='Nonfinite F32 device budget diagnostic'):
        solve(src, rain, tmp_path / 'run', 5, engine=poisoned)
