"""Batched form: every member of an ensemble gives, bit for bit, the run it
gives alone (trace rows, final state, budget), for both grid schedules of
the ensemble step, with members of different mesh kinds, sizes, forcing
and durations (so some members finish while others still step)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ('depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'peak_hi', 'peak_lo', 'u', 'v')


def members():
    from nhflood.workloads import dambreak, multires_quadtree, plain_uniform_256
    a = multires_quadtree(width=2000.0, duration=600)
    depth = np.where(a.mesh.land_type == 0, 1.5, 0.3).astype(np.float32)
    depth[0] = 0.0
    a.initial_depth = depth
    b = multires_quadtree(seed=7, width=1500.0, duration=420, hyetograph_peak=90.0, n_factors=[1.1, .9, 1.2, .8])
    c = plain_uniform_256(n=64)
    c.duration = 900
    d = dambreak(n=96, duration=45)
    return [a, b, c, d]


def alone(w, tile):
    from nhflood.ensemble import tiled_factory
    from nhflood.plain import PlainRun
    run = PlainRun(w, tiled_factory(tile, cfl='fused'))  # the members run the separate CFL pass
    rows = []
    while not run.done:
        tw, ow = run.begin()
        trace = run.engine.run_batch(tw, ow)
        rows.append(trace[:run.finish(trace)])
    state = {n: run.engine.get(n) for n in STATE}
    budget = run.engine.budget_flush()
    run.close()
    return np.concatenate(rows), state, budget


@pytest.mark.parametrize('grid', [0, -1, 3, -2])
def test_members_match_their_single_runs(cuda_available, grid):
    """grid -2: the member graphs, each member on its own plain engine."""
    from nhflood.ensemble import EnsembleRun
    ws = members()
    expected = [alone(w, 256) for w in ws]
    ens = EnsembleRun(ws, tile=None if grid == -2 else 256, grid_blocks=grid)
    assert ens.ensemble.members == 4 and ens.ensemble.tile == (0 if grid == -2 else 256)
    rows = [[] for _ in ws]
    batches = 0
    while not ens.done:
        targets, origins = ens.begin()
        traces = ens.ensemble.run_batch(targets, origins)
        completed = ens.finish(traces)
        for i, n in enumerate(completed):
            rows[i].append(traces[i][:n])
        batches += 1
    assert batches > 1
    for i, (trace, state, budget) in enumerate(expected):
        np.testing.assert_array_equal(np.concatenate(rows[i]), trace, err_msg=f'member {i}')
        eng = ens.runs[i].engine
        for name in STATE:
            np.testing.assert_array_equal(eng.get(name).view(np.uint32), state[name].view(np.uint32),
                                          err_msg=f'member {i} {name}')
        np.testing.assert_array_equal(eng.budget_flush(), budget)
    ens.close()


def test_members_must_share_the_tile_size(cuda_available):
    from nhflood.ensemble import tiled_factory
    from nhflood.model import StepParams
    from nhflood.native import CudaEnsemble
    ws = members()[2:]
    engines = []
    for w, tile in zip(ws, (256, 512)):
        p = StepParams(batch_size=32)
        engines.append(tiled_factory(tile)(w.step_arrays(), p))
    with pytest.raises(RuntimeError, match='tile'):
        CudaEnsemble(engines)
    for e in engines:
        e.close()
