"""Batched form's host logic on the CPU: members of different sizes and
durations advance together, each with its own clock and dt; a member that
has reached its end time takes an empty batch (target = its clock) while
the others go on; every member ends bit-identical to its own plain run.
The CPU restatement stands in for the CUDA step and a sequential stand-in
for the ensemble launch (tests/runner.py), so this checks
nhflood/ensemble.py itself; tests/test_gpu_ensemble.py runs it on the GPU."""
import numpy as np


def members():
    from nhflood.workloads import multires_quadtree, plain_uniform_256
    ws = [multires_quadtree(seed=21, width=600.0, duration=150, uniform_rain=40.0),
          plain_uniform_256(n=24),
          multires_quadtree(seed=22, width=400.0, duration=60, uniform_rain=80.0)]
    ws[1].duration = 100
    return ws


def test_members_match_their_plain_runs_and_finished_members_idle():
    from nhflood.ensemble import EnsembleRun
    from nhflood.model import STATE_F32, STATE_U32
    from nhflood.plain import PlainRun
    from runner import SequentialEnsemble, oracle_factory
    ens = EnsembleRun(members(), engine_factory=oracle_factory, ensemble_factory=SequentialEnsemble)
    steps = np.zeros(3, np.int64)
    frozen = None
    while not ens.done:
        steps += ens.advance()
        if ens.runs[2].done and frozen is None:
            frozen = (steps[2], ens.runs[2].engine.get('depth').copy())
        elif frozen is not None:  # the shortest member keeps taking empty batches
            assert steps[2] == frozen[0]
            assert ens.runs[2].engine.get('depth').tobytes() == frozen[1].tobytes()
    assert frozen is not None and (steps > 0).all()
    assert ens.cell_updates(steps) == int((steps * ens.cells).sum())
    for i, w in enumerate(members()):
        alone = PlainRun(w, oracle_factory)
        while not alone.done:
            alone.advance()
        assert alone.steps == steps[i] == ens.runs[i].steps
        for name in STATE_F32 + STATE_U32:
            assert alone.engine.get(name).tobytes() == ens.runs[i].engine.get(name).tobytes(), (i, name)
        assert np.array_equal(alone.engine.budget_flush(), ens.runs[i].engine.budget_flush())
        alone.close()
    ens.close()
