"""Served form's scheduling logic on the CPU: admission under the memory
budget, first come first served, solves resident together, retirement,
and results equal alone and in the mix. The CPU restatement stands in for
the CUDA step and a sequential stand-in for the ensemble launch, so these
check the host side of nhflood/serving.py; tests/test_gpu_serving.py runs
the same logic on the GPU."""
import numpy as np
import pytest


def requests():
    from nhflood.serving import Request
    from nhflood.workloads import multires_quadtree, plain_uniform_256
    ws = [multires_quadtree(seed=11, width=600.0, duration=120, uniform_rain=60.0),
          plain_uniform_256(n=24),
          multires_quadtree(seed=13, width=500.0, duration=200, uniform_rain=20.0)]
    ws[1].duration = 90
    return [Request(i, 0.0, w) for i, w in enumerate(ws)]


def server(budget, resident=None):
    from nhflood.serving import FloodServer
    from runner import SequentialEnsemble, oracle_factory
    s = FloodServer(hbm_budget=budget, device='cpu', engine_factory=oracle_factory,
                    ensemble_factory=SequentialEnsemble)
    if resident is not None:
        step = s.step

        def counting_step():
            out = step()
            resident.append(len(s.active) + len(out))
            return out
        s.step = counting_step
    return s


def test_served_results_equal_sequential_and_the_budget_holds():
    from nhflood.serving import device_bytes_bound, serve, serve_sequential
    from runner import oracle_factory
    reqs = requests()
    needs = sorted(device_bytes_bound(r.workload) for r in reqs)
    budget = needs[-1] + needs[-2] + 1  # at most the two largest together
    resident = []
    s = server(budget, resident)
    served = {c.id: c for c in serve(reqs, s, realtime=False)}
    s.close()
    assert sorted(served) == [0, 1, 2]
    assert s.peak_used <= budget
    assert max(resident) >= 2
    alone = {c.id: c for c in serve_sequential(requests(), device='cpu', realtime=False,
                                               engine_factory=oracle_factory)}
    for i in range(3):
        a, b = served[i], alone[i]
        assert a.steps == b.steps > 0 and a.cells == b.cells
        np.testing.assert_array_equal(a.depth.view(np.uint32), b.depth.view(np.uint32))
        np.testing.assert_array_equal(a.max_depth.view(np.uint32), b.max_depth.view(np.uint32))
    # every request is admitted after it arrived and finishes after admission
    for c in served.values():
        assert c.arrival <= c.admitted <= c.finished


def test_budget_admits_first_come_first_served():
    """With room for one solve at a time the solves run one after another
    in arrival order, each alone."""
    from nhflood.serving import device_bytes_bound, serve
    reqs = requests()
    budget = max(device_bytes_bound(r.workload) for r in reqs) + 1
    resident = []
    s = server(budget, resident)
    done = serve(reqs, s, realtime=False)
    s.close()
    assert [c.id for c in done] == [0, 1, 2]
    assert max(resident) == 1


def test_request_larger_than_budget_is_rejected():
    s = server(1e6)
    s.submit(requests()[0])
    with pytest.raises(ValueError, match='budget'):
        s.step()
    s.close()
