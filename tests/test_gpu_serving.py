"""Served form: continuous batching under an HBM budget. Each request's
final depth and max-depth frames are identical alone (plain form, one at a
time) and in the mix; the budget bounds what is resident; requests overlap
on the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def requests():
    from nhflood.serving import Request
    from nhflood.workloads import multires_quadtree, plain_uniform_256
    ws = [multires_quadtree(seed=11, width=1500.0, duration=300, uniform_rain=60.0),
          multires_quadtree(seed=12, width=2500.0, duration=200, uniform_rain=90.0),
          plain_uniform_256(n=64),
          multires_quadtree(seed=13, width=1200.0, duration=400, uniform_rain=20.0)]
    ws[2].duration = 240
    return [Request(i, 0.0, w) for i, w in enumerate(ws)]


def test_served_results_equal_sequential_results(cuda_available):
    from nhflood.serving import FloodServer, device_bytes_bound, serve, serve_sequential
    reqs = requests()
    for r in reqs:
        assert device_bytes_bound(r.workload) >= r.prepare()
    needs = sorted(device_bytes_bound(r.workload) for r in reqs)
    budget = needs[-1] + needs[-2] + 1  # at most the two largest together
    server = FloodServer(hbm_budget=budget, tile=256)
    resident = []
    step = server.step

    def counting_step():
        out = step()
        resident.append(len(server.active) + len(out))
        return out
    server.step = counting_step
    served = {c.id: c for c in serve(reqs, server, realtime=False)}
    server.close()
    assert sorted(served) == [0, 1, 2, 3]
    assert server.peak_used <= budget
    assert max(resident) >= 2
    alone = {c.id: c for c in serve_sequential(requests(), tile=256, realtime=False)}
    for i in range(4):
        a, b = served[i], alone[i]
        assert a.steps == b.steps and a.cells == b.cells
        np.testing.assert_array_equal(a.depth.view(np.uint32), b.depth.view(np.uint32))
        np.testing.assert_array_equal(a.max_depth.view(np.uint32), b.max_depth.view(np.uint32))
    assert any(served[i].max_depth.max() > 0.02 for i in range(4))


def test_request_larger_than_budget_is_rejected(cuda_available):
    from nhflood.serving import FloodServer
    reqs = requests()[:1]
    server = FloodServer(hbm_budget=1e6, tile=256)
    server.submit(reqs[0])
    with pytest.raises(ValueError, match='budget'):
        server.step()
    server.close()
