"""Synthetic workload generators: mesh consistency (every face side touches
its cell with the right orientation, every side listed by exactly its
cells), 2:1 balance, hanging interfaces, and the forcing they carry."""
import numpy as np

from nhflood.geometry import MeshGeometry
from nhflood.workloads import dambreak, multires_quadtree, plain_uniform_256, uniform_grid


def check_mesh(m):
    topo = m.topology
    listed = np.zeros(m.s_num, int)
    for c in range(1, m.e_num):
        for d in range(4):
            p, n = m.face_ptr[c, d], m.counts[c, d]
            assert n >= 1
            for sid in m.isl_data[p:p + n]:
                orient = 2 if d in (0, 1) else 1
                assert topo[sid, 0] == orient
                assert topo[sid, 2 if d in (0, 2) else 1] == c
                listed[sid] += 1
    expected = (topo[:, 1] != 0).astype(int) + (topo[:, 2] != 0)
    np.testing.assert_array_equal(listed[1:], expected[1:])
    MeshGeometry.from_mesh(m)  # square cells, exterior sides on faces


def test_tile_major_uniform_grid_is_consistent():
    check_mesh(uniform_grid(70, 45, 2.0, np.zeros((45, 70)), np.ones((45, 70), np.uint8), tile=32))


def test_small_quadtree_is_balanced_and_has_hanging_interfaces():
    w = multires_quadtree(width=2000.0, duration=600)
    check_mesh(w.mesh)
    levels = w.mesh.level[1:]
    assert set(np.unique(levels)) == {0, 1, 2}
    arrays = w.step_arrays()
    assert arrays.hang_cells > 1000 and arrays.hang_edges > 1000
    # every coarse face with two sides has half-length sides
    two = w.mesh.counts[1:] == 2
    assert two.any()
    assert np.isclose(w.mesh.side_length[w.mesh.isl_data[w.mesh.face_ptr[1:][two]]], 0.0).sum() == 0


def test_configs_have_the_stated_shape():
    w = plain_uniform_256()
    assert w.cells == 65536 and w.duration == 3600 and w.yield_step == 300
    assert len(w.forcing.boundaries) == 1 and w.forcing.boundaries[0].kind == 'level'
    assert len(w.forcing.boundaries[0].cells) == 256  # the south edge
    assert w.forcing.boundaries[0].series.values[0] < w.mesh.z[1:].min() - 99
    np.testing.assert_array_equal(w.forcing.rain.millimetres[:, 0], [25.0, 0.0])
    d = dambreak(n=128, duration=60)
    assert d.cells == 128 * 128
    assert np.all(d.initial_depth[1:][d.mesh.x[1:] < 12.8] == 2.0)
    assert np.all(d.initial_depth[1:][d.mesh.x[1:] >= 12.8] == 0.0)
    assert len(d.forcing.boundaries[0].cells) == 4 * 128 - 4


def test_ensemble_parameters_follow_the_batched_configuration():
    from nhflood.workloads import ensemble_members, multires_quadtree, quadtree_width_for
    ps = ensemble_members()
    assert len(ps) == 64
    widths = np.array([p['width'] for p in ps])
    assert widths.min() >= quadtree_width_for(50e3) - 40 and widths.max() <= quadtree_width_for(2e6) + 40
    assert np.all(widths % 20 == 0)
    peaks = np.array([p['hyetograph_peak'] for p in ps])
    assert 25 < np.median(peaks) < 60
    f = np.array([p['n_factors'] for p in ps])
    assert f.min() >= 0.8 and f.max() <= 1.2
    w = multires_quadtree(**dict(ps[3], width=1500.0))
    mm = w.forcing.rain.millimetres[:, 0]
    assert len(mm) == 60 and mm.argmax() in (29, 30)
    assert abs(mm.sum() - ps[3]['hyetograph_peak'] / 2) < 1e-3  # a 1 h triangle holds peak/2 mm
    assert w.land_parameters[2].manning_n == 0.05 * ps[3]['n_factors'][2]


def test_served_request_stream_has_the_configured_distribution():
    from nhflood.serving import device_bytes_estimate
    from nhflood.workloads import multires_quadtree, quadtree_width_for, served_requests
    reqs = served_requests()
    assert len(reqs) == 512
    arrivals = np.array([r['arrival'] for r in reqs])
    assert np.all(np.diff(arrivals) > 0)
    assert 200 < arrivals[-1] < 320  # 512 arrivals at 2 per second
    widths = np.array([r['params']['width'] for r in reqs])
    assert widths.min() >= quadtree_width_for(16e3) - 40 and widths.max() <= quadtree_width_for(4e6) + 40
    d = np.array([r['params']['duration'] for r in reqs])
    assert d.min() >= 600 and d.max() <= 3600
    rain = np.array([r['params']['uniform_rain'] for r in reqs])
    assert rain.min() >= 10 and rain.max() <= 100
    w = multires_quadtree(**dict(reqs[0]['params'], width=1000.0))
    assert w.forcing.rain.millimetres.shape[0] == 1
    assert abs(w.forcing.rain.millimetres[0, 0] - reqs[0]['params']['uniform_rain'] * w.duration / 3600) < 1e-3
    a = w.step_arrays()
    assert device_bytes_estimate(a) > a.nbytes() + 40 * a.e_num


def test_gated_polder_resolves_its_gates_and_opens_them_on_the_oracle():
    """The gate benchmark workload: four gates of 4 x 16 cells through the
    dike, every one commanded at t = 0 (control cells start 1 m deep, the
    trigger is 0.5 m above the highest control bed) and fully open after
    600 s; water reaches the pond through every gate."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / 'oracle'))
    from engine import OracleEngine
    from nhflood import workloads
    from nhflood.plain import PlainRun
    w = workloads.gated_polder(n=128, dx=40.0)
    run = PlainRun(w, lambda a, p: OracleEngine(a, p))
    gate = run.arrays.gate
    assert gate.count == 4 and len(gate.targets) == 4 * 4 * 16
    assert run.engine.gate_state()['commanded'].tolist() == [1, 1, 1, 1]
    while run.elapsed < 700:
        run.advance()
    state = run.engine.gate_state()
    assert state['opened'].tolist() == [1, 1, 1, 1] and state['flow_seen'].tolist() == [1, 1, 1, 1]
    totals = run.engine.gate_flush()
    assert all(totals[4 * g] > 0 for g in range(4))  # pond inflow through every gate
    bed = run.engine.get('bed')
    assert np.all(bed[gate.targets] == np.float32(-1.0))
    run.close()


def test_made_ahead_keeps_a_window_of_the_stream():
    """Served-stream meshes are made in arrival order, at most ``ahead``
    beyond the last one taken, and a request drops its host copies once a
    run holds them."""
    import threading
    from concurrent.futures import ThreadPoolExecutor
    from nhflood.serving import MadeAhead

    made, lock = [], threading.Lock()

    class Fake:
        def __init__(self, cells):
            self.cells = cells

    def make(params):
        with lock:
            made.append(params['n'])
        return Fake(params['n'] * 10)

    stream = [{'id': i, 'arrival': 0.5 * i, 'params': {'n': i}} for i in range(20)]
    with ThreadPoolExecutor(2) as ex:
        source = MadeAhead(make, stream, ex, ahead=4)
        source.wait_first()
        assert sorted(made) == [0, 1, 2, 3]
        reqs = source.requests()
        assert [r.id for r in reqs] == list(range(20))
        w = reqs[0].resolve()
        assert w.cells == 0 and reqs[0].cells == 0
        assert source.submitted == 5           # the window moved by one
        assert reqs[6].resolve().cells == 60   # taking ahead of order fills up to it
        assert source.submitted == 11
        reqs[0].release()
        assert reqs[0].workload is None and reqs[0].arrays is None
        for r in reqs[1:6] + reqs[7:]:
            assert r.resolve().cells == 10 * r.id
    assert sorted(made) == list(range(20))
