"""Autotuner host logic: candidate sweep over the member graphs and the
one-launch tile/grid schedules, winner, JSON cache round trip, cache hits
skip measurement, signatures separate devices and meshes."""
import json

from nhflood import autotune
from nhflood.workloads import plain_uniform_256, dambreak


def test_sweep_picks_fastest_and_caches(tmp_path):
    ws = [plain_uniform_256(n=32), dambreak(n=32, duration=10)]
    calls = []

    def fake(workloads, tile, grids, batch_size, device):
        calls.append(tile)
        if tile == 1024:
            return {g: None for g in grids}  # does not fit
        return {g: float(tile * (2 if g == -1 else 1)) for g in grids}

    def graphs(workloads, batch_size, device):
        calls.append('graphs')
        return 300.0

    cache = tmp_path / 'tune.json'
    s = autotune.choose_schedule(ws, cache=cache, device_name='B200', measure_fn=fake, member_graphs_fn=graphs,
                                 tiles=(256, 512, 1024))
    assert (s.tile, s.grid, s.rate) == (512, -1, 1024.0)
    assert calls == ['graphs', 256, 512, 1024]
    assert len(s.trials) == 7 and [1024, 0, None] in s.trials and [0, -2, 300.0] in s.trials
    data = json.loads(cache.read_text())
    assert len(data) == 1
    again = autotune.choose_schedule(ws, cache=cache, device_name='B200', measure_fn=fake, member_graphs_fn=graphs)
    assert len(calls) == 4 and (again.tile, again.grid) == (512, -1)
    other = autotune.choose_schedule(ws, cache=cache, device_name='H100', measure_fn=fake,
                                     member_graphs_fn=lambda *a: 5000.0)
    assert (other.tile, other.grid) == (0, autotune.MEMBER_GRAPHS)  # the member graphs win
    assert len(json.loads(cache.read_text())) == 2


def test_signature_depends_on_meshes_and_batch():
    a, b = plain_uniform_256(n=32), plain_uniform_256(n=48)
    assert autotune.signature([a], 32, 'B200') != autotune.signature([b], 32, 'B200')
    assert autotune.signature([a], 32, 'B200') != autotune.signature([a], 16, 'B200')
    assert autotune.signature([a, b], 32, 'B200') == autotune.signature([a, b], 32, 'B200')
