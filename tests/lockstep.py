"""Run the CUDA step and the CPU restatement side by side, one time step per
batch, and report the first state array that differs (debugging aid for the
parity tests)."""
from __future__ import annotations

import numpy as np

from nhflood.forcing import Forcing
from nhflood.geometry import MeshGeometry
from nhflood.plain import PlainRun
from nhflood.preprocess import load_mesh, preprocess
from nhflood.workloads import Workload

FIELDS = ('depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'u', 'v', 'peak_hi', 'peak_lo')


def workload_from_case(dc, fc, name='case') -> Workload:
    preprocess(dc, fc)
    mesh, _ = load_mesh(dc)
    geometry = MeshGeometry.from_mesh(mesh)
    forcing = Forcing.load(dc, fc, geometry)
    return Workload(name, mesh, geometry, forcing, dc.land_parameters, duration=dc.duration,
                    yield_step=dc.yield_step, afa=dc.afa, sita=dc.sita, min_h=dc.min_h)


def first_divergence(workload, factory_a, factory_b, max_steps=100000):
    """Returns None when both runs agree to the end, else a report dict."""
    a = PlainRun(workload, factory_a, batch_size=1)
    b = PlainRun(workload, factory_b, batch_size=1)
    try:
        for name in FIELDS:
            x, y = a.engine.get(name), b.engine.get(name)
            if not np.array_equal(x.view(np.uint32), y.view(np.uint32)):
                return dict(step=0, field=name, where=np.flatnonzero(x.view(np.uint32) != y.view(np.uint32))[:8])
        step = 0
        while not a.done and step < max_steps:
            ta, oa = a.begin()
            tb, ob = b.begin()
            ra = a.engine.run_batch(ta, oa)
            rb = b.engine.run_batch(tb, ob)
            a.finish(ra)
            b.finish(rb)
            step += 1
            report = {}
            if not np.array_equal(ra, rb):
                report['trace'] = (ra, rb)
            for name in FIELDS:
                x, y = a.engine.get(name), b.engine.get(name)
                bad = np.flatnonzero(x.view(np.uint32) != y.view(np.uint32))
                if len(bad):
                    report.setdefault('fields', {})[name] = (bad[:8], x[bad[:8]], y[bad[:8]])
            if report:
                report['step'] = step
                report['elapsed'] = a.elapsed
                return report
        return None
    finally:
        a.close()
        b.close()
