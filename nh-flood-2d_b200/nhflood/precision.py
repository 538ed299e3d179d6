"""Precision form: the F32 step against the FP64 build of the same kernels.

The state is F32 on the GPU (the reference's field type); FP64 is used only
for the budget partials and the simulation clock (fixed-point ticks). This
study runs every configuration twice on the GPU, through libnhflood.so (F32)
and libnhflood_f64.so (the multi-pass kernels compiled with double physics,
the clock unchanged), each run taking its own CFL dt as a real FP64 build
would, and compares the depths cell by cell at every yield time.

    python -m nhflood.precision [--cases NAMES] [--out FILE] [--device cuda:0]

Cases, at the configurations' full sizes: the 65,536-cell plain grid
(3600 s), the 1,362,175-cell quadtree (7200 s), the 4096 x 4096 dam break
(1800 s), all 64 ensemble members (3600 s each) and a sample of the served
request stream. Reported per case: max, 99.9th percentile and RMS of
|h32 - h64| over all cells and yield times, and the max-depth extrema gap.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np


def cases(requests: int = 16):
    from . import workloads as W
    stream = W.served_requests()[:requests]
    return {
        'plain_uniform_256': lambda: [W.plain_uniform_256()],
        'multires_quadtree': lambda: [W.multires_quadtree()],
        'dambreak_4096': lambda: [W.dambreak()],
        'ensemble_64': lambda: W.ensemble_scenarios(),
        f'served_first_{requests}': lambda: [W.multires_quadtree(**r['params']) for r in stream],
    }


def compare(workload, device: str = 'cuda:0', batch_size: int = 32) -> dict:
    """Both precisions advanced to every yield time (batch targets end there),
    the depth gap taken there; returns the worst figures and the step counts."""
    from .native import CudaEngine
    from .plain import PlainRun
    runs = {p: PlainRun(workload, lambda a, q, p=p: CudaEngine(a, q, device=device, precision=p),
                        batch_size=batch_size) for p in ('f32', 'f64')}
    step = workload.yield_step
    times = list(np.arange(step, workload.duration, step)) + [float(workload.duration)]
    worst = dict(max_abs_m=0.0, p999_abs_m=0.0, rms_m=0.0, time_s=0.0, max_depth_m=0.0)
    sq_sum, count = 0.0, 0
    try:
        for t in times:
            for r in runs.values():
                while r.elapsed < t - 1e-9 and not r.done:
                    r.advance()
            if runs['f32'].elapsed != runs['f64'].elapsed:
                raise RuntimeError('the two precisions did not stop at the same yield time')
            a = runs['f32'].engine.get('depth').astype(np.float64)[1:]
            b = runs['f64'].engine.get('depth')[1:]
            d = np.abs(a - b)
            if d.size and d.max() >= worst['max_abs_m']:
                worst.update(max_abs_m=float(d.max()), time_s=float(t))
            if d.size:
                worst['p999_abs_m'] = max(worst['p999_abs_m'], float(np.percentile(d, 99.9)))
                worst['max_depth_m'] = max(worst['max_depth_m'], float(b.max()))
                sq_sum += float((d * d).sum())
                count += d.size
        worst['rms_m'] = float(np.sqrt(sq_sum / count)) if count else 0.0
        ea = runs['f32'].engine.get('max_depth').astype(np.float64)[1:]
        eb = runs['f64'].engine.get('max_depth')[1:]
        worst['max_depth_extrema_abs_m'] = float(np.abs(ea - eb).max()) if ea.size else 0.0
        worst['steps_f32'], worst['steps_f64'] = runs['f32'].steps, runs['f64'].steps
        worst['path_f32'] = runs['f32'].engine.path
    finally:
        for r in runs.values():
            r.close()
    return worst


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--cases', default=None, help='comma-separated case names (default: all)')
    ap.add_argument('--requests', type=int, default=16)
    ap.add_argument('--out', default=None)
    ap.add_argument('--device', default='cuda:0')
    args = ap.parse_args()
    table = {}
    available = cases(args.requests)
    for name in (args.cases.split(',') if args.cases else available):
        t0 = time.perf_counter()
        rows = []
        for w in available[name]():
            rows.append(dict(workload=w.name, cells=w.cells, duration_s=w.duration,
                             **compare(w, device=args.device)))
        members = np.array([r['max_abs_m'] for r in rows])
        table[name] = dict(members=rows, max_abs_m=float(members.max()),
                           rms_m=float(np.sqrt(np.mean([r['rms_m'] ** 2 for r in rows]))),
                           seconds=round(time.perf_counter() - t0, 1))
        print(json.dumps({name: {k: v for k, v in table[name].items() if k != 'members'}}), flush=True)
    if args.out:
        Path(args.out).write_text(json.dumps(table, indent=1))


if __name__ == '__main__':
    main()
