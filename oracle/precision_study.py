"""ORACLE-side measurement (test infrastructure, not the product): the depth
error of the F32 step against the same step computed in F64.

The F32 restatement (liboracle.so) is bit-identical to the CUDA step on
every parity case, so its error against the F64 build (liboracle_f64.so:
the same source with real = double, the clock unchanged) is the error of the
GPU's F32 state. Both runs take the same batch targets; at every yield time
the depths are compared cell by cell.

    python oracle/precision_study.py [--same-dt] [--out FILE] [--cases NAMES]

Cases (the configurations' workloads; the large uniform grid is run at
512 x 512 cells with the same 1 m spacing, because its full 16.8M-cell,
1800 s F64 run takes hours on the CPU):
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / 'nh-flood-2d_b200'))

from engine import OracleEngine  # noqa: E402


def cases():
    from nhflood import workloads as W
    ens = W.ensemble_members()
    small = sorted(ens, key=lambda p: p['width'])[:2]
    req = W.served_requests()
    small_req = sorted(req, key=lambda r: r['params']['width'])[:2]
    return {
        'plain_uniform_256': lambda: W.plain_uniform_256(),
        'multires_quadtree': lambda: W.multires_quadtree(),
        'dambreak_512': lambda: W.dambreak(n=512),
        'ensemble_smallest_2': lambda: [W.multires_quadtree(**p) for p in small],
        'served_smallest_2': lambda: [W.multires_quadtree(**r['params']) for r in small_req],
    }


def compare(workload, same_dt: bool = False, yield_step=None):
    """Max/99.9th/RMS |h32 - h64| over all cells at every yield time. With
    same_dt the F64 run takes the F32 run's CFL candidate before every step
    (one step per batch), so both integrate with the identical dt sequence
    and the difference is the arithmetic's alone; otherwise each run picks
    its own dt, as a real F64 build would."""
    from nhflood.plain import PlainRun
    bs = 1 if same_dt else 32
    runs = {p: PlainRun(workload, lambda a, q, p=p: OracleEngine(a, q, precision=p), batch_size=bs)
            for p in ('f32', 'f64')}
    step = yield_step or workload.yield_step
    worst = {'max_abs_m': 0.0, 'p999_abs_m': 0.0, 'rms_m': 0.0, 'time_s': 0.0, 'max_depth_m': 0.0,
             'max_depth_extrema_abs_m': 0.0}
    checkpoints = list(np.arange(step, workload.duration, step)) + [float(workload.duration)]
    for t in checkpoints:
        # batches end at every yield time, so both runs stop exactly there
        # (their dt sequences, and so their batch ends in between, may differ)
        if same_dt:
            while runs['f32'].elapsed < t - 1e-9:
                runs['f64'].engine.set_ndt(runs['f32'].engine.ndt())
                runs['f32'].advance()
                runs['f64'].advance()
        else:
            for r in runs.values():
                while r.elapsed < t - 1e-9:
                    r.advance()
        if runs['f32'].elapsed != runs['f64'].elapsed:
            raise RuntimeError('the two runs did not stop at the same yield time')
        a = runs['f32'].engine.get('depth').astype(np.float64)[1:]
        b = runs['f64'].engine.get('depth')[1:]
        d = np.abs(a - b)
        if d.max() >= worst['max_abs_m']:
            worst.update(max_abs_m=float(d.max()), time_s=float(t))
        worst['p999_abs_m'] = max(worst['p999_abs_m'], float(np.percentile(d, 99.9)))
        worst['rms_m'] = max(worst['rms_m'], float(np.sqrt((d * d).mean())))
        worst['max_depth_m'] = max(worst['max_depth_m'], float(b.max()))
    ea = runs['f32'].engine.get('max_depth').astype(np.float64)[1:]
    eb = runs['f64'].engine.get('max_depth')[1:]
    worst['max_depth_extrema_abs_m'] = float(np.abs(ea - eb).max())
    steps = {p: r.steps for p, r in runs.items()}
    for r in runs.values():
        r.close()
    return worst, steps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--out', default=None)
    ap.add_argument('--cases', default=','.join(cases()))
    ap.add_argument('--same-dt', action='store_true', help='F64 follows the F32 dt sequence')
    args = ap.parse_args()
    table = {}
    for name in args.cases.split(','):
        t0 = time.perf_counter()
        made = cases()[name]()
        members = made if isinstance(made, list) else [made]
        rows = []
        for w in members:
            worst, steps = compare(w, same_dt=args.same_dt)
            rows.append(dict(workload=w.name, cells=w.cells, duration_s=w.duration, steps_f32=steps['f32'],
                             steps_f64=steps['f64'], **worst))
        table[name] = dict(members=rows, seconds=round(time.perf_counter() - t0, 1))
        print(json.dumps({name: table[name]}), flush=True)
    if args.out:
        Path(args.out).write_text(json.dumps(table, indent=1))


if __name__ == '__main__':
    main()
