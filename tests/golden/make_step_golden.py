"""Golden vectors for the local-inertial step from the reference's own source.

    python tests/golden/make_step_golden.py --reference PATH [--jobs N] [--cases NAME ...]

The reference path may also come from the environment variable
NHF_REFERENCE. The script loads nh-flood-2d's unchanged step kernels
(core/solver_compact.py, core/clock.py, core/pressure.py,
core/device_budget.py) under a serial NumPy stand-in for Taichi
(ti_standin.py; reference_step.py binds them to the fields ``_evolve``
creates) and runs every case of tests/step_cases.py through this project's
host loop on them. For each case it writes the trace rows of every batch
(dt bits, clock words, status, CFL candidate, event flag, limiter counts,
minimum donor scale, wet-cell count), the depth and discharge arrays at the
end of every batch and every budget flush to step_golden.npz, twice:

  libm/<case>/...     powf and expf from the C library, the functions
                      Taichi's LLVM CPU backend calls;
  rounded/<case>/...  pow and exp exactly rounded to F32.

tests/test_step_golden.py compares the CPU restatement and the CUDA step
with both. The fixtures are input-independent of this machine: every case
rebuilds its mesh and forcing from committed code and seeds.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / 'step_golden.npz'
MODES = ('libm', 'rounded')


def _paths():
    for p in (HERE, ROOT / 'tests', ROOT / 'nh-flood-2d_b200', ROOT / 'oracle'):
        if str(p) not in sys.path:
            sys.path.insert(0, str(p))


def run_case(job):
    reference, mode, name = job
    _paths()
    import ti_standin
    from reference_step import ReferenceKernels, ReferenceStepEngine
    import step_cases
    ti_standin.set_math(mode)
    kernels = ReferenceKernels(reference)
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as work:
        result = step_cases.record_case(name, Path(work) / name,
                                        lambda arrays, params: ReferenceStepEngine(kernels, arrays, params))
    seconds = time.perf_counter() - t0
    trace = result['trace']
    steps = int((trace[:, 3] == 1).sum())
    print(f'{mode:8s} {name:32s} {steps:6d} steps {seconds:7.1f} s', flush=True)
    return mode, name, result, steps, seconds


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=os.environ.get('NHF_REFERENCE'),
                    help='a checkout of nh-flood-2d (or set NHF_REFERENCE)')
    ap.add_argument('--jobs', type=int, default=os.cpu_count() or 1)
    ap.add_argument('--cases', nargs='*')
    args = ap.parse_args()
    if not args.reference:
        ap.error('give --reference PATH or set NHF_REFERENCE')
    _paths()
    import step_cases
    names = args.cases or list(step_cases.CASES)
    jobs = [(args.reference, mode, name) for mode in MODES for name in names]
    # the longest cases first, so the pool stays busy
    order = {'quadtree_small': 0, 'uniform_64': 1, 'dambreak_48': 2, 'tidal_basin_3600s': 3}
    jobs.sort(key=lambda j: order.get(j[2], 9))
    arrays = dict(np.load(OUT)) if OUT.exists() and args.cases else {}
    meta = {}
    with mp.get_context('spawn').Pool(min(args.jobs, len(jobs))) as pool:
        for mode, name, result, steps, seconds in pool.imap_unordered(run_case, jobs):
            for key, value in result.items():
                arrays[f'{mode}/{name}/{key}'] = value
            meta[f'{mode}/{name}'] = dict(steps=steps, seconds=round(seconds, 1))
    np.savez_compressed(OUT, **arrays)
    info = HERE / 'step_golden.json'
    old = json.loads(info.read_text()) if info.exists() and args.cases else {}
    old.update(meta)
    info.write_text(json.dumps(dict(sorted(old.items())), indent=1) + '\n')
    print(f'wrote {OUT} ({OUT.stat().st_size} bytes)')


if __name__ == '__main__':
    main()
