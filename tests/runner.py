"""Run a case through the real time loop on the oracle or the CUDA engine."""
from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from nhflood.output import read_checkpoint
from nhflood.preprocess import preprocess
from nhflood.run_record import RunRecord
from nhflood.solver_compact import _solve


def oracle_factory(arrays, params):
    from engine import OracleEngine  # oracle/engine.py
    return OracleEngine(arrays, params)


class SequentialEnsemble:
    """The ensemble launch's contract on CPU engines, one member after
    another: a batch of every member from its own target and origin words,
    one trace per member (what CudaEnsemble returns)."""

    def __init__(self, engines, grid_blocks=None):
        self.engines = list(engines)
        self.members = len(self.engines)
        self.rows = None

    def run_batch_async(self, targets, origins):
        self.rows = [e.run_batch(t, o) for e, t, o in zip(self.engines, targets, origins)]

    def read_trace(self):
        return self.rows

    def run_batch(self, targets, origins):
        self.run_batch_async(targets, origins)
        return self.read_trace()

    def close(self):
        self.engines = []


def cuda_factory(arrays, params):
    from nhflood.native import CudaEngine
    return CudaEngine(arrays, params)


def cuda_multipass_factory(arrays, params):
    from nhflood.native import CudaEngine
    params.path = 'multipass'
    return CudaEngine(arrays, params)


FACTORIES = {'oracle': oracle_factory, 'cuda': cuda_factory, 'cuda_multipass': cuda_multipass_factory}


@dataclass
class Result:
    budget: dict
    record: RunRecord
    state: object
    manifest: dict
    path: Path

    @property
    def trace(self) -> np.ndarray:
        return self.record.trace

    @property
    def h(self):
        return self.state.bed + self.state.depth


def run(dc, fc, engine='oracle', *, end_time=None, warmup_only=False, do_preprocess=True) -> Result:
    if do_preprocess:
        preprocess(dc, fc)
    with RunRecord(dc, fc) as record:
        if warmup_only:
            record.data.update(run_kind='warmup', simulation_end=dc.start.isoformat())
        record.hash_inputs(dc, fc)
        budget = _solve(dc, fc, record, end_time=0. if warmup_only else end_time,
                        engine_factory=FACTORIES[engine] if isinstance(engine, str) else engine)
    out = Path(dc.domain_dir)
    manifest = json.loads((out / 'manifest.json').read_text())
    state = read_checkpoint(out / 'output' / 'state_final.fdb')
    return Result(budget, record, state, manifest, out)
