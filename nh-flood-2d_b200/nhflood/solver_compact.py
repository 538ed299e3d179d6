"""Public entry points with the reference's names and semantics
(nh-flood-2d src/nh_flood_2d/core/solver_compact.py:152-176,1011-1016)."""
from __future__ import annotations

from .engine import evolve
from .preprocess import preprocess
from .run_record import RunRecord


def run_simulation(domain_cfg, force_cfg, pipe_cfg=None, *, engine_factory=None):
    """Preprocess and simulate, recording failures from either stage."""
    with RunRecord(domain_cfg, force_cfg, pipe_cfg) as record:
        record.hash_inputs(domain_cfg, force_cfg, pipe_cfg)
        preprocess(domain_cfg, force_cfg)
        return _solve(domain_cfg, force_cfg, record, pipe_cfg, engine_factory=engine_factory)


def solver(domain_cfg, force_cfg, pipe_cfg=None, *, engine_factory=None):
    """Simulate an already preprocessed domain, including configured warmup."""
    with RunRecord(domain_cfg, force_cfg, pipe_cfg) as record:
        record.hash_inputs(domain_cfg, force_cfg, pipe_cfg)
        return _solve(domain_cfg, force_cfg, record, pipe_cfg, engine_factory=engine_factory)


def warmup_solver(domain_cfg, force_cfg, pipe_cfg=None, *, engine_factory=None):
    """Run an already preprocessed domain through warmup, stopping at start."""
    with RunRecord(domain_cfg, force_cfg, pipe_cfg) as record:
        record.data.update(run_kind='warmup', simulation_end=domain_cfg.start.isoformat())
        record.hash_inputs(domain_cfg, force_cfg, pipe_cfg)
        return _solve(domain_cfg, force_cfg, record, pipe_cfg, end_time=0., engine_factory=engine_factory)


def _solve(domain_cfg, force_cfg, record, pipe_cfg=None, end_time=None, *, engine_factory=None):
    end_time = domain_cfg.duration if end_time is None else end_time
    if pipe_cfg is not None:
        raise NotImplementedError('SWMM pipe coupling is not part of this engine')
    return evolve(domain_cfg, force_cfg, record, None, end_time, engine_factory=engine_factory)
