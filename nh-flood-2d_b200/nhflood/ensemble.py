"""Batched form: many scenarios of uneven mesh size advanced together.

Each scenario is a ``PlainRun`` (its own engine, clock, forcing, budget,
extrema: the reference's per-run state, solver_compact.py:179-1008);
``CudaEnsemble`` runs one batch of every scenario per call. A scenario that
has reached its end time keeps taking part with a target equal to its clock,
which the device clock turns into an empty batch (status DONE), so scenarios
of different durations share a batch.

Two schedules. Member graphs (the default): every scenario's engine makes the
plain form's own choice of step form, tile size and CFL placement, and all
scenarios' batch graphs are launched together on their own streams, so small
scenarios fill the GPU beside large ones. One launch: every scenario on the
fused step with one tile size, ONE step launch per slot for all of them; its
tile size and grid (persistent blocks or one block per tile) come from
``nhflood.autotune`` unless given.
"""
from __future__ import annotations

import numpy as np

from .native import CudaEngine, CudaEnsemble
from .plain import PlainRun


def tiled_factory(tile: int, device: str = 'cuda:0', cfl: str = 'pass'):
    """Engines on the fused step with this tile size. Ensemble members take
    the separate CFL pass (one launch for all members per step); a plain run
    may pass cfl='auto'."""
    def factory(arrays, params):
        params.path = f'tile{tile}'
        params.cfl = cfl
        engine = CudaEngine(arrays, params, device=device)
        if not engine.path.startswith('tiled'):
            engine.close()
            raise RuntimeError(f'mesh does not take the fused step with tile {tile}: {engine.path}')
        return engine
    return factory


MEMBER_GRAPHS = -2  # nhf_ensemble_create's grid_blocks for the member-graph schedule


def plain_factory(device: str = 'cuda:0'):
    """Engines with the plain form's own step choice."""
    def factory(arrays, params):
        return CudaEngine(arrays, params, device=device)
    return factory


class EnsembleRun:
    """grid_blocks = -2: the member graphs. A tile size and/or a grid: the
    one-launch schedule, the autotuner filling in what is not given. Neither
    (tune=True): the autotuner's choice among all of them; with tune=False
    the member graphs."""

    def __init__(self, workloads, *, tile: int | None = None, grid_blocks: int | None = None,
                 batch_size: int = 32, device: str = 'cuda:0', tuning_cache=None, tune: bool = False,
                 engine_factory=None, ensemble_factory=None):
        """engine_factory(arrays, params) and ensemble_factory(engines,
        grid_blocks) replace the schedule's CUDA engines and CudaEnsemble
        (the CPU tests of the batching logic pass the CPU restatement and a
        sequential stand-in)."""
        self.workloads = list(workloads)
        self.tuned = None
        if tile is None and grid_blocks is None and tune:
            from .autotune import choose_schedule
            self.tuned = choose_schedule(self.workloads, batch_size=batch_size, device=device, cache=tuning_cache)
            tile, grid_blocks = (None, MEMBER_GRAPHS) if self.tuned.grid == MEMBER_GRAPHS else \
                (self.tuned.tile, self.tuned.grid)
        if grid_blocks == MEMBER_GRAPHS or (tile is None and grid_blocks is None):
            self.schedule = 'member graphs'
            tile, grid_blocks = None, MEMBER_GRAPHS
            factory = plain_factory(device)
        else:
            self.schedule = 'one launch'
            if tile is None or grid_blocks is None:
                from .autotune import choose_schedule
                tuned = choose_schedule(self.workloads, batch_size=batch_size, device=device, cache=tuning_cache,
                                        member_graphs_fn=lambda *a: None)
                tile = tuned.tile if tile is None else tile
                grid_blocks = tuned.grid if grid_blocks is None else grid_blocks
            factory = tiled_factory(tile, device)
        self.tile, self.grid_blocks = tile, grid_blocks
        factory = engine_factory or factory
        self.runs = [PlainRun(w, factory, batch_size=batch_size) for w in self.workloads]
        try:
            self.ensemble = (ensemble_factory or CudaEnsemble)([r.engine for r in self.runs], grid_blocks)
        except Exception:
            for r in self.runs:
                r.close()
            raise
        self.cells = np.array([w.cells for w in self.workloads], np.int64)
        self.h2d_bytes = 0

    @property
    def done(self) -> bool:
        return all(r.done for r in self.runs)

    def begin(self):
        targets, origins = [], []
        self.h2d_bytes = 0
        for r in self.runs:
            if r.done:
                now = r.clock.host_now_seconds
                t, o = r.clock.begin(now, now)
            else:
                t, o = r.begin()
                self.h2d_bytes += r.h2d_bytes
            targets.append(t)
            origins.append(o)
        self.h2d_bytes += 16 * len(self.runs)
        return np.array(targets, np.uint32), np.array(origins, np.uint32)

    def finish(self, traces) -> np.ndarray:
        """Consume one ensemble trace; returns completed steps per scenario."""
        return np.array([r.finish(traces[i]) for i, r in enumerate(self.runs)], np.int64)

    def advance(self) -> np.ndarray:
        targets, origins = self.begin()
        return self.finish(self.ensemble.run_batch(targets, origins))

    def cell_updates(self, completed) -> int:
        return int((np.asarray(completed, np.int64) * self.cells).sum())

    def close(self):
        self.ensemble.close()
        for r in self.runs:
            r.close()
