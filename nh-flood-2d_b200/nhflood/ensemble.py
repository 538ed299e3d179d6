"""Batched form: many scenarios of uneven mesh size advanced together.

Each scenario is a ``PlainRun`` (its own engine, clock, forcing, budget,
extrema: the reference's per-run state, solver_compact.py:179-1008) on the
fused tiled step; ``CudaEnsemble`` runs one batch of every scenario as one
CUDA graph with ONE fused step launch per slot for all of them. A scenario
that has reached its end time keeps taking part with a target equal to its
clock, which the device clock turns into an empty batch (status DONE), so
scenarios of different durations share the graph.

The tile size and the grid schedule (persistent blocks or one block per
tile) come from ``nhflood.autotune`` unless given.
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


class EnsembleRun:
    def __init__(self, workloads, *, tile: int | None = None, grid_blocks: int | None = None,
                 batch_size: int = 32, device: str = 'cuda:0', tuning_cache=None):
        self.workloads = list(workloads)
        if tile is None or grid_blocks is None:
            from .autotune import choose_schedule
            schedule = choose_schedule(self.workloads, batch_size=batch_size, device=device, cache=tuning_cache)
            tile = schedule.tile if tile is None else tile
            grid_blocks = schedule.grid if grid_blocks is None else grid_blocks
        self.tile, self.grid_blocks = tile, grid_blocks
        self.runs = [PlainRun(w, tiled_factory(tile, device), batch_size=batch_size) for w in self.workloads]
        self.ensemble = CudaEnsemble([r.engine for r in self.runs], grid_blocks)
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
