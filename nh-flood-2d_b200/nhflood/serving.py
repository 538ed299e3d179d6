"""Served form: a request loop with continuous batching under an HBM budget.

Requests (flood solves of different mesh sizes) arrive over time. The server
admits a waiting request as soon as its device-memory estimate fits the
budget next to the resident ones (first come, first served), keeps every
admitted solve's state resident on the GPU, and advances all of them
together: each scheduling round is ONE ensemble batch (``CudaEnsemble``:
one fused step launch per slot for all resident solves, each with its own
clock and CFL dt). Solves admitted while a batch runs are built on a side
stream, so their upload and set-up overlap the batch; a solve that reaches
its end time is retired at the end of the round with its final depth and
max-depth (extrema) frames, and its memory goes back to the budget.

Admitted solves are built (arrays, upload, tile plan) by a builder thread on
its own stream, so the scheduling loop keeps launching rounds for the
resident solves meanwhile; a finished build joins at the next round.

Every solve runs the same arithmetic as the plain single run (the ensemble
step is the plain step per member), so a result does not depend on what
else was resident: alone and in the mix are bit-identical.
"""
from __future__ import annotations

import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .ensemble import MEMBER_GRAPHS, plain_factory, tiled_factory
from .plain import PlainRun


def device_bytes_estimate(arrays) -> int:
    """Device bytes one resident solve holds: its uploaded inputs, the
    state (bed, depth, q, rain_time, infiltration, extrema, u, v, peak
    words), and the library scratch of the fused step (centre distances,
    donor factors, face fluxes, second state buffers, budget partials, tile
    plan)."""
    e, s = arrays.e_num, arrays.s_num
    state = 4 * (10 * e + s)
    scratch = 4 * (s + e + 4 * e + 2 * e + s) + 16 * ((e + 255) // 256) * arrays.terms
    plan = 24 * e + 64 * 1024
    return int(arrays.nbytes() + state + scratch + plan + (1 << 20))


def device_bytes_bound(workload) -> int:
    """An upper bound of device_bytes_estimate from the mesh sizes alone
    (before the step arrays are built): hanging-edge tables counted as if
    every side had one."""
    m = workload.mesh
    e, s, isl = m.e_num, m.s_num, len(m.isl_data)
    terms = 4 + 6 * len(workload.forcing.boundaries)
    inputs = 4 * (12 * e + 8 * e + isl) + 21 * s + 16 * e + 44 * s
    state = 4 * (10 * e + s)
    scratch = 4 * (s + e + 4 * e + 2 * e + s) + 16 * ((e + 255) // 256) * terms
    return int(inputs + state + scratch + 24 * e + 64 * 1024 + (1 << 20))


@dataclass
class Request:
    id: int
    arrival: float                 # seconds after the session start
    workload: object               # nhflood.workloads.Workload, or a Future of one
    arrays: object = None          # its StepArrays, built on first need
    need: int = 0                  # device bytes estimate
    cells: int = 0

    def resolve(self):
        """The workload, waiting for it if it is still being made."""
        if hasattr(self.workload, 'result'):
            self.workload = self.workload.result()
        self.cells = self.workload.cells
        return self.workload

    def prepare(self):
        if self.arrays is None:
            self.arrays = self.resolve().step_arrays()
            self.need = device_bytes_estimate(self.arrays)
        return self.need

    def release(self):
        """Drop the host copies once a run holds what it needs."""
        self.workload = None
        self.arrays = None


class MadeAhead:
    """The workloads of a request stream, made by an executor (a process
    pool) in arrival order and only ``ahead`` requests beyond the last one
    taken, so that host memory holds a window of the stream, not all of it.
    ``requests`` gives Request objects whose workload is a ticket that
    waits for its own future when the server first needs it."""

    def __init__(self, make, stream, executor, ahead: int = 32):
        self.make, self.stream, self.executor, self.ahead = make, list(stream), executor, max(1, ahead)
        self.futures = {}
        self.submitted = 0
        self._fill(0)

    def _fill(self, upto: int) -> None:
        while self.submitted < len(self.stream) and self.submitted < upto + self.ahead:
            self.futures[self.submitted] = self.executor.submit(self.make, self.stream[self.submitted]['params'])
            self.submitted += 1

    def take(self, index: int):
        self._fill(index + 1)
        return self.futures.pop(index).result()

    def wait_first(self) -> None:
        """Block until the first window is made (before a timed session)."""
        for f in list(self.futures.values()):
            f.result()

    def requests(self) -> list[Request]:
        return [Request(r['id'], r['arrival'], _Ticket(self, i)) for i, r in enumerate(self.stream)]


class _Ticket:
    def __init__(self, source: MadeAhead, index: int):
        self.source, self.index = source, index

    def result(self):
        return self.source.take(self.index)


@dataclass
class Completed:
    id: int
    arrival: float
    admitted: float
    finished: float
    cells: int
    steps: int
    device_bytes: int
    depth: np.ndarray = field(repr=False)
    max_depth: np.ndarray = field(repr=False)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def cell_updates(self) -> int:
        return self.cells * self.steps


class FloodServer:
    def __init__(self, *, hbm_budget: float = 150e9, tile: int = 256, grid_blocks: int = -2,
                 batch_size: int = 32, device: str = 'cuda:0', clock=None, engine_factory=None,
                 ensemble_factory=None):
        """engine_factory(arrays, params) and ensemble_factory(engines,
        grid_blocks) replace the CUDA step and CudaEnsemble (the scheduling
        logic's CPU tests pass the CPU restatement and a sequential stand-in);
        a device that is not CUDA gets no side stream."""
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.budget = float(hbm_budget)
        self.tile, self.grid_blocks, self.batch_size = tile, grid_blocks, batch_size
        self.engine_factory, self.ensemble_factory = engine_factory, ensemble_factory
        self.side = torch.cuda.Stream(self.device) if self.device.type == 'cuda' else None
        self.waiting: deque[Request] = deque()
        self.building: deque = deque()  # (request, future of its PlainRun, bytes reserved)
        self.builder = ThreadPoolExecutor(max_workers=1, thread_name_prefix='nhflood-build')
        self.active: list[tuple[Request, PlainRun, int, float]] = []  # request, run, bytes, admitted at
        self.used = 0
        self.peak_used = 0
        self.ensemble = None
        self.dirty = False
        self.rounds = 0
        self.clock = clock or time.perf_counter
        self.t0 = self.clock()

    def now(self) -> float:
        return self.clock() - self.t0

    @property
    def busy(self) -> bool:
        return bool(self.waiting or self.building or self.active)

    def submit(self, request: Request) -> None:
        self.waiting.append(request)

    # -- admission and retirement ------------------------------------------
    def _admit(self) -> int:
        """Start building waiting requests, first come first served, while
        their memory bound fits the budget next to what is resident or
        being built."""
        started = 0
        while self.waiting:
            req = self.waiting[0]
            need = device_bytes_bound(req.resolve())
            if need > self.budget:
                raise ValueError(f'request {req.id} needs {need} B, more than the whole budget')
            if self.used + need > self.budget:
                break
            self.waiting.popleft()
            self.used += need
            self.peak_used = max(self.peak_used, self.used)
            self.building.append((req, self.builder.submit(self._build, req), need))
            started += 1
        return started

    def _build(self, req):
        """Builder thread: the solve's arrays, upload and plan on the side stream."""
        # member graphs (grid_blocks -2): the plain form's own step choice;
        # one launch: the fused step with the server's tile size
        factory = self.engine_factory or (plain_factory(str(self.device)) if self.grid_blocks == MEMBER_GRAPHS
                                          else tiled_factory(self.tile, str(self.device)))
        if self.side is None:
            run = PlainRun(req.workload, factory, batch_size=self.batch_size, arrays=req.arrays)
        else:
            with self.torch.cuda.device(self.device), self.torch.cuda.stream(self.side):
                run = PlainRun(req.workload, factory, batch_size=self.batch_size, arrays=req.arrays)
            self.side.synchronize()
        req.release()  # the run holds the workload, the engine the device copy
        return run

    def _join_built(self, wait: bool) -> None:
        """Finished builds join the resident set (in admission order); with
        wait, block for the first one when nothing else can run."""
        while self.building and (self.building[0][1].done() or wait):
            req, future, bound = self.building.popleft()
            run = future.result()
            need = device_bytes_estimate(run.arrays)
            self.used += need - bound
            self.active.append((req, run, need, self.now()))
            self.dirty = True
            wait = False

    def _retire(self) -> list[Completed]:
        done, keep = [], []
        for item in self.active:
            req, run, need, admitted = item
            if not run.done:
                keep.append(item)
                continue
            depth = run.engine.get('depth')
            max_depth = run.engine.get('max_depth')
            done.append(Completed(req.id, req.arrival, admitted, self.now(), run.w.cells, run.steps, need,
                                  depth, max_depth))
            run.close()
            self.used -= need
            self.dirty = True
        self.active = keep
        return done

    def _ensemble(self):
        from .native import CudaEnsemble
        if self.dirty or self.ensemble is None:
            if self.ensemble is not None:
                self.ensemble.close()
            make = self.ensemble_factory or CudaEnsemble
            self.ensemble = make([run.engine for _, run, _, _ in self.active], self.grid_blocks)
            self.dirty = False
        return self.ensemble

    # -- one scheduling round ------------------------------------------------
    def step(self) -> list[Completed]:
        """Launch one batch of every resident solve, admit waiting requests
        while it runs, then consume the traces and retire finished solves."""
        launched = None
        if self.active:
            ens = self._ensemble()
            targets, origins = [], []
            for _, run, _, _ in self.active:
                t, o = run.begin()
                targets.append(t)
                origins.append(o)
            ens.run_batch_async(np.array(targets), np.array(origins))
            launched = ens
        self._admit()
        if launched is not None:
            traces = launched.read_trace()
            for i, (_, run, _, _) in enumerate(self.active[:launched.members]):
                run.finish(traces[i])
            self.rounds += 1
        self._join_built(wait=launched is None)
        return self._retire()

    def close(self):
        for _, future, _ in self.building:
            future.result().close()
        self.building.clear()
        self.builder.shutdown(wait=True)
        if self.ensemble is not None:
            self.ensemble.close()
            self.ensemble = None
        for _, run, _, _ in self.active:
            run.close()
        self.active = []


def serve(requests, server: FloodServer, realtime: bool = True) -> list[Completed]:
    """Replay an arrival stream (sorted by arrival) against the server; in
    real time, requests are submitted when the session clock reaches their
    arrival. Returns the completed solves in completion order."""
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    out: list[Completed] = []
    while pending or server.busy:
        now = server.now()
        while pending and (pending[0].arrival <= now or not realtime):
            server.submit(pending.popleft())
        if not server.busy:
            time.sleep(min(0.05, max(0.0, pending[0].arrival - now)))
            continue
        out.extend(server.step())
    return out


def serve_sequential(requests, *, tile: int = 256, batch_size: int = 32, device: str = 'cuda:0',
                     realtime: bool = True, clock=None, engine_factory=None) -> list[Completed]:
    """The plain form, one solve at a time in arrival order (the baseline of
    the served form): each request waits for the previous one to finish."""
    clock = clock or time.perf_counter
    t0 = clock()
    out = []
    for req in sorted(requests, key=lambda r: r.arrival):
        if realtime:
            wait = req.arrival - (clock() - t0)
            if wait > 0:
                time.sleep(wait)
        started = clock() - t0
        run = PlainRun(req.resolve(), engine_factory or tiled_factory(tile, device, cfl='auto'), batch_size=batch_size)
        req.release()
        while not run.done:
            run.advance()
        out.append(Completed(req.id, req.arrival, started, clock() - t0, run.w.cells, run.steps,
                             device_bytes_estimate(run.arrays), run.engine.get('depth'), run.engine.get('max_depth')))
        run.close()
    return out


def latency_summary(done: list[Completed]) -> dict:
    lat = np.array([c.latency for c in done])
    return {'p50_s': float(np.percentile(lat, 50)), 'p95_s': float(np.percentile(lat, 95)),
            'p99_s': float(np.percentile(lat, 99)), 'mean_s': float(lat.mean()), 'count': len(done)}
