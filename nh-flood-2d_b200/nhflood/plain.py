"""The plain single-run solver as a step-by-batch object, without output I/O.

``PlainRun`` prepares an engine exactly as the time loop does (initialize,
seed state, initial levels, first CFL, initial diagnostics, extrema reset)
and then advances one device batch per ``advance()`` call. Batch targets
follow the time loop's rule (solver_compact.py:930-937): the next yield
output, the next 900 s frame, the next forcing event and the end time, so the
dt sequence is the one a full run produces. Outputs (frames, CSVs,
checkpoints) are skipped: they are host I/O outside the step.
"""
from __future__ import annotations

import bisect

import numpy as np

from .clock import COMPLETED, DONE, TICKS_PER_SECOND, HostClock, seconds_to_ticks, ticks_of, words
from .model import STATE_F32, STATE_U32, StepParams

FRAME = 900


class PlainRun:
    def __init__(self, workload, engine_factory, batch_size: int = 32, arrays=None):
        self.w = workload
        self.params = StepParams(afa=workload.afa, sita=workload.sita, min_h=workload.min_h, batch_size=batch_size)
        self.arrays = workload.step_arrays() if arrays is None else arrays
        self.engine = engine_factory(self.arrays, self.params)
        self.clock = HostClock(0.0, batch_size=batch_size)
        eng = self.engine
        eng.set_clock(words(0))
        eng.initialize()
        state = workload.initial_state()
        if state is not None:
            for name in ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed'):
                eng.set(name, getattr(state, name))
        bed = eng.get('bed')
        targets = np.zeros(self.arrays.e_num, np.float32)
        for b in workload.forcing.boundaries:
            if b.kind == 'level':
                targets[b.cells] = np.maximum(b.series.at(0.) - bed[b.cells].astype(float), 0.)
        eng.apply_initial_levels(targets)
        eng.set_active(1)
        if self.arrays.gate is not None:
            eng.gate_check()  # check_gates before the first CFL (solver_compact.py:885-888)
        eng.compute_cfl()
        eng.initial_diagnostics()
        eng.reset_extrema()
        self.elapsed = 0.0
        self.next_output = float(min(workload.yield_step, workload.duration))
        self.next_frame = float(min(FRAME, workload.duration))
        self.event_ticks = sorted(seconds_to_ticks(float(t)) for t in workload.forcing.events
                                  if 0 <= t <= workload.duration)
        self.event_samples = {seconds_to_ticks(float(t)): float(t) for t in workload.forcing.events}
        self.rain_index = -1
        self.coefficients = np.zeros((max(1, len(workload.forcing.boundaries)), 2), np.float32)
        self.steps = 0
        self.pending = None
        self.h2d_bytes = 0

    @property
    def done(self) -> bool:
        return self.elapsed >= self.w.duration

    def forcing_inputs(self):
        """(coefficients, rain rates or None, raining) for the next batch."""
        sample = self.event_samples.get(seconds_to_ticks(self.clock.host_now_seconds), self.elapsed)
        f = self.w.forcing
        for bi, b in enumerate(f.boundaries):
            i = min(int(np.searchsorted(b.series.times, sample, side='right')) - 1, len(b.series.times) - 2)
            self.coefficients[bi, 0] = b.series.at(sample)
            self.coefficients[bi, 1] = ((b.series.values[i + 1] - b.series.values[i])
                                        / (b.series.times[i + 1] - b.series.times[i]))
        rates = None
        index = f.rain.index_at(sample)
        if index != self.rain_index:
            rates = f.rain.rates(index).astype(np.float32)
            self.rain_index = index
        return self.coefficients, rates, True

    def target(self) -> float:
        t = min(self.next_output, self.next_frame, float(self.w.duration))
        i = bisect.bisect_right(self.event_ticks, seconds_to_ticks(self.clock.host_now_seconds))
        if i < len(self.event_ticks):
            t = min(t, self.event_ticks[i] / TICKS_PER_SECOND)
        return t

    def begin(self):
        coef, rates, raining = self.forcing_inputs()
        self.engine.set_forcing(coef, rates, raining)
        self.h2d_bytes = coef.nbytes + (rates.nbytes if rates is not None else 0) + 4 + 16
        return self.clock.begin(self.target(), self.clock.host_now_seconds)

    def finish(self, rows) -> int:
        """Consume a batch trace; returns completed steps."""
        self.clock.read_trace(rows)
        status = rows[:, 3]
        stops = np.flatnonzero(status != COMPLETED)
        completed = int(stops[0]) if len(stops) else len(rows)
        if completed:
            last = rows[completed - 1]
            self.elapsed = ticks_of(last[1], last[2]) / TICKS_PER_SECOND
        if completed < len(rows) and int(status[completed]) != DONE:
            raise RuntimeError(f'Device clock status {int(status[completed])} at {self.elapsed}s')
        self.steps += completed
        if abs(self.elapsed - self.next_output) < 1e-9 or self.elapsed == self.w.duration:
            self.next_output = min(self.next_output + self.w.yield_step, float(self.w.duration))
        if abs(self.elapsed - self.next_frame) < 1e-9 or self.elapsed == self.w.duration:
            self.next_frame = min(self.next_frame + FRAME, float(self.w.duration))
        return completed

    def adopt(self, other: 'PlainRun') -> None:
        """Continue from another run of the same workload, on another engine:
        its state arrays, clock and batch bookkeeping; the next CFL candidate
        is recomputed from the adopted state (as the step itself computes it)."""
        for name in STATE_F32 + STATE_U32:
            self.engine.set(name, other.engine.get(name))
        if self.arrays.gate is not None:
            self.engine.set_gate_state(other.engine.gate_state())
        self.engine.set_clock(other.engine.get_clock())
        self.clock.now_ticks = other.clock.now_ticks
        self.elapsed, self.steps = other.elapsed, other.steps
        self.next_output, self.next_frame = other.next_output, other.next_frame
        self.rain_index = -1  # upload the rain rates with the next batch
        self.engine.compute_cfl()

    def advance(self) -> int:
        """One synchronous batch through the public engine call."""
        if self.done:
            return 0
        target_words, origin_words = self.begin()
        return self.finish(self.engine.run_batch(target_words, origin_words))

    def close(self):
        self.engine.close()
