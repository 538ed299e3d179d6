"""Host mirror of the two-U32 fixed-point device clock (2**-40 s per tick).

The device side (dt choice, tick conversion, snapping, commit) runs inside
the step kernels; this module keeps the host protocol of the reference's
StepClock (core/clock.py:14-28,48-92,187-203): exact seconds -> ticks with
round-half-even, batch begin checks and the trace read-back that advances
the exact host copy of the clock.
"""
from __future__ import annotations

import math

import numpy as np

TICKS_PER_SECOND = 1 << 40
MAX_TICKS = (1 << 64) - 1
DONE, COMPLETED, BAD_CFL, BAD_DT, OVERSHOOT = 0, 1, 2, 3, 4


def seconds_to_ticks(seconds: float) -> int:
    """Exact conversion of a finite nonnegative F64 to ticks, half to even."""
    seconds = float(seconds)
    if not math.isfinite(seconds) or seconds < 0:
        raise ValueError('Clock seconds must be finite and nonnegative')
    num, den = seconds.as_integer_ratio()
    q, r = divmod(num * TICKS_PER_SECOND, den)
    if 2 * r > den or (2 * r == den and q & 1):
        q += 1
    if q > MAX_TICKS:
        raise ValueError('Clock exceeds the two-U32 range')
    return q


def words(ticks: int) -> np.ndarray:
    return np.array([ticks >> 32, ticks & 0xffffffff], dtype=np.uint32)


def ticks_of(hi, lo) -> int:
    return (int(hi) << 32) | int(lo)


class HostClock:
    """Exact host copy of the device clock and the batch protocol."""

    def __init__(self, initial_seconds: float, batch_size: int = 32, min_dt: float = 1e-4):
        if not isinstance(batch_size, int) or not 1 <= batch_size <= 64:
            raise ValueError('batch_size must be between 1 and 64')
        if not math.isfinite(min_dt) or not 0 < min_dt <= 1:
            raise ValueError('min_dt must be finite and in (0, 1]')
        self.batch_size = batch_size
        self.min_dt = float(np.float32(min_dt))
        if self.min_dt <= 0:
            raise ValueError('min_dt rounds to zero in F32')
        self.now_ticks = seconds_to_ticks(initial_seconds)
        self.pending = False

    @property
    def host_now_seconds(self) -> float:
        return self.now_ticks / TICKS_PER_SECOND

    def begin(self, target_seconds: float, batch_origin_seconds: float):
        """Return (target words, origin words) for the next device batch."""
        if self.pending:
            raise RuntimeError('Read the previous batch trace before begin')
        if not math.isfinite(batch_origin_seconds) or abs(batch_origin_seconds - self.host_now_seconds) >= 1e-6:
            raise ValueError('batch_origin_seconds differs from the last end tick')
        target = seconds_to_ticks(target_seconds)
        if target < self.now_ticks:
            raise ValueError('Target precedes the current clock')
        self.pending = True
        return words(target), words(self.now_ticks)

    def read_trace(self, rows: np.ndarray) -> np.ndarray:
        """Advance the host clock over completed rows of a batch trace."""
        if not self.pending:
            raise RuntimeError('Call begin before reading a trace')
        # rows complete up to the first other status, which ends the batch
        status = np.asarray(rows)[:, 3]
        stops = np.flatnonzero(status != COMPLETED)
        n = int(stops[0]) if len(stops) else len(rows)
        if n:
            self.now_ticks = ticks_of(rows[n - 1][1], rows[n - 1][2])
        # an unknown status is refused after the completed rows before it
        # have advanced the clock, and the batch stays pending
        if n < len(rows) and int(status[n]) not in (BAD_CFL, BAD_DT, OVERSHOOT, DONE):
            raise RuntimeError(f'Unknown clock trace status {int(status[n])}')
        self.pending = False
        return rows
