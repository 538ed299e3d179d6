"""The step clock (two u32 words of 2**-40 s ticks), on the CPU restatement
of the device clock and the host mirror: the reference's tests/test_clock.py
cases, driven with a pinned CFL candidate before every batch."""
from fractions import Fraction

import numpy as np
import pytest

from engine import OracleEngine
from nhflood.clock import BAD_CFL, COMPLETED, DONE, HostClock
from nhflood.model import StepParams
from nhflood.workloads import dambreak

SCALE = 1 << 40


def end_ticks(row):
    return (int(row[1]) << 32) | int(row[2])


def dt_of(row):
    return np.array([row[0]], np.uint32).view(np.float32)[0]


class Clocked:
    """A dry 4 x 4 grid whose steps take a given CFL candidate."""

    def __init__(self, initial, batch_size, min_dt=1e-4):
        w = dambreak(n=4, duration=10)
        w.initial_depth = None
        self.host = HostClock(initial, batch_size=batch_size, min_dt=min_dt)
        params = StepParams(batch_size=batch_size, min_dt=float(np.float32(min_dt)))
        self.eng = OracleEngine(w.step_arrays(), params, threads=1)
        self.eng.initialize()
        self.eng.set_clock(np.array([self.host.now_ticks >> 32, self.host.now_ticks & 0xffffffff], np.uint32))
        self.eng.set_active(1)
        self.eng.set_forcing(np.zeros((1, 2), np.float32), np.zeros(self.eng.arrays.n_rates, np.float32), False)

    def batch(self, target, origin, candidate):
        t, o = self.host.begin(target, origin)
        self.eng.set_ndt(candidate)
        rows = self.eng.run_batch(t, o)
        self.host.read_trace(rows)
        return rows


def test_regular_f32_dt_is_encoded_exactly_and_traced():
    c = Clocked(0., 2)
    rows = c.batch(1., 0., 0.2)
    assert rows[0, 3] == COMPLETED
    expected = Fraction.from_float(float(np.float32(0.2))) * SCALE
    assert expected.denominator == 1 and end_ticks(rows[0]) == expected.numerator
    assert dt_of(rows[0]) == np.float32(0.2)
    assert c.host.host_now_seconds >= float(np.float32(0.2))


def test_short_event_below_min_dt_uses_a_positive_physical_step():
    initial = 169199.9999999
    c = Clocked(initial, 2)
    rows = c.batch(169200., initial, 0.25)
    assert rows[0, 3] == COMPLETED
    assert 0. < dt_of(rows[0]) < 1e-4
    assert rows[1, 3] == DONE
    assert c.host.host_now_seconds == 169200.


def test_two_word_carry_and_exact_batch_origin():
    initial = 1 / 256 - 0.0002
    c = Clocked(initial, 1)
    first = c.batch(initial + 0.0005, initial, 0.0005)[0]
    assert first[3] == COMPLETED
    assert first[1] == 1 and first[2] > 0  # 2**32 ticks = 1/256 s carried into the high word
    assert c.host.now_ticks == end_ticks(first)
    target, origin = c.host.begin(c.host.host_now_seconds + 0.001, c.host.host_now_seconds)
    np.testing.assert_array_equal(origin, np.array(first[1:3], np.uint32))


@pytest.mark.parametrize('initial, expected_snap', [(169199.7999991, True), (169199.7999989, False)])
def test_snap_threshold_is_checked_without_a_zero_length_update(initial, expected_snap):
    c = Clocked(initial, 1)
    row = c.batch(169200., initial, 0.2)[0]
    assert row[3] == COMPLETED
    assert (end_ticks(row) == 169200 * SCALE) is expected_snap


def test_bad_cfl_stops_batch_before_physics_or_clock_advance():
    c = Clocked(0., 2)
    row = c.batch(1., 0., 5e-5)[0]
    assert row[3] == BAD_CFL
    assert c.host.host_now_seconds == 0.


def test_target_already_reached_produces_only_unused_trace_slots():
    c = Clocked(47 * 3600., 2)
    rows = c.batch(47 * 3600., 47 * 3600., 0.25)
    assert not rows.any()
    assert c.host.host_now_seconds == 47 * 3600.


def test_47h_end_step_preserves_actual_dt_and_exact_event_tick():
    initial = 47 * 3600. - 0.25
    c = Clocked(initial, 1)
    row = c.batch(47 * 3600., initial, 0.25)[0]
    assert dt_of(row) == np.float32(0.25)
    assert end_ticks(row) == 47 * 3600 * SCALE
    assert c.host.host_now_seconds == 47 * 3600.


def test_host_rejects_out_of_range_clock_and_stale_batch_origin():
    with pytest.raises(ValueError):
        HostClock(-1.)
    with pytest.raises(ValueError):
        HostClock(194.181 * 86400.)
    clock = HostClock(1.)
    with pytest.raises(ValueError):
        clock.begin(2., 0.)
    clock.begin(2., 1.)
    with pytest.raises(RuntimeError):
        clock.begin(2., 1.)


def test_sub_microsecond_candidate_rounds_to_nearest_even_tick():
    small = np.nextafter(np.float32(2 ** -20), np.float32(1.0))
    exact = Fraction.from_float(float(small)) * SCALE
    assert exact.denominator > 1
    c = Clocked(0., 1, min_dt=float(small))
    row = c.batch(1., 0., float(small))[0]
    assert row[3] == COMPLETED
    assert end_ticks(row) == round(exact)
    assert abs(end_ticks(row) / SCALE - float(small)) <= 0.5 / SCALE
