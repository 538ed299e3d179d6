"""The step against golden vectors from the reference's own kernel source.

tests/golden/step_golden.npz holds, for every case of tests/step_cases.py,
what nh-flood-2d's unchanged step kernels produced when
tests/golden/make_step_golden.py ran them under a serial NumPy stand-in for
Taichi: tick, compute_cfl, prepare_step, finish_step and the other kernels
of core/solver_compact.py:364-641, StepClock.choose/commit
(core/clock.py:94-181), PressureReconstruction (core/pressure.py:65-129)
and DeviceBudget (core/device_budget.py:28-84). Every case is recorded
twice: with the C library's powf/expf ("libm", the functions Taichi's CPU
backend calls) and with pow/exp exactly rounded to F32 ("rounded", the
rounding this project's friction power and Horton exponential give).

The bar of the comparison:
  * "rounded": bit for bit over the whole case. Every trace row (dt bits,
    clock words, status, CFL candidate, event flag, limited cell and face
    counts, minimum donor scale, wet-cell count) and the depth and
    discharge arrays at the end of every batch are identical.
  * "libm": every trace row bit for bit up to the first step where the
    two roundings part, which must come after LIBM_HORIZON_S = 20 s of
    simulated time (or not at all), and depth within 1 mm and discharge
    within 1e-4 m2/s at every batch end before that step. The C library's powf/expf are not exactly rounded (about 7 calls
    in 10,000 are one unit in the last place off), so the two roundings
    part eventually; ``first_difference`` reports where. On the steep
    60 s quadtree case the first differing value is a minimum donor scale
    after 481 identical steps (22.3 s), and the chaotic shock-laden flow
    then grows the gap to centimetres by 60 s, as any second F32 or F64
    rounding of the same scheme does on such terrain.
  * Budget flushes in both: the reference adds F32 values into per-block
    F32 sums (atomic adds) and then exactly; this project adds the same F32
    values in F64. The two agree to the F32 rounding of block sums:
    |a - b| <= 2e-6 * sum |terms| + 1e-9 m3 per flush.
The mesh indexing and face connectivity the step reads are built by the
same committed code on both sides (tests/test_golden_host.py checks them
against the reference's own preprocessing).
"""
from pathlib import Path

import numpy as np
import pytest

import step_cases

GOLDEN = Path(__file__).resolve().parent / 'golden' / 'step_golden.npz'
DEPTH_TOL = 1e-3  # m
Q_TOL = 1e-4      # m2/s
MODES = ('rounded', 'libm')
LIBM_HORIZON_S = 20.0


@pytest.fixture(scope='module')
def golden():
    return np.load(GOLDEN)


def fixture(golden, mode, name):
    return {k: golden[f'{mode}/{name}/{k}'] for k in ('trace', 'depth', 'q', 'budget')}


def first_difference(a, b):
    """(row, column) of the first trace entry that differs, or None."""
    if a.shape != b.shape:
        n = min(len(a), len(b))
        bad = np.argwhere(a[:n] != b[:n])
        return tuple(bad[0]) if len(bad) else (n, -1)
    bad = np.argwhere(a != b)
    return tuple(int(x) for x in bad[0]) if len(bad) else None


def completed(trace):
    return trace[trace[:, 3] == 1]


def end_seconds(rows):
    return (rows[:, 1].astype(np.int64) * 2 ** 32 + rows[:, 2]) / 2 ** 40


def batch_ends(trace, batch=32):
    """Clock tick of each batch's last completed step (None for an empty batch)."""
    out = []
    for rows in trace.reshape(-1, batch, trace.shape[1]):
        done = rows[rows[:, 3] == 1]
        out.append((int(done[-1, 1]) << 32 | int(done[-1, 2])) if len(done) else None)
    return out


def check(got, ref, mode, name):
    """Raise on a difference beyond the bar of ``mode``; return the first
    differing completed-step (row, column), or None."""
    a, b = completed(got['trace']), completed(ref['trace'])
    first = first_difference(a, b)
    if mode == 'rounded':
        assert first is None, (name, first)
        assert got['trace'].shape == ref['trace'].shape, name
        for key in ('depth', 'q'):
            assert got[key].shape == ref[key].shape, (name, key)
            np.testing.assert_array_equal(got[key].view(np.uint32), ref[key].view(np.uint32), err_msg=f'{name} {key}')
    else:
        times = end_seconds(b)
        until = float('inf')
        if first is not None:
            until = times[min(first[0], len(times) - 1)]  # the step where the roundings part
            assert until > min(LIBM_HORIZON_S, times.max()), (name, first, until)
        ends_got, ends_ref = batch_ends(got['trace']), batch_ends(ref['trace'])
        matched = [(ends_ref.index(t), i) for i, t in enumerate(ends_got)
                   if t is not None and t in ends_ref and t / 2 ** 40 < until]
        assert matched, name
        for j, i in matched:
            assert np.abs(got['depth'][i].astype(np.float64) - ref['depth'][j]).max(initial=0) <= DEPTH_TOL, name
            assert np.abs(got['q'][i].astype(np.float64) - ref['q'][j]).max(initial=0) <= Q_TOL, name
    bg, br = got['budget'], ref['budget']
    assert bg.shape == br.shape, (name, bg.shape, br.shape)
    if br.size and (mode == 'rounded' or first is None):
        scale = np.abs(br).sum(axis=1, keepdims=True)
        assert np.all(np.abs(bg - br) <= 2e-6 * scale + 1e-9), (name, np.abs(bg - br).max())
    return first


def test_golden_vectors_cover_every_case(golden):
    names = {k.split('/')[1] for k in golden.files}
    assert names == set(step_cases.CASES)
    for mode in MODES:
        for name in step_cases.CASES:
            trace = golden[f'{mode}/{name}/trace']
            assert (trace[:, 3] == 1).sum() > 0, (mode, name)
    # the cases reach the parts of the step they are there for
    assert completed(golden['rounded/grid3_limiter_theta07/trace'])[:, 6].sum() > 0  # donor limiter
    assert completed(golden['rounded/quadtree_small/trace'])[:, 9].max() > 2000     # a wet quadtree
    assert golden['rounded/quadtree_small/depth'].shape[1] == 2663


@pytest.mark.parametrize('name', sorted(step_cases.CASES))
def test_oracle_matches_the_reference_source(golden, tmp_path, name):
    """The CPU restatement (oracle/step_ref.c) against the reference's kernels."""
    from runner import oracle_factory
    got = step_cases.record_case(name, tmp_path / name, oracle_factory)
    for mode in MODES:
        first = check(got, fixture(golden, mode, name), mode, name)
        if first is not None:
            print(f'{name}: {mode} fixtures first differ at completed step {first[0]}, trace column {first[1]}')


def cuda_factory(path):
    def factory(arrays, params):
        from nhflood.native import CudaEngine
        params.path = {'multipass': 'multipass', 'pass': 'tiled', 'lattice': 'lattice'}.get(path, 'auto')
        params.cfl = 'pass' if path == 'pass' else 'auto'
        return CudaEngine(arrays, params)
    return factory


@pytest.mark.gpu
@pytest.mark.parametrize('path', ['auto', 'pass', 'multipass', 'lattice'])
@pytest.mark.parametrize('name', sorted(step_cases.CASES))
def test_cuda_step_matches_the_reference_source(golden, tmp_path, cuda_available, name, path):
    """The CUDA step, through the C ABI, against the reference's kernels."""
    got = step_cases.record_case(name, tmp_path / name, cuda_factory(path))
    for mode in MODES:
        check(got, fixture(golden, mode, name), mode, name)
