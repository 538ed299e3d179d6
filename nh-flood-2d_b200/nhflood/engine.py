"""The time loop around the device step: the replacement for the reference's
``_evolve`` (nh-flood-2d src/nh_flood_2d/core/solver_compact.py:179-1008).

Same inputs (domain/force configs, prepared mesh tables, optional restart
checkpoint), same per-batch protocol (upload forcing when it changes, begin a
batch of up to ``batch_size`` device steps towards the next event, read one
trace back) and the same outputs: frames, extrema, checkpoints, stations,
``mass_balance.csv``, ``step_statistics.csv`` and the manifest. The step
itself runs in an ``Engine`` (nhflood.native.CudaEngine by default).
"""
from __future__ import annotations

import bisect
import csv
import hashlib
import json
import math
from datetime import timedelta
from pathlib import Path
from time import perf_counter

import numpy as np

from .clock import BAD_CFL, COMPLETED, DONE, TICKS_PER_SECOND, HostClock, seconds_to_ticks, ticks_of, words
from .forcing import Forcing
from .gate import GateController, GateLayout, append_gate_balance
from .geometry import MeshGeometry, connected_still_water
from .model import MIN_DT, StepParams, build_step_arrays
from .output import (append_station_samples, read_checkpoint, resolve_station_cells, write_bed,
                     write_checkpoint, write_depth_frame, write_extrema)
from .preprocess import load_mesh
from .run_record import WaterBudget, finite_totals

CHECKPOINT_INTERVAL_S = 30 * 60
FRAME_INTERVAL_S = 900
STATS_FIELDS = ['time', 'elapsed_seconds', 'steps', 'standard_dt_min_s', 'standard_dt_max_s', 'standard_dt_mean_s',
                'standard_steps', 'event_short_steps', 'event_dt_min_s', 'event_dt_sum_s', 'cfl_min_s',
                'limited_cell_steps', 'limited_face_steps', 'minimum_donor_scale',
                'limiting_edge', 'lower_cell', 'higher_cell', 'lower_depth_m',
                'higher_depth_m', 'face_depth_m', 'face_velocity_m_s']


def f32_of_bits(bits) -> float:
    return float(np.array(bits, dtype=np.uint32).view(np.float32))


def default_engine(arrays, params):
    from .native import CudaEngine
    return CudaEngine(arrays, params)


def evolve(domain_cfg, force_cfg, record, coupling, end_time, engine_factory=None, batch_size=32):
    if coupling is not None:
        raise NotImplementedError('SWMM pipe coupling is not part of this engine')
    mesh, side_flags = load_mesh(domain_cfg)
    geometry = MeshGeometry.from_mesh(mesh)
    forcing = Forcing.load(domain_cfg, force_cfg, geometry)
    return evolve_loaded(domain_cfg, record, end_time, mesh, side_flags, geometry, forcing,
                         engine_factory=engine_factory, batch_size=batch_size, gate_cfg=force_cfg.gate)


def evolve_loaded(domain_cfg, record, end_time, mesh, side_flags, geometry, forcing, *, engine_factory=None,
                  batch_size=32, state=None, gate_cfg=None):
    """The time loop on an already loaded mesh and forcing. ``state`` may be an
    in-memory Checkpoint used instead of ``domain_cfg.restart_state``;
    ``gate_cfg`` is the force config's gate block (a layout is resolved and
    validated whenever it is present, the controller runs when enabled)."""
    params = StepParams(afa=domain_cfg.afa, sita=domain_cfg.sita, min_h=domain_cfg.min_h, batch_size=batch_size)
    arrays = build_step_arrays(mesh, side_flags, geometry, forcing, domain_cfg.land_parameters, domain_cfg.sita)
    if state is None and domain_cfg.restart_state:
        state = read_checkpoint(domain_cfg.restart_state)
    # the gate layout and closed bed come from the mesh bed (solver_compact.py:202-203, 297-299)
    layout = (GateLayout.load(gate_cfg, geometry.bounds, mesh.land_type, mesh.topology, forcing.boundaries,
                              arrays.bed) if gate_cfg is not None else None)
    controller = None
    if gate_cfg is not None and gate_cfg.enabled:
        controller = GateController.build(gate_cfg, layout, arrays.bed, mesh.land_type, mesh.topology,
                                          _clock_origin(domain_cfg, state))
        arrays.gate = controller.tables
    engine = (engine_factory or default_engine)(arrays, params)
    try:
        record.device(engine.backend, engine.device_name)
        return _run(domain_cfg, record, end_time, mesh, geometry, forcing, arrays, engine, batch_size, state,
                    gate_cfg=gate_cfg, layout=layout, controller=controller)
    finally:
        engine.close()


def _clock_origin(domain_cfg, state) -> float:
    """Seconds of clock before formal time 0 (solver_compact.py:280-284)."""
    meta = json.loads(state.metadata_json) if state else {}
    if meta.get('run_state', False):
        return meta['clock_origin_before_start_s']
    return domain_cfg.warmup_duration


def _run(domain_cfg, record, end_time, mesh, geometry, forcing, arrays, engine, batch_size, state=None, *,
         gate_cfg=None, layout=None, controller=None):
    e_num, s_num = mesh.e_num, mesh.s_num
    b_num = len(forcing.boundaries)
    afa, sita, min_h = domain_cfg.afa, domain_cfg.sita, domain_cfg.min_h
    record.data['budget_accumulator'].update(terms=4 + 6 * b_num, blocks=(e_num + 255) // 256)

    # -- restart state and clock origin (solver_compact.py:280-296)
    if state is None and domain_cfg.restart_state:
        state = read_checkpoint(domain_cfg.restart_state)
    state_meta = json.loads(state.metadata_json) if state else {}
    continuation = bool(state_meta.get('run_state', False))
    origin_before_start = _clock_origin(domain_cfg, state)
    initial_clock = ((state.clock_hi * 2 ** 32 + state.clock_lo) / 2 ** 40 if state else 0.)
    if state:
        end_tick = seconds_to_ticks(end_time + origin_before_start)
        state_tick = (state.clock_hi << 32) | state.clock_lo
        if state_tick > end_tick:
            raise ValueError('Checkpoint time is later than the requested simulation end')
        if continuation and state_tick == end_tick:
            record.data['completion_reason'] = 'checkpoint_at_end'
    clock = HostClock(initial_clock, batch_size=batch_size)
    engine.set_clock(words(clock.now_ticks))
    station_cells = resolve_station_cells(domain_cfg.stations, geometry)
    station_names = list(station_cells)
    station_ids = np.array(list(station_cells.values()), dtype=np.int32)
    record.data['pressure_gradient'] = dict(method='tangential_subedge_reconstruction',
                                            hanging_edges=arrays.hang_edges, gradient_cells=arrays.hang_cells)

    # -- initialize + identity checks + restore (solver_compact.py:689-724)
    engine.initialize()
    inputs = record.data['input_sha256']
    state_identity = {
        'ne_sha256': inputs.get(str(Path(domain_cfg.ne).resolve())),
        'ns_sha256': inputs.get(str(Path(domain_cfg.ns).resolve())),
        'gate_config': gate_cfg.model_dump_json() if gate_cfg is not None else 'null',
    }
    boundary_identity = [dict(name=b.name, kind=b.kind, selected_edges_sha256=hashlib.sha256(
        np.sort(b.side_ids).astype('<i8').tobytes()).hexdigest()) for b in forcing.boundaries]
    land_json = domain_cfg.model_dump(mode='json')['land_parameters']
    if state:
        if len(state.depth) != e_num or len(state.q) != s_num:
            raise ValueError('Checkpoint size differs from mesh')
        for key in state_identity:
            if state_meta[key] != state_identity[key]:
                raise ValueError(f'Checkpoint {key} differs from the current mesh/configuration')
        if continuation:
            if state_meta.get('boundary_identity') != boundary_identity:
                raise ValueError('Checkpoint boundary identity or order differs from configuration')
            expected = {'start': domain_cfg.start.isoformat(), 'sita': sita, 'min_h': min_h,
                        'land_parameters': land_json}
            physics = {k: v for k, v in state_meta['physics_config'].items() if k != 'afa'}
            if physics != expected:
                raise ValueError('Checkpoint clock or physical parameters differ from configuration')
        for name in ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed'):
            engine.set(name, getattr(state, name))
        engine.set('peak_hi', state.first_time_hi)
        engine.set('peak_lo', state.first_time_lo)
        if controller is not None and continuation:
            engine.set_gate_state(controller.restore(state_meta['gate_controller']))
    bed_np = engine.get('bed')
    root = Path(domain_cfg.output_dir)
    record.data.update(bed_events=[], output={
        'root': 'output', 'frame_interval_s': FRAME_INTERVAL_S, 'station_budget_interval_s': domain_cfg.yield_step,
        'frames': 'F32 depth only; bed.fdb plus manifest gate_control reconstruct water level',
        'extrema_time_origin': (domain_cfg.start - timedelta(seconds=origin_before_start)).isoformat(),
        'clock_quantum_s': 2. ** -40,
        'extrema_window': 'simulation' if end_time > 0 else 'warmup',
    })

    # -- loop bookkeeping (solver_compact.py:734-767)
    s = _Loop()
    s.elapsed = clock.host_now_seconds - origin_before_start
    ys = domain_cfg.yield_step
    s.next_output = min((math.floor(s.elapsed / ys) + 1) * ys, 0. if s.elapsed < 0. else end_time)
    s.next_frame = min((math.floor(s.elapsed / FRAME_INTERVAL_S) + 1) * FRAME_INTERVAL_S,
                       0. if s.elapsed < 0. else end_time)
    previous_steps = state_meta['total_steps'] if continuation else 0
    previous_warmup_steps = state_meta['total_warmup_steps'] if continuation else 0
    discharge_peaks = np.zeros(b_num, dtype=np.float64)
    record.data['gate_cell_count'] = int(np.count_nonzero(layout.cell_gate >= 0)) if layout is not None else 0
    record.data['station_cells'] = station_cells
    coefficients = np.zeros((max(1, b_num), 2), dtype=np.float32)
    previous_coefficients = np.full_like(coefficients, np.nan)
    event_samples = {seconds_to_ticks(float(t) + origin_before_start): float(t)
                     for t in forcing.events if -origin_before_start <= t <= end_time}
    event_ticks = sorted(event_samples)
    stats_file = (Path(domain_cfg.domain_dir) / 'step_statistics.csv').open('w', newline='')
    stats_writer = csv.DictWriter(stats_file, fieldnames=STATS_FIELDS)
    stats_writer.writeheader()
    interval_dts, interval_event_dts = [], []
    interval_activity = [0, 0, 1.]
    total_activity = [0, 0, 1.]
    engine.reset_limits()
    dt_hasher = hashlib.sha256()
    q_exact = np.zeros(b_num, dtype=np.float64)
    device_totals = np.zeros(4 + 6 * b_num, dtype=np.float64)
    rain_state = {'index': -1, 'volume_rate': np.float64(0)}
    area_f64 = geometry.area

    def upload_forcing(seconds, warming):
        # A quantized clock can sit half a tick before a knot: use the knot's exact time.
        sample = 0. if warming else event_samples.get(seconds_to_ticks(clock.host_now_seconds), seconds)
        for bi, b in enumerate(forcing.boundaries):
            i = min(int(np.searchsorted(b.series.times, sample, side='right')) - 1, len(b.series.times) - 2)
            coefficients[bi, 0] = b.series.at(sample)
            coefficients[bi, 1] = 0. if warming else ((b.series.values[i + 1] - b.series.values[i])
                                                      / (b.series.times[i + 1] - b.series.times[i]))
        rates = None
        if not warming:
            index = forcing.rain.index_at(sample)
            if index != rain_state['index']:
                r = forcing.rain.rates(index)
                rates = r.astype(np.float32)
                rain_state['volume_rate'] = np.sum(r[forcing.rain.pixel_index[1:]] * area_f64[1:], dtype=np.float64)
                rain_state['index'] = index
        changed = not np.array_equal(previous_coefficients, coefficients)
        if changed:
            previous_coefficients[:] = coefficients
        engine.set_forcing(coefficients if changed else None, rates, not warming)

    def checkpoint(path, depth_np):
        metadata = dict(state_identity, run_state=True, boundary_identity=boundary_identity,
                        clock_origin_before_start_s=origin_before_start,
                        physics_config={'start': domain_cfg.start.isoformat(), 'afa': afa, 'sita': sita,
                                        'min_h': min_h, 'land_parameters': land_json},
                        total_steps=previous_steps + s.steps,
                        total_warmup_steps=previous_warmup_steps + s.warmup_steps,
                        elapsed_seconds=s.elapsed,
                        budget={'initial_storage_m3': budget.initial, 'rainfall_m3': float(budget.rain),
                                'requested_discharge_m3': budget.discharge.tolist(),
                                'device_totals': device_totals.tolist()})
        if controller is not None:
            metadata['gate_controller'] = controller.snapshot()
        tick_count = seconds_to_ticks(clock.host_now_seconds)
        peak_hi, peak_lo = engine.get('peak_hi'), engine.get('peak_lo')
        write_checkpoint(path, depth=depth_np, bed=engine.get('bed'), q=engine.get('q'),
                         rain_time=engine.get('rain_time'), infiltration=engine.get('infiltration'),
                         clock_hi=tick_count >> 32, clock_lo=tick_count & 0xffffffff,
                         gate_open=controller.gate_open if controller is not None else False,
                         metadata_json=json.dumps(metadata), max_depth=engine.get('max_depth'),
                         first_time_hi=peak_hi, first_time_lo=peak_lo, max_speed=engine.get('max_speed'))
        s.last_checkpoint_wall = perf_counter()

    def write_output(seconds, phase, *, frame=False, final=False):
        nonlocal device_totals
        date = domain_cfg.start + timedelta(seconds=seconds)
        s.outputs += 1
        device_totals = device_totals + finite_totals(engine.budget_flush())
        budget.set_device_terms(device_totals)
        depth_np = engine.get('depth')
        storage = float(np.sum(depth_np.astype(float) * area_f64, dtype=np.float64))
        row = budget.output(date, seconds, storage, phase)
        if controller is not None:
            controller.pull(engine)
            record.data['gate_control'] = controller.report(depth_np, area_f64, seconds)
            append_gate_balance(Path(domain_cfg.domain_dir) / 'gate_balance.csv', date, seconds,
                                record.data['gate_control'])
            record.write()
        if len(station_names):
            samples = engine.sample_stations(station_ids)
            append_station_samples(root / 'stations.csv', elapsed_seconds=seconds, time=date.isoformat(),
                                   samples={name: dict(cell_id=station_cells[name],
                                                       **dict(zip(('depth', 'level', 'u', 'v'), map(float, samples[i]))))
                                            for i, name in enumerate(station_names)})
        if frame:
            write_depth_frame(Path(domain_cfg.frame_dir) / f'depth_{int(seconds)}.fdb', depth_np)
        if seconds == 0. or final:
            checkpoint(root / ('state_final.fdb' if final else 'state_start.fdb'), depth_np)
        elif frame and perf_counter() - s.last_checkpoint_wall >= CHECKPOINT_INTERVAL_S:
            checkpoint(root / 'state_latest.fdb', depth_np)
        limits, ids = engine.limits()
        regular, shortened = np.array(interval_dts), np.array(interval_event_dts)
        stats_writer.writerow(dict(
            time=date.isoformat(), elapsed_seconds=seconds, steps=len(regular) + len(shortened),
            standard_steps=len(regular),
            standard_dt_min_s=float(regular.min()) if len(regular) else '',
            standard_dt_max_s=float(regular.max()) if len(regular) else '',
            standard_dt_mean_s=float(regular.mean()) if len(regular) else '',
            event_short_steps=len(shortened), event_dt_min_s=float(shortened.min()) if len(shortened) else '',
            event_dt_sum_s=float(shortened.sum()) if len(shortened) else 0.,
            limited_cell_steps=interval_activity[0], limited_face_steps=interval_activity[1],
            minimum_donor_scale=interval_activity[2],
            cfl_min_s=float(limits[0]), limiting_edge=int(ids[0]), lower_cell=int(ids[1]), higher_cell=int(ids[2]),
            lower_depth_m=float(limits[1]), higher_depth_m=float(limits[2]), face_depth_m=float(limits[3]),
            face_velocity_m_s=float(limits[4])))
        stats_file.flush()
        interval_dts.clear()
        interval_event_dts.clear()
        interval_activity[:] = [0, 0, 1.]
        engine.reset_limits()
        print(f't={seconds:.6f}s phase={phase} storage={storage:.9g} residual={row["residual_m3"]:.9g} m3', flush=True)

    def supported_dt():
        candidate, si, h = engine.cfl()
        if candidate < MIN_DT:
            cells = arrays.topology[si, 1:]
            depths = engine.get('depth')[cells]
            q = float(engine.get('q')[si])
            raise RuntimeError(f'CFL {candidate:.12g}s below supported minimum {MIN_DT}s; '
                               f'edge={si}, cells={cells.tolist()}, depth_m={depths.tolist()}, '
                               f'face_depth_m={h}, unit_discharge_m2_s={q}, velocity_m_s={q / h if h else 0.}')
        return candidate

    # -- initial water (solver_compact.py:857-892)
    if state is None and domain_cfg.warmup_duration > 0:
        initial_depth, initialization = connected_still_water(
            bed_np, np.full(s_num, -999., dtype=np.float32), arrays.sbf, arrays.topology,
            forcing.boundaries, geometry.area)
        engine.set('depth', initial_depth)
        record.data['initialization'] = dict(method='connected_still_water', **initialization)
    else:
        record.data['initialization'] = dict(method='checkpoint' if state else 'dry')
    write_bed(root / 'bed.fdb', state.bed if state else arrays.bed)
    initial_depth = engine.get('depth')
    initial_storage = float(np.sum(initial_depth.astype(float) * geometry.area, dtype=np.float64))
    budget = WaterBudget(Path(domain_cfg.domain_dir) / 'mass_balance.csv', forcing.boundaries, initial_storage)
    if continuation:
        saved = state_meta['budget']
        budget.initial = saved['initial_storage_m3']
        budget.rain = np.float64(saved['rainfall_m3'])
        budget.discharge[:] = saved['requested_discharge_m3']
        if 'device_totals' in saved:
            device_totals = np.array(saved['device_totals'], dtype=np.float64)
        else:  # exact integer units of 2**-149 written by the Taichi solver
            device_totals = np.array([math.ldexp(float(u), -149) for u in saved['device_units']])
    if not continuation:
        targets = np.zeros(e_num, dtype='float32')
        for b in forcing.boundaries:
            if b.kind == 'level':
                targets[b.cells] = np.maximum(b.series.at(0.) - bed_np[b.cells].astype(float), 0.)
        engine.apply_initial_levels(targets)
    engine.set_active(1)
    if controller is not None:
        if controller.initial_storage is None:
            controller.initialize_inventory(engine.get('depth'), area_f64)
        engine.gate_check()
    engine.compute_cfl()
    engine.initial_diagnostics()
    if s.elapsed == 0. and end_time > 0.:
        engine.reset_extrema()

    phase_started = perf_counter()
    s.last_checkpoint_wall = phase_started
    preprocess_seconds = phase_started - record.clock
    warmup_seconds = 0.
    formal_started = phase_started if s.elapsed >= 0. and end_time > s.elapsed else None
    write_output(s.elapsed, 'warmup' if s.elapsed < 0 or end_time == 0 else 'simulation', frame=True,
                 final=s.elapsed == end_time)
    try:
        # -- batches (solver_compact.py:918-985)
        while s.elapsed < end_time:
            warming = s.elapsed < 0.
            target = min(s.next_output, s.next_frame, 0. if warming else end_time)
            if not warming:
                now_tick = seconds_to_ticks(clock.host_now_seconds)
                i = bisect.bisect_right(event_ticks, now_tick)
                if i < len(event_ticks):
                    target = min(target, event_ticks[i] / TICKS_PER_SECOND - origin_before_start)
            upload_forcing(s.elapsed, warming)
            target_words, origin_words = clock.begin(target + origin_before_start, clock.host_now_seconds)
            rows = clock.read_trace(engine.run_batch(target_words, origin_words))
            for row in rows:
                status = int(row[3])
                if status == DONE:
                    break
                if status != COMPLETED:
                    if status == BAD_CFL:
                        supported_dt()
                    raise RuntimeError(f'Device clock status {status} at {s.elapsed}s')
                scale = f32_of_bits(row[8])
                for activity in (interval_activity, total_activity):
                    activity[0] += int(row[6])
                    activity[1] += int(row[7])
                    activity[2] = min(activity[2], scale)
                dt = f32_of_bits(row[0])
                for bi, b in enumerate(forcing.boundaries):
                    q_exact[bi] = b.series.at(0. if warming else s.elapsed + dt / 2.)
                budget.add_forcing(dt, 0. if warming else rain_state['volume_rate'], q_exact)
                s.elapsed = ticks_of(row[1], row[2]) / 2 ** 40 - origin_before_start
                s.steps += 1
                s.warmup_steps += int(warming)
                s.min_dt, s.max_dt, s.integrated_dt = min(s.min_dt, dt), max(s.max_dt, dt), s.integrated_dt + dt
                np.maximum(discharge_peaks, q_exact, out=discharge_peaks)
                (interval_event_dts if row[5] else interval_dts).append(dt)
                s.trace_rows.append(row.copy())
            completed = rows[rows[:, 3] == COMPLETED, 0].astype('uint32')
            dt_hasher.update(completed.tobytes())
            is_output = abs(s.elapsed - s.next_output) < 1e-9 or s.elapsed == end_time
            is_frame = abs(s.elapsed - s.next_frame) < 1e-9 or s.elapsed == end_time
            if is_output or is_frame:
                if warming and s.elapsed == 0. and end_time > 0.:
                    engine.reset_extrema()
                write_output(s.elapsed, 'warmup' if s.elapsed < 0 or end_time == 0 else 'simulation',
                             frame=is_frame, final=s.elapsed == end_time)
                if warming and s.elapsed == 0.:
                    warmup_seconds = perf_counter() - phase_started
                    if end_time > 0.:
                        formal_started = perf_counter()
                if is_output:
                    s.next_output = min(s.next_output + ys, 0. if s.elapsed < 0 else end_time)
                if is_frame:
                    s.next_frame = min(s.next_frame + FRAME_INTERVAL_S, 0. if s.elapsed < 0 else end_time)
        write_extrema(root / 'extrema.fdb', engine.get('max_depth'), engine.get('peak_hi'),
                      engine.get('peak_lo'), engine.get('max_speed'))
        final_depth = engine.get('depth')
        record.data.update(
            steps=s.steps, warmup_steps=s.warmup_steps, mass_balance_final=budget.last_row,
            dt_seconds={'min': s.min_dt if s.steps else 0., 'max': s.max_dt, 'sum': s.integrated_dt},
            dt_sequence_sha256=dt_hasher.hexdigest(),
            limiter_activity=dict(limited_cell_steps=total_activity[0], limited_face_steps=total_activity[1],
                                  minimum_donor_scale=total_activity[2]),
            requested_discharge_peak_m3_s={b.name: float(discharge_peaks[i])
                                           for i, b in enumerate(forcing.boundaries) if b.kind == 'discharge'},
            gate_open=bool(np.any(engine.gate_state()['commanded'])) if controller is not None else False,
            storage_depth_one_ulp_volume_m3=float(np.sum(np.abs(np.spacing(final_depth[1:])) * geometry.area[1:],
                                                         dtype=np.float64)))
        peak = engine.peak_memory()
        if peak is not None:
            record.data['peak_device_memory_bytes'] = peak
        phase_finished = perf_counter()
        if end_time == 0.:
            warmup_seconds = phase_finished - phase_started
        formal_seconds = phase_finished - formal_started if formal_started is not None else 0.
        steps, warm = s.steps, s.warmup_steps
        record.data['timing_seconds'] = dict(
            preprocess_and_setup=preprocess_seconds, warmup=warmup_seconds, simulation=formal_seconds,
            warmup_per_step=warmup_seconds / warm if warm else None,
            simulation_per_step=formal_seconds / (steps - warm) if steps > warm else None)
        record.data['budget_accumulator']['output_transfers'] = s.outputs
        record.trace = np.array(s.trace_rows, dtype=np.uint32).reshape(-1, 10)
    finally:
        budget.close()
        stats_file.close()
    return budget.last_row


class _Loop:
    def __init__(self):
        self.elapsed = 0.
        self.next_output = 0.
        self.next_frame = 0.
        self.steps = 0
        self.warmup_steps = 0
        self.min_dt = float('inf')
        self.max_dt = 0.
        self.integrated_dt = 0.
        self.last_checkpoint_wall = 0.
        self.outputs = 0
        self.trace_rows = []
