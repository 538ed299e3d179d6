"""The time loop around the device step, in place of the reference's
``_evolve`` (nh-flood-2d src/nh_flood_2d/core/solver_compact.py:179-1008).

It takes the same inputs (domain/force configs, the prepared mesh tables,
an optional restart checkpoint) and writes the same outputs: frames,
extrema, checkpoints, stations, ``mass_balance.csv``,
``step_statistics.csv`` and the manifest. It follows the same per-batch
protocol: upload the forcing when it changes, begin a batch of up to
``batch_size`` device steps towards the next event, read one trace back.
The step itself runs in an ``Engine`` (nhflood.native.CudaEngine by
default).

``TimeLoop`` holds the run's state, and each phase of a run is one method:
restoring a checkpoint, the initial water, the start of the device state,
the forcing of a batch, the bookkeeping of a batch's trace, an output, and
the final records. ``IntervalStats`` collects one step_statistics.csv row.
"""
from __future__ import annotations

import bisect
import csv
import hashlib
import json
import math
from dataclasses import dataclass, field
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
_STATE_ARRAYS = ('depth', 'bed', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed')


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
                                          clock_origin(domain_cfg, state))
        arrays.gate = controller.tables
    engine = (engine_factory or default_engine)(arrays, params)
    try:
        record.device(engine.backend, engine.device_name)
        loop = TimeLoop(domain_cfg, record, end_time, mesh, geometry, forcing, arrays, engine, batch_size,
                        state, gate_cfg=gate_cfg, layout=layout, controller=controller)
        return loop.run()
    finally:
        engine.close()


def clock_origin(domain_cfg, state) -> float:
    """Seconds of clock before formal time 0 (solver_compact.py:280-284)."""
    meta = json.loads(state.metadata_json) if state else {}
    if meta.get('run_state', False):
        return meta['clock_origin_before_start_s']
    return domain_cfg.warmup_duration


@dataclass
class IntervalStats:
    """One step_statistics.csv row: the dts of the interval's regular and
    event-shortened steps and its limiter activity."""
    regular: list = field(default_factory=list)
    shortened: list = field(default_factory=list)
    limited_cells: int = 0
    limited_faces: int = 0
    min_scale: float = 1.

    def add(self, dt, event_short, cells, faces, scale):
        (self.shortened if event_short else self.regular).append(dt)
        self.add_activity(cells, faces, scale)

    def add_activity(self, cells, faces, scale):
        self.limited_cells += cells
        self.limited_faces += faces
        self.min_scale = min(self.min_scale, scale)

    def row(self, date, seconds, limits, ids) -> dict:
        regular, shortened = np.array(self.regular), np.array(self.shortened)

        def summary(values, reduce):
            return float(reduce(values)) if len(values) else ''
        return dict(time=date.isoformat(), elapsed_seconds=seconds, steps=len(regular) + len(shortened),
                    standard_steps=len(regular), standard_dt_min_s=summary(regular, np.min),
                    standard_dt_max_s=summary(regular, np.max), standard_dt_mean_s=summary(regular, np.mean),
                    event_short_steps=len(shortened), event_dt_min_s=summary(shortened, np.min),
                    event_dt_sum_s=float(shortened.sum()) if len(shortened) else 0.,
                    limited_cell_steps=self.limited_cells, limited_face_steps=self.limited_faces,
                    minimum_donor_scale=self.min_scale, cfl_min_s=float(limits[0]), limiting_edge=int(ids[0]),
                    lower_cell=int(ids[1]), higher_cell=int(ids[2]), lower_depth_m=float(limits[1]),
                    higher_depth_m=float(limits[2]), face_depth_m=float(limits[3]),
                    face_velocity_m_s=float(limits[4]))


class TimeLoop:
    """One run of the time loop over an engine (see the module doc)."""

    def __init__(self, domain_cfg, record, end_time, mesh, geometry, forcing, arrays, engine, batch_size,
                 state=None, *, gate_cfg=None, layout=None, controller=None):
        self.cfg, self.record, self.end_time = domain_cfg, record, end_time
        self.mesh, self.geometry, self.forcing = mesh, geometry, forcing
        self.arrays, self.engine, self.controller = arrays, engine, controller
        self.gate_cfg, self.layout = gate_cfg, layout
        if state is None and domain_cfg.restart_state:
            state = read_checkpoint(domain_cfg.restart_state)
        self.state = state
        self.meta = json.loads(state.metadata_json) if state else {}
        self.continuation = bool(self.meta.get('run_state', False))
        self.origin = clock_origin(domain_cfg, state)
        initial = (state.clock_hi * 2 ** 32 + state.clock_lo) / 2 ** 40 if state else 0.
        self.clock = HostClock(initial, batch_size=batch_size)
        self.nb = len(forcing.boundaries)
        self.root = Path(domain_cfg.output_dir)
        self.area = geometry.area
        # per-run bookkeeping
        self.steps = self.warmup_steps = self.outputs = 0
        self.min_dt, self.max_dt, self.integrated_dt = float('inf'), 0., 0.
        self.trace_rows = []
        self.interval, self.total = IntervalStats(), IntervalStats()
        self.discharge_peaks = np.zeros(self.nb, dtype=np.float64)
        self.q_exact = np.zeros(self.nb, dtype=np.float64)
        self.device_totals = np.zeros(4 + 6 * self.nb, dtype=np.float64)
        self.dt_hasher = hashlib.sha256()
        self.coefficients = np.zeros((max(1, self.nb), 2), dtype=np.float32)
        self.uploaded = np.full_like(self.coefficients, np.nan)
        self.rain_index, self.rain_volume_rate = -1, np.float64(0)
        self.last_checkpoint_wall = 0.
        # forcing knots inside the run, by their clock tick (solver_compact.py:764-766)
        self.event_samples = {seconds_to_ticks(float(t) + self.origin): float(t)
                              for t in forcing.events if -self.origin <= t <= end_time}
        self.event_ticks = sorted(self.event_samples)

    # -- identity -----------------------------------------------------------
    def _identity(self):
        inputs = self.record.data['input_sha256']
        cfg = self.cfg
        self.state_identity = {
            'ne_sha256': inputs.get(str(Path(cfg.ne).resolve())),
            'ns_sha256': inputs.get(str(Path(cfg.ns).resolve())),
            'gate_config': self.gate_cfg.model_dump_json() if self.gate_cfg is not None else 'null',
        }
        self.boundary_identity = [dict(name=b.name, kind=b.kind, selected_edges_sha256=hashlib.sha256(
            np.sort(b.side_ids).astype('<i8').tobytes()).hexdigest()) for b in self.forcing.boundaries]
        self.land_json = cfg.model_dump(mode='json')['land_parameters']

    def _physics_config(self, with_afa):
        """The physics block of a checkpoint's metadata; restart compares it
        without afa (the CFL factor does not change the saved state)."""
        cfg = self.cfg
        physics = {'start': cfg.start.isoformat()}
        if with_afa:
            physics['afa'] = cfg.afa
        physics.update(sita=cfg.sita, min_h=cfg.min_h, land_parameters=self.land_json)
        return physics

    # -- restart (solver_compact.py:280-296, 689-724) -------------------------
    def _check_end(self):
        state = self.state
        end_tick = seconds_to_ticks(self.end_time + self.origin)
        state_tick = (state.clock_hi << 32) | state.clock_lo
        if state_tick > end_tick:
            raise ValueError('Checkpoint time is later than the requested simulation end')
        if self.continuation and state_tick == end_tick:
            self.record.data['completion_reason'] = 'checkpoint_at_end'

    def _restore(self):
        state, meta = self.state, self.meta
        if len(state.depth) != self.mesh.e_num or len(state.q) != self.mesh.s_num:
            raise ValueError('Checkpoint size differs from mesh')
        for key, value in self.state_identity.items():
            if meta[key] != value:
                raise ValueError(f'Checkpoint {key} differs from the current mesh/configuration')
        if self.continuation:
            if meta.get('boundary_identity') != self.boundary_identity:
                raise ValueError('Checkpoint boundary identity or order differs from configuration')
            saved = {k: v for k, v in meta['physics_config'].items() if k != 'afa'}
            if saved != self._physics_config(False):
                raise ValueError('Checkpoint clock or physical parameters differ from configuration')
        for name in _STATE_ARRAYS:
            self.engine.set(name, getattr(state, name))
        self.engine.set('peak_hi', state.first_time_hi)
        self.engine.set('peak_lo', state.first_time_lo)
        if self.controller is not None and self.continuation:
            self.engine.set_gate_state(self.controller.restore(meta['gate_controller']))

    # -- initial water and device state (solver_compact.py:857-892) ----------
    def _initial_water(self, bed):
        if self.state is None and self.cfg.warmup_duration > 0:
            depth, info = connected_still_water(bed, np.full(self.mesh.s_num, -999., dtype=np.float32),
                                                self.arrays.sbf, self.arrays.topology, self.forcing.boundaries,
                                                self.geometry.area)
            self.engine.set('depth', depth)
            self.record.data['initialization'] = dict(method='connected_still_water', **info)
        else:
            self.record.data['initialization'] = dict(method='checkpoint' if self.state else 'dry')

    def _open_budget(self):
        depth = self.engine.get('depth')
        initial = float(np.sum(depth.astype(float) * self.geometry.area, dtype=np.float64))
        self.budget = WaterBudget(Path(self.cfg.domain_dir) / 'mass_balance.csv', self.forcing.boundaries, initial)
        if self.continuation:
            saved = self.meta['budget']
            self.budget.initial = saved['initial_storage_m3']
            self.budget.rain = np.float64(saved['rainfall_m3'])
            self.budget.discharge[:] = saved['requested_discharge_m3']
            if 'device_totals' in saved:
                self.device_totals = np.array(saved['device_totals'], dtype=np.float64)
            else:  # exact integer units of 2**-149 written by the Taichi solver
                self.device_totals = np.array([math.ldexp(float(u), -149) for u in saved['device_units']])

    def _start_device(self, bed, elapsed):
        eng = self.engine
        if not self.continuation:
            targets = np.zeros(self.mesh.e_num, dtype='float32')
            for b in self.forcing.boundaries:
                if b.kind == 'level':
                    targets[b.cells] = np.maximum(b.series.at(0.) - bed[b.cells].astype(float), 0.)
            eng.apply_initial_levels(targets)
        eng.set_active(1)
        if self.controller is not None:
            if self.controller.initial_storage is None:
                self.controller.initialize_inventory(eng.get('depth'), self.area)
            eng.gate_check()
        eng.compute_cfl()
        eng.initial_diagnostics()
        if elapsed == 0. and self.end_time > 0.:
            eng.reset_extrema()

    # -- one batch ------------------------------------------------------------
    def _target(self, elapsed, warming) -> float:
        target = min(self.next_output, self.next_frame, 0. if warming else self.end_time)
        if not warming:
            i = bisect.bisect_right(self.event_ticks, seconds_to_ticks(self.clock.host_now_seconds))
            if i < len(self.event_ticks):
                target = min(target, self.event_ticks[i] / TICKS_PER_SECOND - self.origin)
        return target

    def _upload_forcing(self, elapsed, warming):
        """Boundary line coefficients (uploaded when they change) and, on a new
        rain interval, its rates (solver_compact.py:769-790). A quantized clock
        can sit half a tick before a knot, so the knot's exact time is used."""
        sample = 0. if warming else self.event_samples.get(seconds_to_ticks(self.clock.host_now_seconds), elapsed)
        for bi, b in enumerate(self.forcing.boundaries):
            t, v = b.series.times, b.series.values
            i = min(int(np.searchsorted(t, sample, side='right')) - 1, len(t) - 2)
            self.coefficients[bi, 0] = b.series.at(sample)
            self.coefficients[bi, 1] = 0. if warming else (v[i + 1] - v[i]) / (t[i + 1] - t[i])
        rates = None
        if not warming:
            rain = self.forcing.rain
            index = rain.index_at(sample)
            if index != self.rain_index:
                values = rain.rates(index)
                rates = values.astype(np.float32)
                self.rain_volume_rate = np.sum(values[rain.pixel_index[1:]] * self.area[1:], dtype=np.float64)
                self.rain_index = index
        changed = not np.array_equal(self.uploaded, self.coefficients)
        if changed:
            self.uploaded[:] = self.coefficients
        self.engine.set_forcing(self.coefficients if changed else None, rates, not warming)

    def _refuse_status(self, status, elapsed):
        if status == BAD_CFL:
            candidate, si, h = self.engine.cfl()
            if candidate < MIN_DT:
                cells = self.arrays.topology[si, 1:]
                depths = self.engine.get('depth')[cells]
                q = float(self.engine.get('q')[si])
                raise RuntimeError(f'CFL {candidate:.12g}s below supported minimum {MIN_DT}s; '
                                   f'edge={si}, cells={cells.tolist()}, depth_m={depths.tolist()}, '
                                   f'face_depth_m={h}, unit_discharge_m2_s={q}, velocity_m_s={q / h if h else 0.}')
        raise RuntimeError(f'Device clock status {status} at {elapsed}s')

    def _consume(self, rows, elapsed, warming) -> float:
        """Book every completed step of a batch trace; returns the new elapsed time."""
        for row in rows:
            status = int(row[3])
            if status == DONE:
                break
            if status != COMPLETED:
                self._refuse_status(status, elapsed)
            dt = f32_of_bits(row[0])
            scale = f32_of_bits(row[8])
            self.interval.add(dt, row[5], int(row[6]), int(row[7]), scale)
            self.total.add_activity(int(row[6]), int(row[7]), scale)
            for bi, b in enumerate(self.forcing.boundaries):
                self.q_exact[bi] = b.series.at(0. if warming else elapsed + dt / 2.)
            self.budget.add_forcing(dt, 0. if warming else self.rain_volume_rate, self.q_exact)
            elapsed = ticks_of(row[1], row[2]) / 2 ** 40 - self.origin
            self.steps += 1
            self.warmup_steps += int(warming)
            self.min_dt, self.max_dt = min(self.min_dt, dt), max(self.max_dt, dt)
            self.integrated_dt += dt
            np.maximum(self.discharge_peaks, self.q_exact, out=self.discharge_peaks)
            self.trace_rows.append(row.copy())
        self.dt_hasher.update(rows[rows[:, 3] == COMPLETED, 0].astype('uint32').tobytes())
        return elapsed

    # -- outputs ---------------------------------------------------------------
    def _checkpoint(self, path, depth, elapsed):
        budget = self.budget
        metadata = dict(self.state_identity, run_state=True, boundary_identity=self.boundary_identity,
                        clock_origin_before_start_s=self.origin, physics_config=self._physics_config(True),
                        total_steps=self.previous_steps + self.steps,
                        total_warmup_steps=self.previous_warmup_steps + self.warmup_steps,
                        elapsed_seconds=elapsed,
                        budget={'initial_storage_m3': budget.initial, 'rainfall_m3': float(budget.rain),
                                'requested_discharge_m3': budget.discharge.tolist(),
                                'device_totals': self.device_totals.tolist()})
        if self.controller is not None:
            metadata['gate_controller'] = self.controller.snapshot()
        tick = seconds_to_ticks(self.clock.host_now_seconds)
        eng = self.engine
        write_checkpoint(path, depth=depth, bed=eng.get('bed'), q=eng.get('q'), rain_time=eng.get('rain_time'),
                         infiltration=eng.get('infiltration'), clock_hi=tick >> 32, clock_lo=tick & 0xffffffff,
                         gate_open=self.controller.gate_open if self.controller is not None else False,
                         metadata_json=json.dumps(metadata), max_depth=eng.get('max_depth'),
                         first_time_hi=eng.get('peak_hi'), first_time_lo=eng.get('peak_lo'),
                         max_speed=eng.get('max_speed'))
        self.last_checkpoint_wall = perf_counter()

    def _stations(self, seconds, date):
        samples = self.engine.sample_stations(self.station_ids)
        rows = {name: dict(cell_id=self.station_cells[name],
                           **dict(zip(('depth', 'level', 'u', 'v'), map(float, samples[i]))))
                for i, name in enumerate(self.station_names)}
        append_station_samples(self.root / 'stations.csv', elapsed_seconds=seconds, time=date.isoformat(),
                               samples=rows)

    def _output(self, seconds, phase, *, frame=False, final=False):
        """Budget row, gate report, stations, frame, checkpoint and statistics
        row of one output time (solver_compact.py:792-855)."""
        eng = self.engine
        date = self.cfg.start + timedelta(seconds=seconds)
        self.outputs += 1
        self.device_totals = self.device_totals + finite_totals(eng.budget_flush())
        self.budget.set_device_terms(self.device_totals)
        depth = eng.get('depth')
        storage = float(np.sum(depth.astype(float) * self.area, dtype=np.float64))
        row = self.budget.output(date, seconds, storage, phase)
        if self.controller is not None:
            self.controller.pull(eng)
            self.record.data['gate_control'] = self.controller.report(depth, self.area, seconds)
            append_gate_balance(Path(self.cfg.domain_dir) / 'gate_balance.csv', date, seconds,
                                self.record.data['gate_control'])
            self.record.write()
        if self.station_names:
            self._stations(seconds, date)
        if frame:
            write_depth_frame(Path(self.cfg.frame_dir) / f'depth_{int(seconds)}.fdb', depth)
        if seconds == 0. or final:
            self._checkpoint(self.root / ('state_final.fdb' if final else 'state_start.fdb'), depth, seconds)
        elif frame and perf_counter() - self.last_checkpoint_wall >= CHECKPOINT_INTERVAL_S:
            self._checkpoint(self.root / 'state_latest.fdb', depth, seconds)
        limits, ids = eng.limits()
        self.stats_writer.writerow(self.interval.row(date, seconds, limits, ids))
        self.stats_file.flush()
        self.interval = IntervalStats()
        eng.reset_limits()
        print(f't={seconds:.6f}s phase={phase} storage={storage:.9g} residual={row["residual_m3"]:.9g} m3', flush=True)

    def _phase(self, elapsed):
        return 'warmup' if elapsed < 0 or self.end_time == 0 else 'simulation'

    def _final_records(self, timing):
        eng = self.engine
        final_depth = eng.get('depth')
        data = self.record.data
        data.update(
            steps=self.steps, warmup_steps=self.warmup_steps, mass_balance_final=self.budget.last_row,
            dt_seconds={'min': self.min_dt if self.steps else 0., 'max': self.max_dt, 'sum': self.integrated_dt},
            dt_sequence_sha256=self.dt_hasher.hexdigest(),
            limiter_activity=dict(limited_cell_steps=self.total.limited_cells,
                                  limited_face_steps=self.total.limited_faces,
                                  minimum_donor_scale=self.total.min_scale),
            requested_discharge_peak_m3_s={b.name: float(self.discharge_peaks[i])
                                           for i, b in enumerate(self.forcing.boundaries) if b.kind == 'discharge'},
            gate_open=bool(np.any(eng.gate_state()['commanded'])) if self.controller is not None else False,
            storage_depth_one_ulp_volume_m3=float(np.sum(np.abs(np.spacing(final_depth[1:])) * self.area[1:],
                                                         dtype=np.float64)))
        peak = eng.peak_memory()
        if peak is not None:
            data['peak_device_memory_bytes'] = peak
        data['timing_seconds'] = timing
        data['budget_accumulator']['output_transfers'] = self.outputs
        self.record.trace = np.array(self.trace_rows, dtype=np.uint32).reshape(-1, 10)

    # -- the run -------------------------------------------------------------------
    def run(self):
        cfg, eng, record, end_time = self.cfg, self.engine, self.record, self.end_time
        record.data['budget_accumulator'].update(terms=4 + 6 * self.nb, blocks=(self.mesh.e_num + 255) // 256)
        if self.state:
            self._check_end()
        eng.set_clock(words(self.clock.now_ticks))
        self.station_cells = resolve_station_cells(cfg.stations, self.geometry)
        self.station_names = list(self.station_cells)
        self.station_ids = np.array(list(self.station_cells.values()), dtype=np.int32)
        record.data['pressure_gradient'] = dict(method='tangential_subedge_reconstruction',
                                                hanging_edges=self.arrays.hang_edges,
                                                gradient_cells=self.arrays.hang_cells)
        eng.initialize()
        self._identity()
        if self.state:
            self._restore()
        bed = eng.get('bed')
        record.data.update(bed_events=[], output={
            'root': 'output', 'frame_interval_s': FRAME_INTERVAL_S, 'station_budget_interval_s': cfg.yield_step,
            'frames': 'F32 depth only; bed.fdb plus manifest gate_control reconstruct water level',
            'extrema_time_origin': (cfg.start - timedelta(seconds=self.origin)).isoformat(),
            'clock_quantum_s': 2. ** -40,
            'extrema_window': 'simulation' if end_time > 0 else 'warmup',
        })
        elapsed = self.clock.host_now_seconds - self.origin
        ys = cfg.yield_step
        after = 0. if elapsed < 0. else end_time
        self.next_output = min((math.floor(elapsed / ys) + 1) * ys, after)
        self.next_frame = min((math.floor(elapsed / FRAME_INTERVAL_S) + 1) * FRAME_INTERVAL_S, after)
        self.previous_steps = self.meta['total_steps'] if self.continuation else 0
        self.previous_warmup_steps = self.meta['total_warmup_steps'] if self.continuation else 0
        record.data['gate_cell_count'] = (int(np.count_nonzero(self.layout.cell_gate >= 0))
                                          if self.layout is not None else 0)
        record.data['station_cells'] = self.station_cells
        self.stats_file = (Path(cfg.domain_dir) / 'step_statistics.csv').open('w', newline='')
        self.stats_writer = csv.DictWriter(self.stats_file, fieldnames=STATS_FIELDS)
        self.stats_writer.writeheader()
        eng.reset_limits()
        self._initial_water(bed)
        write_bed(self.root / 'bed.fdb', self.state.bed if self.state else self.arrays.bed)
        self._open_budget()
        self._start_device(bed, elapsed)

        started = perf_counter()
        self.last_checkpoint_wall = started
        preprocess_seconds = started - record.clock
        warmup_seconds = 0.
        formal_started = started if elapsed >= 0. and end_time > elapsed else None
        self._output(elapsed, self._phase(elapsed), frame=True, final=elapsed == end_time)
        try:
            while elapsed < end_time:  # batches (solver_compact.py:918-985)
                warming = elapsed < 0.
                target = self._target(elapsed, warming)
                self._upload_forcing(elapsed, warming)
                target_words, origin_words = self.clock.begin(target + self.origin, self.clock.host_now_seconds)
                rows = self.clock.read_trace(eng.run_batch(target_words, origin_words))
                elapsed = self._consume(rows, elapsed, warming)
                is_output = abs(elapsed - self.next_output) < 1e-9 or elapsed == end_time
                is_frame = abs(elapsed - self.next_frame) < 1e-9 or elapsed == end_time
                if not (is_output or is_frame):
                    continue
                if warming and elapsed == 0. and end_time > 0.:
                    eng.reset_extrema()
                self._output(elapsed, self._phase(elapsed), frame=is_frame, final=elapsed == end_time)
                if warming and elapsed == 0.:
                    warmup_seconds = perf_counter() - started
                    if end_time > 0.:
                        formal_started = perf_counter()
                after = 0. if elapsed < 0 else end_time
                if is_output:
                    self.next_output = min(self.next_output + ys, after)
                if is_frame:
                    self.next_frame = min(self.next_frame + FRAME_INTERVAL_S, after)
            write_extrema(self.root / 'extrema.fdb', eng.get('max_depth'), eng.get('peak_hi'), eng.get('peak_lo'),
                          eng.get('max_speed'))
            finished = perf_counter()
            if end_time == 0.:
                warmup_seconds = finished - started
            formal_seconds = finished - formal_started if formal_started is not None else 0.
            steps, warm = self.steps, self.warmup_steps
            self._final_records(dict(
                preprocess_and_setup=preprocess_seconds, warmup=warmup_seconds, simulation=formal_seconds,
                warmup_per_step=warmup_seconds / warm if warm else None,
                simulation_per_step=formal_seconds / (steps - warm) if steps > warm else None))
        finally:
            self.budget.close()
            self.stats_file.close()
        return self.budget.last_row
