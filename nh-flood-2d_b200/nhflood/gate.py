"""Gate control: the layout of gate channels and ponds on the mesh, and the
host side of the device-side gate controller.

Follows the reference's
  * ``GateLayout.load``      – preprocess/gate.py:8-96 (gate components by
    shared subedges, inside/control points, validation);
  * ``GateController``       – core/gate.py:35-268 (irreversible per-gate
    command, bed motion, post-limiter exchange accounting, snapshot/restore,
    report);
  * ``append_gate_balance``  – core/gate.py:12-32 (``gate_balance.csv``).

The per-step work (trigger check, bed motion, exchange and source terms) runs
on the device next to the step (``nhf_gate_*`` in ``include/nhflood.h``); this
module resolves the layout, builds the device tables, keeps the cumulative
FP64 totals between outputs and writes the reports. The device accumulates
each step's terms per 256-entry block in FP64 with a compensated running sum,
where the reference adds F32 values into exact integer digits; a restored
reference checkpoint's integer units are converted exactly.
"""
from __future__ import annotations

import csv
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .clock import seconds_to_ticks
from .run_record import finite_totals

FIRST_FLOW_DEFINITION = ('End of first completed step with nonzero post-limiter gate-to-pond subedge volume '
                         'in either direction')
BALANCE_FIELDS = ['time', 'elapsed_seconds', 'region', 'pond_in_m3', 'pond_out_m3',
                  'pond_net_m3', 'river_in_m3', 'river_out_m3', 'channel_storage_m3',
                  'initial_storage_m3', 'storage_m3', 'overtopping_in_m3', 'overtopping_out_m3',
                  'rain_m3', 'infiltration_m3', 'positivity_m3', 'pipe_m3', 'boundary_m3',
                  'rounding_m3', 'residual_m3', 'river_net_m3']


def _components(selected: np.ndarray, topology: np.ndarray) -> np.ndarray:
    """Connected components of the selected cells over shared subedges. Each
    component is numbered by the rank of its lowest cell id, the order in
    which the reference's seed loop meets them. Union by pointer jumping:
    every round hooks the larger root of each edge under the smaller one."""
    n = len(selected)
    lo, hi = topology[1:, 1].astype(np.int64), topology[1:, 2].astype(np.int64)
    keep = selected[lo] & selected[hi] & (lo != hi)
    lo, hi = lo[keep], hi[keep]
    parent = np.arange(n, dtype=np.int64)

    def compress():
        while True:
            grand = parent[parent]
            if np.array_equal(grand, parent):
                return
            parent[:] = grand

    while len(lo):
        rl, rh = parent[lo], parent[hi]
        a, b = np.minimum(rl, rh), np.maximum(rl, rh)
        moving = a != b
        if not np.any(moving):
            break
        # several edges may hook one root: any smaller root is valid, and
        # the rounds repeat until every edge joins one root
        np.minimum.at(parent, b[moving], a[moving])
        compress()
    component = np.full(n, -1, dtype=np.int32)
    cells = np.flatnonzero(selected)
    roots = parent[cells]
    order = np.unique(roots)  # a root is its component's lowest cell
    component[cells] = np.searchsorted(order, roots).astype(np.int32)
    return component


def _locate(bounds: np.ndarray, point, label: str) -> int:
    """First cell (id order, cell 0 excluded) whose closed rectangle holds the
    point (preprocess/gate.py:44-53, the station-sampling convention)."""
    x, y = point
    hits = np.flatnonzero((bounds[:, 0] <= x) & (x <= bounds[:, 2]) & (bounds[:, 1] <= y) & (y <= bounds[:, 3]))
    hits = hits[hits != 0]
    if not len(hits):
        raise ValueError(f'{label}: point lies outside the mesh')
    return int(hits[0])


@dataclass
class GateLayout:
    """cell_gate[e]: gate index of each cell (-1 off gates); controls[G]: the
    control cell of each gate; cells[g]: the sorted cells of gate g."""
    cell_gate: np.ndarray
    controls: np.ndarray
    cells: list

    @classmethod
    def load(cls, config, bounds, land_types, topology, boundaries, bed) -> 'GateLayout':
        """preprocess/gate.py:15-96, with the same checks and messages."""
        land_types = np.asarray(land_types)
        topology = np.asarray(topology)
        selected = land_types == config.land_type
        selected[0] = False
        pond = land_types == config.pond_land_type
        pond[0] = False
        if np.any(selected & pond):
            raise ValueError('Gate and pond cells must not overlap')
        if not np.any(pond):
            raise ValueError('pond_land_type selects no pond cells')
        component = _components(selected, topology)
        n_groups = int(component.max()) + 1 if np.any(selected) else 0
        groups = [np.flatnonzero(component == g).astype(np.int32) for g in range(n_groups)]
        bed32 = np.asarray(bed).astype(np.float32)
        lo, hi = topology[1:, 1], topology[1:, 2]
        interior = (lo != 0) & (hi != 0)
        cell_gate = np.full(len(land_types), -1, dtype=np.int32)
        controls, cells, claimed = [], [], set()
        for index, gate in enumerate(config.gates):
            inside = _locate(bounds, gate.inside_point, f'{gate.name}.inside_point')
            group = int(component[inside])
            if group < 0:
                raise ValueError(f'{gate.name}: inside_point is not on a gate cell')
            if group in claimed:
                raise ValueError('Each gate component must correspond to exactly one gate')
            claimed.add(group)
            control = _locate(bounds, gate.control_point, f'{gate.name}.control_point')
            if selected[control]:
                raise ValueError(f'{gate.name}: control_point is on a gate cell')
            # compared on the F32 solver bed: an equal decimal target is allowed
            if not np.all(np.float32(config.open_elevation) <= bed32[groups[group]]):
                raise ValueError(f'{gate.name}: open_elevation exceeds a closed gate bed')
            inner_lo = interior & (component[lo] == group) & (component[hi] != group)
            inner_hi = interior & (component[hi] == group) & (component[lo] != group)
            neighbours = np.concatenate([hi[inner_lo], lo[inner_hi]])
            pond_side = bool(np.any(pond[neighbours]))
            river_side = bool(np.any(~pond[neighbours] & ~selected[neighbours]))
            if not pond_side or not river_side:
                raise ValueError(f'{gate.name}: gate needs internal edges to pond and non-pond non-gate cells')
            controls.append(control)
            cells.append(groups[group])
            cell_gate[groups[group]] = index
        if len(claimed) != len(groups):
            raise ValueError('Each gate component must correspond to exactly one gate')
        for boundary in boundaries:
            if boundary.kind == 'level' and np.any(selected[boundary.cells]):
                raise ValueError('Gate cells must not overlap a level boundary')
        return cls(cell_gate, np.array(controls, dtype=np.int32), cells)


@dataclass
class GateTables:
    """What the device controller reads (``nhf_gate`` / ``ora_gate``).

    flux_sides lists, in side order, the sides whose post-limiter volume the
    controller records (core/gate.py:131-153): gate/non-gate sides and sides
    between pond and non-pond cells outside the gates. Exchange terms are
    accumulated per 256 entries of this list, source terms per 256 cells."""
    count: int
    cell_gate: np.ndarray   # i32 [e]
    pond: np.ndarray        # i32 [e], pond[0] = 0
    closed: np.ndarray      # f32 [e] closed (initial working) bed
    targets: np.ndarray     # i32 [n_targets] gate cells, gate by gate
    controls: np.ndarray    # i32 [G]
    flux_sides: np.ndarray  # i32 [n_flux]
    formal_tick: int
    trigger_level: float
    opening_seconds: float
    open_elevation: float

    @property
    def terms(self) -> int:
        return 10 * self.count + 8


STATE_FIELDS = (('commanded', np.int32, 1), ('command', np.uint32, 2), ('flow_seen', np.int32, 1),
                ('first_flow', np.uint32, 2), ('opened', np.int32, 1), ('opened_at', np.uint32, 2))


def flux_sides(cell_gate: np.ndarray, pond: np.ndarray, topology: np.ndarray) -> np.ndarray:
    lo, hi = topology[:, 1], topology[:, 2]
    gl, gr = cell_gate[lo] >= 0, cell_gate[hi] >= 0
    record = (gl != gr) | (~gl & ~gr & (pond[lo] != pond[hi]))
    record[0] = False
    return np.flatnonzero(record).astype(np.int32)


@dataclass
class GateController:
    """Host side of core/gate.py:35-268 for one run."""
    config: object
    layout: GateLayout
    tables: GateTables
    totals: np.ndarray = None
    initial_storage: float | None = None
    initial_channel_storage: np.ndarray | None = None
    state: dict = field(default_factory=dict)

    @classmethod
    def build(cls, config, layout, bed, land_types, topology, origin_seconds) -> 'GateController':
        pond = (np.asarray(land_types) == config.pond_land_type).astype(np.int32)
        pond[0] = 0
        cell_gate = layout.cell_gate.astype(np.int32)
        tables = GateTables(
            count=len(config.gates), cell_gate=cell_gate, pond=pond,
            closed=np.asarray(bed, dtype=np.float32).copy(),
            targets=np.concatenate(layout.cells).astype(np.int32) if layout.cells else np.zeros(0, np.int32),
            controls=layout.controls.astype(np.int32), flux_sides=flux_sides(cell_gate, pond, np.asarray(topology)),
            formal_tick=seconds_to_ticks(origin_seconds), trigger_level=float(config.trigger_level),
            opening_seconds=float(config.opening_seconds), open_elevation=float(config.open_elevation))
        g = tables.count
        state = {name: np.zeros((g, width) if width > 1 else g, dtype=dtype) for name, dtype, width in STATE_FIELDS}
        return cls(config, layout, tables, np.zeros(tables.terms, dtype=np.float64), state=state)

    # term layout (core/gate.py:55-60)
    @property
    def offset(self) -> int:
        return 4 * self.tables.count

    @property
    def channel_source_offset(self) -> int:
        return self.offset + 8

    def pull(self, engine) -> None:
        """Fold the device's interval totals into the cumulative ones and copy
        the controller words back."""
        self.totals = self.totals + finite_totals(engine.gate_flush())
        self.state = engine.gate_state()

    def initialize_inventory(self, depth, area) -> None:
        pond = self.tables.pond.astype(bool)
        self.initial_storage = float(np.sum(depth[pond].astype(float) * area[pond]))
        self.initial_channel_storage = np.array([np.sum(depth[cells].astype(float) * area[cells])
                                                 for cells in self.layout.cells])

    def snapshot(self) -> dict:
        s = self.state
        return dict(commanded=s['commanded'].tolist(), command_ticks=s['command'].tolist(),
                    flow_seen=s['flow_seen'].tolist(), first_flow_ticks=s['first_flow'].tolist(),
                    opened=s['opened'].tolist(), opened_ticks=s['opened_at'].tolist(),
                    initial_storage_m3=self.initial_storage,
                    initial_channel_storage_m3=self.initial_channel_storage.tolist(),
                    budget_totals_m3=self.totals.tolist())

    def restore(self, saved: dict) -> dict:
        """Controller words for the device (and the host's inventory and
        totals) from a checkpoint's ``gate_controller`` block."""
        state = {'commanded': np.array(saved['commanded'], dtype=np.int32),
                 'command': np.array(saved['command_ticks'], dtype=np.uint32),
                 'flow_seen': np.array(saved['flow_seen'], dtype=np.int32),
                 'first_flow': np.array(saved['first_flow_ticks'], dtype=np.uint32),
                 'opened': np.array(saved['opened'], dtype=np.int32),
                 'opened_at': np.array(saved['opened_ticks'], dtype=np.uint32)}
        g = self.tables.count
        for name, dtype, width in STATE_FIELDS:
            state[name] = state[name].reshape((g, width) if width > 1 else g).astype(dtype)
        self.state = state
        self.initial_storage = saved['initial_storage_m3']
        self.initial_channel_storage = np.array(saved['initial_channel_storage_m3'], dtype=float)
        if 'budget_totals_m3' in saved:
            self.totals = np.array(saved['budget_totals_m3'], dtype=np.float64)
        else:  # exact integer units of 2**-149 written by the Taichi solver
            self.totals = np.array([math.ldexp(float(u), -149) for u in saved['budget_units']], dtype=np.float64)
        return state

    @property
    def gate_open(self) -> bool:
        return bool(np.any(self.state['commanded']))

    def report(self, depth, area, clock_seconds) -> dict:
        """The manifest's ``gate_control`` block (core/gate.py:208-268)."""
        totals = self.totals
        s = self.state
        formal = self.tables.formal_tick
        cfg = self.config

        def seconds(words):
            return ((int(words[0]) << 32) | int(words[1])) / 2 ** 40 - formal / 2 ** 40

        closed_bed = self.tables.closed
        gates = []
        for i, gate in enumerate(cfg.gates):
            commanded = bool(s['commanded'][i])
            command = seconds(s['command'][i]) if commanded else None
            end = command + cfg.opening_seconds if command is not None else None
            cells = self.layout.cells[i]
            channel_storage = float(np.sum(depth[cells].astype(float) * area[cells]))
            base = self.channel_source_offset + 6 * i
            sources = totals[base:base + 6]
            river_net = float(totals[4 * i + 2] - totals[4 * i + 3])
            pond_net = float(totals[4 * i] - totals[4 * i + 1])
            channel_net = river_net - pond_net + sources[0] - sources[1] + sources[2] + sources[3] + sources[4] + sources[5]
            channel_budget = dict(
                initial_storage_m3=float(self.initial_channel_storage[i]), storage_m3=channel_storage,
                river_net_m3=river_net, pond_net_m3=pond_net, rain_m3=float(sources[0]),
                infiltration_m3=float(sources[1]), positivity_m3=float(sources[2]), pipe_m3=float(sources[3]),
                boundary_m3=float(sources[4]), rounding_m3=float(sources[5]),
                residual_m3=float(channel_storage - self.initial_channel_storage[i] - channel_net))
            gates.append(dict(
                name=gate.name, cell_ids=cells.tolist(), closed_elevation=closed_bed[cells].tolist(),
                command_clock_ticks=s['command'][i].tolist() if commanded else None,
                control_cell=int(self.layout.controls[i]), command_seconds=command,
                first_effective_flow_seconds=seconds(s['first_flow'][i]) if s['flow_seen'][i] else None,
                fully_open_seconds=end if end is not None and clock_seconds >= end else None,
                first_fully_open_sample_seconds=seconds(s['opened_at'][i]) if s['opened'][i] else None,
                scheduled_fully_open_seconds=end,
                pond_in_m3=float(totals[4 * i]), pond_out_m3=float(totals[4 * i + 1]), pond_net_m3=pond_net,
                river_in_m3=float(totals[4 * i + 2]), river_out_m3=float(totals[4 * i + 3]),
                channel_storage_m3=channel_storage, channel_budget=channel_budget))
        t = totals[self.offset:self.offset + 8]
        pond = self.tables.pond.astype(bool)
        storage = float(np.sum(depth[pond].astype(float) * area[pond]))
        net = sum(g['pond_net_m3'] for g in gates) + t[0] - t[1] + t[2] - t[3] + t[4] + t[5] + t[6] + t[7]
        return dict(
            enabled=True, trigger_level=cfg.trigger_level, pond_land_type=cfg.pond_land_type,
            opening_seconds=cfg.opening_seconds, open_elevation=cfg.open_elevation,
            clock_origin_before_start_s=formal / 2 ** 40, clock_quantum_s=2. ** -40,
            first_effective_flow_definition=FIRST_FLOW_DEFINITION, gates=gates,
            pond_budget=dict(initial_storage_m3=self.initial_storage, storage_m3=storage,
                             overtopping_in_m3=float(t[0]), overtopping_out_m3=float(t[1]), rain_m3=float(t[2]),
                             infiltration_m3=float(t[3]), positivity_m3=float(t[4]), pipe_m3=float(t[5]),
                             boundary_m3=float(t[6]), rounding_m3=float(t[7]),
                             residual_m3=float(storage - self.initial_storage - net)))


def append_gate_balance(path, date, seconds, report) -> None:
    """One row per gate and one for the pond control volume at each output
    time (core/gate.py:12-32)."""
    path = Path(path)
    header = not path.exists()
    with path.open('a', newline='') as stream:
        writer = csv.DictWriter(stream, fieldnames=BALANCE_FIELDS)
        if header:
            writer.writeheader()
        for gate in report['gates']:
            row = dict(time=date.isoformat(), elapsed_seconds=seconds, region=gate['name'])
            row.update({key: gate[key] for key in BALANCE_FIELDS[3:9]})
            row.update({key: value for key, value in gate['channel_budget'].items() if key != 'pond_net_m3'})
            writer.writerow(row)
        writer.writerow(dict(time=date.isoformat(), elapsed_seconds=seconds, region='pond_control_volume',
                             **report['pond_budget']))
