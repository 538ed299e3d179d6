"""The reference's own step kernels as an engine of the host time loop.

Test infrastructure for make_step_golden.py. ``ReferenceKernels`` loads,
from a checkout of nh-flood-2d, the unchanged source of

  * core/solver_compact.py: the kernels and functions nested in ``_evolve``
    (prepare_step, tick, compute_cfl, finish_step, initialize,
    apply_initial_levels, initial_diagnostics, reset_extrema, velocity,
    add_diagnostic, update_pressure) and the module-level face_discharge
    and boundary_neighbor_sum;
  * core/clock.py (StepClock), core/pressure.py (PressureReconstruction),
    core/device_budget.py (DeviceBudget) and util/ti.py (copy_to_taichi);

with ti_standin installed as ``taichi``. ``ReferenceStepEngine`` creates
the fields that ``_evolve`` creates (solver_compact.py:233-336), under the
same names, from nhflood's step arrays, binds the kernels to them and
exposes the engine interface of nhflood.model.Engine, so that nhflood's
host loop (``_solve``) or ``PlainRun`` drives the reference's kernels
exactly as it drives the CUDA step. A batch replays the reference's graph
(solver_compact.py:894-909) slot by slot: prepare_step, update_pressure
(on meshes with hanging edges), tick, compute_cfl, finish_step.

The wet-cell count that the trace's tenth column carries is not a
reference output: it is counted here after each active step as the cells
whose depth is at least min_h, the predicate of ``velocity``
(solver_compact.py:359).
"""
from __future__ import annotations

import ast
import builtins
import math
import sys
import types
from pathlib import Path
from typing import no_type_check

import numpy as np

import ti_standin as ti

KERNELS = ('velocity', 'prepare_step', 'finish_step', 'add_diagnostic', 'initialize', 'apply_initial_levels',
           'tick', 'compute_cfl', 'initial_diagnostics', 'reset_extrema', 'update_pressure')
MODULE_FUNCTIONS = ('face_discharge', 'boundary_neighbor_sum')
TRACE_COLS = 10
STATE = {'bed': 'ez_t', 'depth': 'depth_t', 'q': 'sq_t', 'rain_time': 'cumulative_rain_time_t',
         'infiltration': 'infiltration_t', 'max_depth': 'max_depth_t', 'max_speed': 'max_speed_t', 'u': 'u_t',
         'v': 'v_t', 'peak_hi': 'peak_hi_t', 'peak_lo': 'peak_lo_t'}


def _package(name, path):
    module = sys.modules.get(name)
    if module is None:
        module = types.ModuleType(name)
        module.__path__ = [str(path)]
        sys.modules[name] = module
    return module


class ReferenceKernels:
    """The reference's step source, loaded once per process."""

    def __init__(self, root):
        root = Path(root)
        pkg = root / 'src' / 'nh_flood_2d'
        if not (pkg / 'core' / 'solver_compact.py').exists():
            raise FileNotFoundError(f'{pkg}: no nh-flood-2d checkout')
        ti.install()
        # Package objects only: nh_flood_2d/core/__init__.py imports fastdb4py.
        _package('nh_flood_2d', pkg)
        _package('nh_flood_2d.core', pkg / 'core')
        _package('nh_flood_2d.util', pkg / 'util')
        ti.load_module(pkg / 'util' / 'ti.py', 'nh_flood_2d.util.ti', 'nh_flood_2d.util')
        self.clock = ti.load_module(pkg / 'core' / 'clock.py', 'nh_flood_2d.core.clock', 'nh_flood_2d.core')
        self.pressure = ti.load_module(pkg / 'core' / 'pressure.py', 'nh_flood_2d.core.pressure', 'nh_flood_2d.core')
        self.budget = ti.load_module(pkg / 'core' / 'device_budget.py', 'nh_flood_2d.core.device_budget',
                                     'nh_flood_2d.core')
        path = pkg / 'core' / 'solver_compact.py'
        tree = ast.parse(path.read_text(), filename=str(path))
        evolve = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == '_evolve')
        nested = {n.name: n for n in ast.walk(evolve) if isinstance(n, ast.FunctionDef) and n.name in KERNELS}
        top = {n.name: n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in MODULE_FUNCTIONS}
        missing = set(KERNELS) - set(nested) | set(MODULE_FUNCTIONS) - set(top)
        if missing:
            raise LookupError(f'{path}: missing {sorted(missing)}')
        module = ast.Module(body=[top[n] for n in MODULE_FUNCTIONS] + [nested[n] for n in KERNELS], type_ignores=[])
        self.code = compile(ti.transform(module), str(path), 'exec')
        self.free = sorted(_free_names(module) - set(KERNELS) - set(MODULE_FUNCTIONS))
        self.source = str(path)


def _free_names(module) -> set:
    """Names the functions read but never bind: the closure of ``_evolve``."""
    loaded, bound = set(), set()
    for node in ast.walk(module):
        if isinstance(node, ast.Name):
            (loaded if isinstance(node.ctx, ast.Load) else bound).add(node.id)
        elif isinstance(node, ast.arg):
            bound.add(node.arg)
        elif isinstance(node, ast.FunctionDef):
            bound.add(node.name)
    return loaded - bound - set(dir(builtins))


class ReferenceStepEngine:
    """nhflood.model.Engine over the reference's kernels (see module doc)."""

    backend = 'reference-source'
    device_name = 'reference kernels under a serial NumPy stand-in for Taichi'

    def __init__(self, kernels: ReferenceKernels, arrays, params):
        if getattr(arrays, 'gate', None) is not None:
            raise NotImplementedError('gate controller cases are not replayed on the reference kernels')
        a = arrays
        e, s, b = a.e_num, a.s_num, a.b_num
        self.kernels, self.arrays, self.params = kernels, a, params
        self.batch_size = params.batch_size
        self.min_h = params.min_h

        def new(dtype, shape):
            return ti.field(dtype, shape)

        def copy(values, dtype, shape=None):
            values = np.asarray(values)
            f = ti.field(dtype, values.shape if shape is None else shape)
            f.from_numpy(values)
            return f

        f32, i32, u32, u8 = ti.f32, ti.i32, ti.u32, ti.u8
        nb = max(1, b)
        fields = dict(
            ex_t=copy(a.x, f32), ey_t=copy(a.y, f32), ez_t=copy(a.bed, f32), area_t=copy(a.area, f32),
            eq_t=new(f32, (e, 4)), increment_t=new(f32, e), rain_depth_t=new(f32, e), ndt_t=new(f32, ()),
            dh_t=new(f32, s), sq_t=new(f32, s), donor_scale_t=new(f32, e), limited_cells_t=new(u32, ()),
            limited_faces_t=new(u32, ()), minimum_scale_t=new(f32, ()), cfl_t=new(f32, s),
            flow_depth_t=new(f32, s), sdc_t=new(f32, s), sl_t=copy(a.length, f32), side_n_t=copy(a.side_n, f32),
            infiltration_f0_t=copy(a.f0, f32), infiltration_fc_t=copy(a.fc, f32), infiltration_k_t=copy(a.k, f32),
            sbf_t=copy(a.sbf, u8), sts_t=copy(np.asarray(a.topology).reshape(-1), i32, (s, 3)),
            isl_data_t=copy(a.isl_data, i32), face_ptr_t=copy(a.face_ptr, i32), face_count_t=copy(a.face_count, i32),
            face_qn_t=new(f32, (e, 4)), u_t=new(f32, e), v_t=new(f32, e), depth_t=new(f32, e), pipe_q_t=new(f32, e),
            ssq_t=new(f32, e), cumulative_rain_time_t=new(f32, e), infiltration_t=new(f32, e),
            boundary_id_t=copy(a.boundary_id, i32),
            open_face_t=copy(np.zeros((1, 4), np.float32) if a.open_face is None else a.open_face, f32),
            weight_t=copy(a.weight, f32), kind_t=copy(a.kind, i32), values_t=new(f32, nb),
            level_values_t=new(f32, nb), level_initial_t=new(f32, e), rain_index_t=copy(a.rain_index, i32),
            rain_rates_t=new(f32, a.n_rates), raining_t=new(i32, ()), batch_slot_t=new(i32, ()),
            coefficients_t=new(f32, (nb, 2)), max_depth_t=new(f32, e), max_speed_t=new(f32, e),
            peak_hi_t=new(u32, e), peak_lo_t=new(u32, e), widths_t=copy(a.width, f32), heights_t=copy(a.height, f32),
            pipe_volume_t=new(f32, 1), pipe_correction_t=new(f32, 1), cfl_arg_t=new(i32, ()),
            limit_value_t=new(f32, 5), limit_ids_t=new(i32, 3))
        clock = kernels.clock.StepClock(0., batch_size=params.batch_size)
        has_hanging = a.hcells is not None and len(a.hcells) > 0
        pressure = None
        if has_hanging:
            geometry = kernels.pressure.HangingGeometry(
                np.asarray(a.edge_index, np.int32), np.asarray(a.offsets, np.float32),
                np.asarray(a.slots, np.int32), np.asarray(a.hcells, np.int32), np.asarray(a.axes, np.int32))
            pressure = kernels.pressure.PressureReconstruction(
                geometry, bed=fields['ez_t'], depth=fields['depth_t'], x=fields['ex_t'], y=fields['ey_t'],
                lengths=fields['sl_t'], topology=fields['sts_t'], face_ptr=fields['face_ptr_t'],
                face_count=fields['face_count_t'], sides=fields['isl_data_t'], min_h=params.min_h)
        # the digits need (277 + bit length of the step bound + 15) // 16 words; a
        # generous bound only adds words (solver_compact.py:267-273)
        device_budget = kernels.budget.DeviceBudget((e + 255) // 256, 4 + 6 * b, 1 << 24)
        ns = ti.namespace(np=np, math=math, no_type_check=no_type_check, e_num=e, s_num=s, b_num=b,
                          g=9.81, afa=params.afa, sita=params.sita, min_h=params.min_h, clock=clock,
                          has_hanging=has_hanging, pressure=pressure, gate_enabled=False, coupled_enabled=False,
                          controller=None, device_budget=device_budget, diagnostic_t=device_budget.step, **fields)
        unresolved = [n for n in kernels.free if n not in ns]
        if unresolved:
            raise LookupError(f'closure names without a value: {unresolved}')
        exec(kernels.code, ns)
        self.ns, self.clock, self.device_budget = ns, clock, device_budget
        self.has_hanging = has_hanging
        self._flushed = np.zeros(4 + 6 * b, np.float64)

    # -- state ----------------------------------------------------------
    def get(self, name):
        return self.ns[STATE[name]].to_numpy()

    def set(self, name, values):
        self.ns[STATE[name]].from_numpy(np.asarray(values))

    def initialize(self):
        self.ns['initialize']()

    def set_clock(self, words):
        self.clock.now.from_numpy(np.asarray(words, np.uint32))

    def get_clock(self):
        return self.clock.now.to_numpy().astype(np.uint32)

    def set_active(self, active):
        self.clock.active[None] = int(active)

    def set_forcing(self, coefficients, rain_rates, raining):
        if coefficients is not None:
            self.ns['coefficients_t'].from_numpy(np.asarray(coefficients, np.float32))
        if rain_rates is not None:
            self.ns['rain_rates_t'].from_numpy(np.asarray(rain_rates, np.float32))
        self.ns['raining_t'][None] = int(bool(raining))

    # -- kernels ----------------------------------------------------------
    def apply_initial_levels(self, targets):
        """solver_compact.py:878-882: the level targets, the kernel, one budget collection."""
        self.ns['level_initial_t'].from_numpy(np.asarray(targets, np.float32))
        self.ns['apply_initial_levels']()
        self.device_budget.collect()
        self.device_budget.step_finished()

    def compute_cfl(self):
        self.ns['compute_cfl']()

    def initial_diagnostics(self):
        self.ns['initial_diagnostics']()

    def reset_extrema(self):
        self.ns['reset_extrema']()

    def run_batch(self, target_words, origin_words):
        """One replay of the batch graph (solver_compact.py:894-909) after
        clock.begin's uploads (clock.py:85-87). A slot whose prepare_step
        leaves the clock inactive skips update_pressure, tick and compute_cfl:
        every statement of those three kernels is guarded by clock.active."""
        ns, clock = self.ns, self.clock
        clock.next.from_numpy(np.asarray(target_words, np.uint32))
        clock.origin.from_numpy(np.asarray(origin_words, np.uint32))
        clock.trace.fill(0)
        ns['batch_slot_t'][None] = 0
        wet = np.zeros(self.batch_size, np.uint32)
        min_h = np.float32(self.min_h)
        for slot in range(self.batch_size):
            ns['prepare_step']()
            if clock.active[None] == 1:
                if self.has_hanging:
                    ns['update_pressure']()
                ns['tick']()
                ns['compute_cfl']()
                wet[slot] = np.count_nonzero(ns['depth_t'].arr[1:] >= min_h)
            ns['finish_step']()
        rows = np.zeros((self.batch_size, TRACE_COLS), np.uint32)
        rows[:, :9] = clock.trace.to_numpy()
        rows[:, 9] = wet
        return rows

    def budget_flush(self):
        """The interval's terms: DeviceBudget.flush returns cumulative totals."""
        totals = self.device_budget.flush()
        out = totals - self._flushed
        self._flushed = totals
        return out

    def cfl(self):
        si = int(self.ns['cfl_arg_t'][None])
        return float(self.ns['ndt_t'][None]), si, float(self.ns['flow_depth_t'][si])

    def ndt(self):
        return float(self.ns['ndt_t'][None])

    def limits(self):
        return self.ns['limit_value_t'].to_numpy(), self.ns['limit_ids_t'].to_numpy()

    def reset_limits(self):
        self.ns['limit_value_t'][0] = float('inf')

    def sample_stations(self, ids):
        ids = np.asarray(ids, dtype=np.int64)
        d, z = self.get('depth'), self.get('bed')
        out = np.zeros((len(ids), 4), np.float32)
        if len(ids):
            out[:, 0], out[:, 1] = d[ids], z[ids] + d[ids]
            out[:, 2], out[:, 3] = self.get('u')[ids], self.get('v')[ids]
        return out

    def peak_memory(self):
        return None

    def close(self):
        pass
