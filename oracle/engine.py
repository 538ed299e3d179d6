"""ORACLE — test infrastructure only.

ctypes wrapper that runs the CPU restatement (step_ref.c) behind the same
engine interface the time loop uses for the CUDA step, so a whole solver run
can be replayed on the CPU and compared bit for bit. Only tests/, the smoke
check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_uint32, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / '_build' / 'liboracle.so'
LIB_PATH_F64 = HERE / '_build' / 'liboracle_f64.so'  # same step with real = double (precision study)
TRACE_COLS = 10
STATE_F32 = ('bed', 'depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'u', 'v')
STATE_U32 = ('peak_hi', 'peak_lo')


def build() -> Path:
    sources = [HERE / 'step_ref.c', HERE / 'mathref.c', HERE / 'step_ref.h', HERE / 'Makefile']
    for lib in (LIB_PATH, LIB_PATH_F64):
        if not lib.exists() or any(p.stat().st_mtime > lib.stat().st_mtime for p in sources):
            subprocess.run(['make', '-s', '-C', str(HERE)], check=True)
            break
    return LIB_PATH


_PTRS = ('x', 'y', 'area', 'width', 'height', 'f0', 'fc', 'k', 'boundary_id', 'rain_index',
         'face_ptr', 'face_count', 'isl_data', 'weight', 'topology', 'length', 'side_n', 'sbf', 'kind',
         'open_face')
_HANG = ('edge_index', 'offsets', 'slots', 'hcells', 'axes')
_STATE = ('bed', 'depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'u', 'v',
          'peak_hi', 'peak_lo', 'pipe_q')


def _mesh_type(real):
    class OraMeshT(ctypes.Structure):
        _fields_ = ([(n, c_int32) for n in ('e_num', 's_num', 'b_num', 'n_rates', 'isl_len', 'batch_size')]
                    + [(n, real) for n in ('g', 'afa', 'sita', 'min_h')] + [('min_dt', c_float)]
                    + [(n, c_void_p) for n in _PTRS]
                    + [('hang_cells', c_int32), ('hang_edges', c_int32)]
                    + [(n, c_void_p) for n in _HANG]
                    + [(n, c_void_p) for n in _STATE])
    return OraMeshT


_GATE_TABLES = ('cell_gate', 'pond', 'closed', 'targets', 'controls', 'flux_sides')
_GATE_WORDS = ('commanded', 'flow_seen', 'opened', 'command', 'first_flow', 'opened_at')


class OraGate(ctypes.Structure):
    _fields_ = ([('count', c_int32), ('n_targets', c_int32), ('n_flux', c_int32)]
                + [(n, c_void_p) for n in _GATE_TABLES] + [('formal_tick', c_uint32 * 2)]
                + [(n, c_float) for n in ('trigger_level', 'opening_seconds', 'open_elevation')]
                + [(n, c_void_p) for n in _GATE_WORDS])


OraMesh = _mesh_type(c_float)
_MESH = {'f32': OraMesh, 'f64': _mesh_type(c_double)}
_REAL = {'f32': c_float, 'f64': c_double}
_LIBS = {}
_LIB = None


def library(precision: str = 'f32'):
    """The F32 restatement, or with precision='f64' the same step in F64."""
    global _LIB
    if precision not in _LIBS:
        build()
        lib = ctypes.CDLL(str(LIB_PATH if precision == 'f32' else LIB_PATH_F64))
        H = c_void_p
        U2 = POINTER(c_uint32)
        R = _REAL[precision]
        RP = POINTER(R)
        for name, res, args in [
            ('ora_create', H, [POINTER(_MESH[precision])]), ('ora_destroy', None, [H]),
            ('ora_initialize', None, [H]),
            ('ora_set_threads', None, [c_int]), ('ora_set_clock', None, [H, U2]), ('ora_get_clock', None, [H, U2]),
            ('ora_set_active', None, [H, c_int]),
            ('ora_set_forcing', None, [H, RP, RP, c_int]),
            ('ora_apply_initial_levels', None, [H, RP]), ('ora_compute_cfl', None, [H]),
            ('ora_initial_diagnostics', None, [H]), ('ora_reset_extrema', None, [H]),
            ('ora_run_batch', None, [H, U2, U2, U2]), ('ora_budget_flush', None, [H, POINTER(c_double)]),
            ('ora_budget_terms', c_int, [H]), ('ora_ndt', R, [H]), ('ora_cfl_arg', c_int32, [H]),
            ('ora_set_ndt', None, [H, c_float]),
            ('ora_limits', None, [H, RP, POINTER(c_int32)]), ('ora_reset_limits', None, [H]),
            ('ora_read_eq', None, [H, RP]), ('ora_read_flow_depth', None, [H, RP]),
            ('ora_read_gradients', None, [H, RP]), ('ora_update_pressure', None, [H]),
            ('ora_pressure_difference', R, [H, c_int, c_int, c_int, R]),
            ('ora_ln', c_double, [c_double]), ('ora_exp', c_double, [c_double]),
            ('ora_powf', c_float, [c_float, c_float]), ('ora_expf', c_float, [c_float]),
            ('ora_gate_attach', None, [H, POINTER(OraGate)]), ('ora_gate_check', None, [H]),
            ('ora_gate_terms', c_int, [H]), ('ora_gate_flush', None, [H, POINTER(c_double)]),
        ]:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIBS[precision] = lib
        if precision == 'f32':
            _LIB = lib
    return _LIBS[precision]


def set_threads(n: int) -> None:
    library().ora_set_threads(int(n))


class OracleEngine:
    """The restated reference step on the CPU (OpenMP), engine interface."""

    backend = 'cpu-oracle'

    def __init__(self, arrays, params, threads: int | None = None, precision: str = 'f32'):
        self.lib = library(precision)
        self.precision = precision
        self.real = np.float32 if precision == 'f32' else np.float64
        self.creal = _REAL[precision]
        if threads:
            self.lib.ora_set_threads(int(threads))
        self.device_name = f'CPU restatement ({os.cpu_count()} cores)'
        self.arrays = arrays
        self.batch_size = params.batch_size
        self.keep = {}
        e, s = arrays.e_num, arrays.s_num

        def keep(name, a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype)
            self.keep[name] = a
            return a.ctypes.data

        m = _MESH[precision]()
        m.e_num, m.s_num, m.b_num, m.n_rates = e, s, arrays.b_num, arrays.n_rates
        m.isl_len, m.batch_size = len(arrays.isl_data), params.batch_size
        m.g, m.afa, m.sita, m.min_h, m.min_dt = params.g, params.afa, params.sita, params.min_h, params.min_dt
        f32 = self.real
        for name, dtype in [('x', f32), ('y', f32), ('area', f32), ('width', f32), ('height', f32), ('f0', f32),
                            ('fc', f32), ('k', f32), ('boundary_id', np.int32), ('rain_index', np.int32),
                            ('face_ptr', np.int32), ('face_count', np.int32), ('isl_data', np.int32),
                            ('weight', f32), ('topology', np.int32), ('length', f32), ('side_n', f32),
                            ('sbf', np.uint8), ('kind', np.int32), ('open_face', f32)]:
            setattr(m, name, keep(name, getattr(arrays, name), dtype))
        m.hang_cells, m.hang_edges = arrays.hang_cells, arrays.hang_edges
        for name, dtype in [('edge_index', np.int32), ('offsets', f32), ('slots', np.int32),
                            ('hcells', np.int32), ('axes', np.int32)]:
            setattr(m, name, keep(name, getattr(arrays, name), dtype))
        self.state = {'bed': np.ascontiguousarray(arrays.bed, dtype=f32).copy()}
        for name in STATE_F32:
            if name != 'bed':
                self.state[name] = np.zeros(s if name == 'q' else e, dtype=f32)
        for name in STATE_U32:
            self.state[name] = np.zeros(e, dtype=np.uint32)
        for name in _STATE:
            setattr(m, name, self.state[name].ctypes.data if name in self.state else None)
        self._mesh = m
        self.h = self.lib.ora_create(ctypes.byref(m))
        self.terms = self.lib.ora_budget_terms(self.h)
        self._trace = np.zeros((self.batch_size, TRACE_COLS), np.uint32)
        self.gate = getattr(arrays, 'gate', None)
        if self.gate is not None:
            self._attach_gate(self.gate)

    def _attach_gate(self, t):
        from nhflood.gate import STATE_FIELDS
        g = OraGate()
        g.count, g.n_targets, g.n_flux = t.count, len(t.targets), len(t.flux_sides)
        for name in _GATE_TABLES:
            dtype = self.real if name == 'closed' else np.int32
            a = np.ascontiguousarray(getattr(t, name), dtype=dtype)
            self.keep['gate_' + name] = a
            setattr(g, name, a.ctypes.data)
        g.formal_tick[0], g.formal_tick[1] = t.formal_tick >> 32, t.formal_tick & 0xffffffff
        g.trigger_level, g.opening_seconds, g.open_elevation = t.trigger_level, t.opening_seconds, t.open_elevation
        self.gate_words = {name: np.zeros((t.count, width) if width > 1 else t.count, dtype=dtype)
                           for name, dtype, width in STATE_FIELDS}
        for name in _GATE_WORDS:
            setattr(g, name, self.gate_words[name].ctypes.data)
        self._gate = g
        self.lib.ora_gate_attach(self.h, ctypes.byref(g))
        self.gate_terms = self.lib.ora_gate_terms(self.h)

    def gate_check(self):
        self.lib.ora_gate_check(self.h)

    def gate_flush(self):
        out = np.zeros(self.gate_terms, np.float64)
        self.lib.ora_gate_flush(self.h, out.ctypes.data_as(POINTER(c_double)))
        return out

    def gate_state(self) -> dict:
        return {name: a.copy() for name, a in self.gate_words.items()}

    def set_gate_state(self, state: dict) -> None:
        for name, a in self.gate_words.items():
            a[...] = np.asarray(state[name]).astype(a.dtype).reshape(a.shape)

    def get(self, name):
        return self.state[name].copy()

    def set(self, name, values):
        arr = np.asarray(values)
        if arr.shape != self.state[name].shape:
            raise ValueError(f'{name}: shape {arr.shape} differs from {self.state[name].shape}')
        self.state[name][...] = arr.astype(self.state[name].dtype)

    def initialize(self):
        self.lib.ora_initialize(self.h)

    def set_clock(self, words):
        w = np.ascontiguousarray(words, np.uint32)
        self.lib.ora_set_clock(self.h, w.ctypes.data_as(POINTER(c_uint32)))

    def get_clock(self):
        w = np.zeros(2, np.uint32)
        self.lib.ora_get_clock(self.h, w.ctypes.data_as(POINTER(c_uint32)))
        return w

    def set_active(self, active):
        self.lib.ora_set_active(self.h, int(active))

    def _ptr(self, a):
        return a.ctypes.data_as(POINTER(self.creal))

    def set_forcing(self, coefficients, rain_rates, raining):
        coef = None if coefficients is None else np.ascontiguousarray(coefficients, self.real)
        rates = None if rain_rates is None else np.ascontiguousarray(rain_rates, self.real)
        self.lib.ora_set_forcing(self.h, self._ptr(coef) if coef is not None else None,
                                 self._ptr(rates) if rates is not None else None, int(bool(raining)))

    def apply_initial_levels(self, targets):
        t = np.ascontiguousarray(targets, self.real)
        self.lib.ora_apply_initial_levels(self.h, self._ptr(t))

    def compute_cfl(self):
        self.lib.ora_compute_cfl(self.h)

    def initial_diagnostics(self):
        self.lib.ora_initial_diagnostics(self.h)

    def reset_extrema(self):
        self.lib.ora_reset_extrema(self.h)

    def run_batch(self, target_words, origin_words):
        t = np.ascontiguousarray(target_words, np.uint32)
        o = np.ascontiguousarray(origin_words, np.uint32)
        self.lib.ora_run_batch(self.h, t.ctypes.data_as(POINTER(c_uint32)), o.ctypes.data_as(POINTER(c_uint32)),
                               self._trace.ctypes.data_as(POINTER(c_uint32)))
        return self._trace.copy()

    def budget_flush(self):
        out = np.zeros(self.terms, np.float64)
        self.lib.ora_budget_flush(self.h, out.ctypes.data_as(POINTER(c_double)))
        return out

    def cfl(self):
        si = int(self.lib.ora_cfl_arg(self.h))
        fd = np.zeros(self.arrays.s_num, self.real)
        self.lib.ora_read_flow_depth(self.h, self._ptr(fd))
        return float(self.lib.ora_ndt(self.h)), si, float(fd[si])

    def ndt(self) -> float:
        return float(self.lib.ora_ndt(self.h))

    def set_ndt(self, value: float) -> None:
        """Precision study only: the CFL candidate the next step uses."""
        self.lib.ora_set_ndt(self.h, float(value))

    def limits(self):
        values = np.zeros(5, self.real)
        ids = np.zeros(3, np.int32)
        self.lib.ora_limits(self.h, self._ptr(values), ids.ctypes.data_as(POINTER(c_int32)))
        return values, ids

    def reset_limits(self):
        self.lib.ora_reset_limits(self.h)

    def sample_stations(self, ids):
        ids = np.asarray(ids, dtype=np.int64)
        d, z = self.state['depth'], self.state['bed']
        out = np.zeros((len(ids), 4), self.real)
        if len(ids):
            out[:, 0] = d[ids]
            out[:, 1] = z[ids] + d[ids]
            out[:, 2] = self.state['u'][ids]
            out[:, 3] = self.state['v'][ids]
        return out

    def read_eq(self):
        out = np.zeros((self.arrays.e_num, 4), self.real)
        self.lib.ora_read_eq(self.h, self._ptr(out))
        return out

    def read_gradients(self):
        out = np.zeros((max(1, self.arrays.hang_cells), 2), self.real)
        self.lib.ora_read_gradients(self.h, self._ptr(out))
        return out[:self.arrays.hang_cells]

    def peak_memory(self):
        return None

    def close(self):
        if getattr(self, 'h', None):
            self.lib.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
