"""ctypes binding of libnhflood.so (include/nhflood.h) and the CUDA engine.

Device arrays are torch CUDA tensors owned by ``CudaEngine``; the library
receives their addresses and owns only its scratch. There is no CPU
fallback: constructing the engine without a GPU or without the built
library raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int32, c_uint32, c_void_p

import numpy as np

from .model import STATE_F32, STATE_U32, Engine, StepArrays, StepParams

NHF_TRACE_COLS = 10

_MESH_INTS = ('e_num', 's_num', 'b_num', 'n_rates', 'isl_len', 'hang_cells', 'hang_edges')
_MESH_PTRS = ('x', 'y', 'area', 'width', 'height', 'f0', 'fc', 'k', 'weight', 'boundary_id', 'rain_index',
              'face_ptr', 'face_count', 'isl_data', 'topology', 'length', 'side_n', 'sbf', 'kind',
              'open_face', 'edge_index', 'offsets', 'slots', 'hcells', 'axes',
              'bed', 'depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'u', 'v',
              'peak_hi', 'peak_lo')


class NhfMesh(ctypes.Structure):
    _fields_ = [(n, c_int32) for n in _MESH_INTS] + [(n, c_void_p) for n in _MESH_PTRS]


def _params_type(real):
    class Params(ctypes.Structure):
        _fields_ = [('g', real), ('afa', real), ('sita', real), ('min_h', real),
                    ('min_dt', c_float), ('batch_size', c_int32), ('path', c_int32), ('cfl_mode', c_int32)]
    return Params


NhfParams = _params_type(c_float)
# nhf_real of each build: the F32 step (libnhflood.so) and its FP64 build
# (libnhflood_f64.so, the multi-pass kernels with double physics)
PRECISIONS = {'f32': (c_float, np.float32, NhfParams), 'f64': (c_double, np.float64, _params_type(c_double))}


_GATE_TABLES = ('cell_gate', 'pond', 'closed', 'targets', 'controls', 'flux_sides')
_GATE_WORDS = ('commanded', 'flow_seen', 'opened', 'command', 'first_flow', 'opened_at')


class NhfGate(ctypes.Structure):
    _fields_ = ([('count', c_int32), ('n_targets', c_int32), ('n_flux', c_int32)]
                + [(n, c_void_p) for n in _GATE_TABLES] + [('formal_tick', c_uint32 * 2)]
                + [(n, c_float) for n in ('trigger_level', 'opening_seconds', 'open_elevation')]
                + [(n, c_void_p) for n in _GATE_WORDS])


_LIBS = {}


def library(path=None, precision: str = 'f32'):
    """Load (and declare) libnhflood.so, or with precision='f64' its FP64
    build libnhflood_f64.so; raises if it is missing."""
    if precision in _LIBS and path is None:
        return _LIBS[precision]
    from .build import LIBRARY, LIBRARY_F64
    path = path or (LIBRARY if precision == 'f32' else LIBRARY_F64)
    if not path.exists():
        raise RuntimeError(f'{path} is missing: build it with `python -m nhflood.build` '
                           '(the CUDA step has no CPU fallback)')
    lib = ctypes.CDLL(str(path))
    real, _, params_type = PRECISIONS[precision]
    H = c_void_p
    sig = {
        'nhf_create': (c_int32, [POINTER(NhfMesh), POINTER(params_type), c_void_p, POINTER(c_void_p)]),
        'nhf_real_bytes': (c_int32, []),
        'nhf_destroy': (c_int32, [H]),
        'nhf_last_error': (ctypes.c_char_p, [H]),
        'nhf_version': (ctypes.c_char_p, []),
        'nhf_initialize': (c_int32, [H]),
        'nhf_set_clock': (c_int32, [H, POINTER(c_uint32)]),
        'nhf_get_clock': (c_int32, [H, POINTER(c_uint32)]),
        'nhf_set_active': (c_int32, [H, c_int32]),
        'nhf_set_forcing': (c_int32, [H, POINTER(real), POINTER(real), c_int32]),
        'nhf_apply_initial_levels': (c_int32, [H, c_void_p]),
        'nhf_compute_cfl': (c_int32, [H]),
        'nhf_initial_diagnostics': (c_int32, [H]),
        'nhf_reset_extrema': (c_int32, [H]),
        'nhf_run_batch': (c_int32, [H, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32)]),
        'nhf_run_batch_async': (c_int32, [H, POINTER(c_uint32), POINTER(c_uint32)]),
        'nhf_read_trace': (c_int32, [H, POINTER(c_uint32)]),
        'nhf_budget_flush': (c_int32, [H, POINTER(c_double)]),
        'nhf_budget_terms': (c_int32, [H]),
        'nhf_get_cfl': (c_int32, [H, POINTER(real), POINTER(c_int32), POINTER(real)]),
        'nhf_limits': (c_int32, [H, POINTER(real), POINTER(c_int32)]),
        'nhf_reset_limits': (c_int32, [H]),
        'nhf_sample_stations': (c_int32, [H, POINTER(c_int32), c_int32, POINTER(real)]),
        'nhf_read_eq': (c_int32, [H, c_void_p]),
        'nhf_read_gradients': (c_int32, [H, c_void_p]),
        'nhf_synchronize': (c_int32, [H]),
        'nhf_stream': (c_void_p, [H]),
        'nhf_path': (ctypes.c_char_p, [H]),
        'nhf_cfl_noalloc': (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_float, c_float,
                                      c_void_p, c_void_p, c_void_p]),
        'nhf_cfl_noalloc_error': (ctypes.c_char_p, []),
        'nhf_gate_attach': (c_int32, [H, POINTER(NhfGate)]),
        'nhf_gate_check': (c_int32, [H]),
        'nhf_gate_terms': (c_int32, [H]),
        'nhf_gate_flush': (c_int32, [H, POINTER(c_double)]),
        'nhf_ensemble_create': (c_int32, [POINTER(c_void_p), c_int32, c_int32, c_void_p, POINTER(c_void_p)]),
        'nhf_ensemble_destroy': (c_int32, [H]),
        'nhf_ensemble_last_error': (ctypes.c_char_p, [H]),
        'nhf_ensemble_info': (c_int32, [H, POINTER(c_int32)]),
        'nhf_ensemble_stream': (c_void_p, [H]),
        'nhf_ensemble_run_batch': (c_int32, [H, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32)]),
        'nhf_ensemble_run_batch_async': (c_int32, [H, POINTER(c_uint32), POINTER(c_uint32)]),
        'nhf_ensemble_read_trace': (c_int32, [H, POINTER(c_uint32)]),
    }
    if precision == 'f64':  # the FP64 build has the single-mesh entry points only
        sig = {k: v for k, v in sig.items() if not k.startswith(('nhf_ensemble', 'nhf_cfl_noalloc'))}
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.nhf_real_bytes() != ctypes.sizeof(real):
        raise RuntimeError(f'{path}: nhf_real of {lib.nhf_real_bytes()} bytes, expected {ctypes.sizeof(real)}')
    _LIBS[precision] = lib
    return lib


def exported_symbols() -> list[str]:
    """Names declared in include/nhflood.h that the library must export."""
    return ['nhf_create', 'nhf_destroy', 'nhf_last_error', 'nhf_version', 'nhf_real_bytes', 'nhf_initialize',
            'nhf_set_clock',
            'nhf_get_clock', 'nhf_set_active', 'nhf_set_forcing', 'nhf_apply_initial_levels',
            'nhf_compute_cfl', 'nhf_initial_diagnostics', 'nhf_reset_extrema', 'nhf_run_batch',
            'nhf_run_batch_async', 'nhf_read_trace', 'nhf_budget_flush', 'nhf_budget_terms', 'nhf_get_cfl',
            'nhf_limits', 'nhf_reset_limits', 'nhf_sample_stations', 'nhf_read_eq', 'nhf_read_gradients',
            'nhf_synchronize', 'nhf_stream', 'nhf_path', 'nhf_cfl_noalloc', 'nhf_cfl_noalloc_error',
            'nhf_gate_attach', 'nhf_gate_check', 'nhf_gate_terms', 'nhf_gate_flush',
            'nhf_ensemble_create', 'nhf_ensemble_destroy', 'nhf_ensemble_last_error', 'nhf_ensemble_info',
            'nhf_ensemble_stream', 'nhf_ensemble_run_batch', 'nhf_ensemble_run_batch_async',
            'nhf_ensemble_read_trace']


def path_code(path) -> int:
    """nhf_params.path for a StepParams.path: 'auto', 'multipass', 'lattice'
    (uniform grids), 'tiled' (the fused tiled step, tile size by mesh size)
    or 'tile256' / 'tile512' / 'tile1024' (fused step with that tile size)."""
    if path == 'auto':
        return 0
    if path == 'multipass':
        return 1
    if path == 'lattice':
        return 2
    if path == 'tiled':
        return 3
    if isinstance(path, str) and path.startswith('tile') and path[4:] in ('256', '512', '1024'):
        return int(path[4:])
    raise ValueError(f'unknown step path {path!r}')


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(POINTER(c_uint32))


class CudaEngine(Engine):
    """The step on one CUDA device through libnhflood.so."""

    backend = 'cuda'

    def __init__(self, arrays: StepArrays, params: StepParams, device='cuda:0', precision: str = 'f32'):
        """precision 'f64' runs the FP64 build of the multi-pass kernels
        (libnhflood_f64.so): the same F32 inputs, every physics quantity in
        double, the clock and its trace in F32."""
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError('CudaEngine needs a CUDA device; the step has no CPU fallback')
        self.torch = torch
        self.precision = precision
        self.creal, self.real, self._params_type = PRECISIONS[precision]
        self.lib = library(precision=precision)
        self.arrays = arrays
        self.params = params
        self.device = torch.device(device)
        self.device_name = torch.cuda.get_device_name(self.device)
        self.batch_size = params.batch_size
        dev = self.device
        real = self.real
        self.treal = torch.float32 if precision == 'f32' else torch.float64

        def put(a, dtype=None):
            if a is None:
                return None
            t = torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype)))
            return t.to(dev)

        e, s = arrays.e_num, arrays.s_num
        self.t = {
            'x': put(arrays.x, real), 'y': put(arrays.y, real), 'area': put(arrays.area, real),
            'width': put(arrays.width, real), 'height': put(arrays.height, real), 'f0': put(arrays.f0, real),
            'fc': put(arrays.fc, real), 'k': put(arrays.k, real),
            'weight': put(arrays.weight, real), 'boundary_id': put(arrays.boundary_id),
            'rain_index': put(arrays.rain_index), 'face_ptr': put(arrays.face_ptr),
            'face_count': put(arrays.face_count),
            'isl_data': put(arrays.isl_data if len(arrays.isl_data) else np.zeros(1, np.int32)),
            'topology': put(arrays.topology), 'length': put(arrays.length, real),
            'side_n': put(arrays.side_n, real),
            'sbf': put(arrays.sbf), 'kind': put(arrays.kind), 'open_face': put(arrays.open_face, real),
            'edge_index': put(arrays.edge_index), 'offsets': put(arrays.offsets, real), 'slots': put(arrays.slots),
            'hcells': put(arrays.hcells), 'axes': put(arrays.axes),
            'bed': put(arrays.bed, real),
        }
        with torch.cuda.device(dev):
            for name in STATE_F32:
                if name != 'bed':
                    self.t[name] = torch.zeros(s if name == 'q' else e, dtype=self.treal, device=dev)
            for name in STATE_U32:
                self.t[name] = torch.zeros(e, dtype=torch.int32, device=dev)
        mesh = NhfMesh()
        mesh.e_num, mesh.s_num, mesh.b_num = e, s, arrays.b_num
        mesh.n_rates, mesh.isl_len = arrays.n_rates, len(arrays.isl_data)
        mesh.hang_cells, mesh.hang_edges = arrays.hang_cells, arrays.hang_edges
        for name in _MESH_PTRS:
            tensor = self.t.get(name)
            setattr(mesh, name, tensor.data_ptr() if tensor is not None else None)
        self._mesh = mesh
        path = path_code(params.path)
        cfl_mode = {'auto': 0, 'fused': 1, 'pass': 2}[params.cfl]
        if arrays.gate is not None:
            # the controller runs on the fused step with 256-cell tiles and the
            # separate CFL pass, or on the multi-pass step
            if path not in (0, 1, 256) or (path != 1 and params.cfl == 'fused'):
                raise ValueError('gate control needs path "auto", "tile256" or "multipass" and a separate CFL pass')
            if path != 1:
                path, cfl_mode = 256, 2
        if precision == 'f64' and arrays.gate is not None:
            raise ValueError('the FP64 build has no gate controller')
        p = self._params_type(params.g, params.afa, params.sita, params.min_h, params.min_dt, params.batch_size,
                              path, cfl_mode)
        handle = c_void_p()
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev).cuda_stream
            rc = self.lib.nhf_create(ctypes.byref(mesh), ctypes.byref(p), c_void_p(stream), ctypes.byref(handle))
        if rc != 0:
            raise RuntimeError(f'nhf_create failed ({rc}): {self.lib.nhf_last_error(None).decode()}')
        self.h = handle
        self.terms = self.lib.nhf_budget_terms(self.h)
        self.path = self.lib.nhf_path(self.h).decode()
        self._trace = np.zeros((self.batch_size, NHF_TRACE_COLS), dtype=np.uint32)
        self.gate = arrays.gate
        if self.gate is not None:
            self._attach_gate(self.gate)

    def _attach_gate(self, tables):
        """Device copies of the controller tables and words, attached to the
        handle (nhf_gate_attach)."""
        from .gate import STATE_FIELDS
        torch, dev = self.torch, self.device
        gate = NhfGate()
        gate.count, gate.n_targets, gate.n_flux = tables.count, len(tables.targets), len(tables.flux_sides)
        self.gt = {}
        for name in _GATE_TABLES:
            a = getattr(tables, name)
            a = np.ascontiguousarray(a, dtype=self.real if name == 'closed' else np.int32)
            t = torch.from_numpy(a if len(a) else np.zeros(1, a.dtype)).to(dev)
            self.gt[name] = t
            setattr(gate, name, t.data_ptr())
        gate.formal_tick[0], gate.formal_tick[1] = tables.formal_tick >> 32, tables.formal_tick & 0xffffffff
        gate.trigger_level, gate.opening_seconds = tables.trigger_level, tables.opening_seconds
        gate.open_elevation = tables.open_elevation
        self.gate_fields = STATE_FIELDS
        for name, dtype, width in STATE_FIELDS:
            t = torch.zeros((tables.count, width) if width > 1 else tables.count, dtype=torch.int32, device=dev)
            self.gt[name] = t
            setattr(gate, name, t.data_ptr())
        self._gate = gate
        self._check(self.lib.nhf_gate_attach(self.h, ctypes.byref(gate)), 'nhf_gate_attach')
        self.gate_terms = self.lib.nhf_gate_terms(self.h)

    def gate_check(self):
        self._check(self.lib.nhf_gate_check(self.h), 'nhf_gate_check')

    def gate_flush(self):
        out = np.zeros(self.gate_terms, dtype=np.float64)
        self._check(self.lib.nhf_gate_flush(self.h, out.ctypes.data_as(POINTER(c_double))), 'nhf_gate_flush')
        return out

    def gate_state(self) -> dict:
        """The controller words (commanded, command ticks, first flow,
        opened) as host arrays."""
        out = {}
        for name, dtype, _ in self.gate_fields:
            out[name] = self.gt[name].cpu().numpy().view(dtype) if dtype == np.uint32 else \
                self.gt[name].cpu().numpy().astype(dtype)
        return out

    def set_gate_state(self, state: dict) -> None:
        for name, dtype, _ in self.gate_fields:
            t = self.gt[name]
            a = np.ascontiguousarray(np.asarray(state[name]).astype(dtype).reshape(tuple(t.shape)))
            t.copy_(self.torch.from_numpy(a.view(np.int32)))

    # -- helpers ----------------------------------------------------------
    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f'{what} failed ({rc}): {self.lib.nhf_last_error(self.h).decode()}')

    def get(self, name):
        t = self.t[name]
        out = t.cpu().numpy()
        return out.view(np.uint32) if name in STATE_U32 else out

    def set(self, name, values):
        t = self.t[name]
        arr = np.ascontiguousarray(values)
        if name in STATE_U32:
            arr = arr.astype(np.uint32).view(np.int32)
        else:
            arr = arr.astype(self.real)
        if arr.shape != tuple(t.shape):
            raise ValueError(f'{name}: shape {arr.shape} differs from {tuple(t.shape)}')
        t.copy_(self.torch.from_numpy(arr))

    def initialize(self):
        self._check(self.lib.nhf_initialize(self.h), 'nhf_initialize')

    def set_clock(self, words):
        w, p = _u32(words)
        self._check(self.lib.nhf_set_clock(self.h, p), 'nhf_set_clock')

    def get_clock(self):
        w = np.zeros(2, np.uint32)
        self._check(self.lib.nhf_get_clock(self.h, w.ctypes.data_as(POINTER(c_uint32))), 'nhf_get_clock')
        return w

    def set_active(self, active):
        self._check(self.lib.nhf_set_active(self.h, int(active)), 'nhf_set_active')

    def set_forcing(self, coefficients, rain_rates, raining):
        coef = None if coefficients is None else np.ascontiguousarray(coefficients, dtype=self.real)
        rates = None if rain_rates is None else np.ascontiguousarray(rain_rates, dtype=self.real)
        if coef is not None and coef.shape != (max(1, self.arrays.b_num), 2):
            raise ValueError(f'coefficients must be [{max(1, self.arrays.b_num)}, 2], got {coef.shape}')
        if rates is not None and rates.shape != (self.arrays.n_rates,):
            raise ValueError(f'rain rates must be [{self.arrays.n_rates}], got {rates.shape}')
        self._check(self.lib.nhf_set_forcing(
            self.h, coef.ctypes.data_as(POINTER(self.creal)) if coef is not None else None,
            rates.ctypes.data_as(POINTER(self.creal)) if rates is not None else None, int(bool(raining))),
            'nhf_set_forcing')

    def apply_initial_levels(self, targets):
        t = self.torch.from_numpy(np.ascontiguousarray(targets, dtype=self.real)).to(self.device)
        self._check(self.lib.nhf_apply_initial_levels(self.h, c_void_p(t.data_ptr())), 'nhf_apply_initial_levels')
        self.torch.cuda.current_stream(self.device).synchronize()  # t stays alive until the kernel has read it

    def compute_cfl(self):
        self._check(self.lib.nhf_compute_cfl(self.h), 'nhf_compute_cfl')

    def initial_diagnostics(self):
        self._check(self.lib.nhf_initial_diagnostics(self.h), 'nhf_initial_diagnostics')

    def reset_extrema(self):
        self._check(self.lib.nhf_reset_extrema(self.h), 'nhf_reset_extrema')

    def run_batch(self, target_words, origin_words):
        t, tp = _u32(target_words)
        o, op = _u32(origin_words)
        self._check(self.lib.nhf_run_batch(self.h, tp, op, self._trace.ctypes.data_as(POINTER(c_uint32))),
                    'nhf_run_batch')
        return self._trace.copy()

    def run_batch_async(self, target_words, origin_words):
        t, tp = _u32(target_words)
        o, op = _u32(origin_words)
        self._check(self.lib.nhf_run_batch_async(self.h, tp, op), 'nhf_run_batch_async')

    def read_trace(self):
        self._check(self.lib.nhf_read_trace(self.h, self._trace.ctypes.data_as(POINTER(c_uint32))), 'nhf_read_trace')
        return self._trace.copy()

    def budget_flush(self):
        out = np.zeros(self.terms, dtype=np.float64)
        self._check(self.lib.nhf_budget_flush(self.h, out.ctypes.data_as(POINTER(c_double))), 'nhf_budget_flush')
        return out

    def cfl(self):
        ndt, arg, h = self.creal(), c_int32(), self.creal()
        self._check(self.lib.nhf_get_cfl(self.h, ctypes.byref(ndt), ctypes.byref(arg), ctypes.byref(h)), 'nhf_get_cfl')
        return float(ndt.value), int(arg.value), float(h.value)

    def limits(self):
        values = np.zeros(5, self.real)
        ids = np.zeros(3, np.int32)
        self._check(self.lib.nhf_limits(self.h, values.ctypes.data_as(POINTER(self.creal)),
                                        ids.ctypes.data_as(POINTER(c_int32))), 'nhf_limits')
        return values, ids

    def reset_limits(self):
        self._check(self.lib.nhf_reset_limits(self.h), 'nhf_reset_limits')

    def sample_stations(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((len(ids), 4), self.real)
        if len(ids):
            self._check(self.lib.nhf_sample_stations(self.h, ids.ctypes.data_as(POINTER(c_int32)), len(ids),
                                                     out.ctypes.data_as(POINTER(self.creal))), 'nhf_sample_stations')
        return out

    def read_eq(self):
        out = self.torch.zeros((self.arrays.e_num, 4), dtype=self.treal, device=self.device)
        self._check(self.lib.nhf_read_eq(self.h, c_void_p(out.data_ptr())), 'nhf_read_eq')
        return out.cpu().numpy()

    def stream(self):
        """torch view of the library stream the batches run on."""
        return self.torch.cuda.ExternalStream(self.lib.nhf_stream(self.h), device=self.device)

    def synchronize(self):
        self._check(self.lib.nhf_synchronize(self.h), 'nhf_synchronize')

    def peak_memory(self):
        return int(self.torch.cuda.max_memory_allocated(self.device))

    def close(self):
        if getattr(self, 'h', None):
            self.lib.nhf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaEnsemble:
    """Member CudaEngines advanced together (nhf_ensemble_*), each with its
    own clock and dt: with grid_blocks = -2 every member's own batch graph,
    all launched together on their own streams; otherwise one fused step
    launch per slot for all members, which must then be on the fused tiled
    step with one tile size. Batches are ordered after the current torch
    stream and the members' creation streams."""

    def __init__(self, engines, grid_blocks: int = 0):
        if not engines:
            raise ValueError('an ensemble needs at least one member')
        self.lib = library()
        self.engines = list(engines)
        self.torch = engines[0].torch
        self.device = engines[0].device
        self.batch_size = engines[0].batch_size
        handles = (c_void_p * len(engines))(*[e.h.value for e in engines])
        handle = c_void_p()
        with self.torch.cuda.device(self.device):
            stream = self.torch.cuda.current_stream(self.device).cuda_stream
            rc = self.lib.nhf_ensemble_create(handles, len(engines), int(grid_blocks), c_void_p(stream),
                                              ctypes.byref(handle))
        if rc != 0:
            raise RuntimeError(f'nhf_ensemble_create failed ({rc}): {self.lib.nhf_ensemble_last_error(None).decode()}')
        self.h = handle
        info = (c_int32 * 6)()
        self.lib.nhf_ensemble_info(self.h, info)
        self.members, self.tile, self.grid, self.tiles, _, self.shared_bytes = list(info)
        n = len(engines)
        self._targets = np.zeros((n, 2), np.uint32)
        self._origins = np.zeros((n, 2), np.uint32)
        self._trace = np.zeros((n, self.batch_size, NHF_TRACE_COLS), np.uint32)

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f'{what} failed ({rc}): {self.lib.nhf_ensemble_last_error(self.h).decode()}')

    def _words(self, targets, origins):
        self._targets[:] = np.asarray(targets, np.uint32).reshape(-1, 2)
        self._origins[:] = np.asarray(origins, np.uint32).reshape(-1, 2)
        return (self._targets.ctypes.data_as(POINTER(c_uint32)), self._origins.ctypes.data_as(POINTER(c_uint32)))

    def run_batch(self, targets, origins):
        """targets, origins: [members][2] tick words; returns the traces
        [members][batch_size][NHF_TRACE_COLS]."""
        tp, op = self._words(targets, origins)
        self._check(self.lib.nhf_ensemble_run_batch(self.h, tp, op, self._trace.ctypes.data_as(POINTER(c_uint32))),
                    'nhf_ensemble_run_batch')
        return self._trace.copy()

    def run_batch_async(self, targets, origins):
        tp, op = self._words(targets, origins)
        self._check(self.lib.nhf_ensemble_run_batch_async(self.h, tp, op), 'nhf_ensemble_run_batch_async')

    def read_trace(self):
        self._check(self.lib.nhf_ensemble_read_trace(self.h, self._trace.ctypes.data_as(POINTER(c_uint32))),
                    'nhf_ensemble_read_trace')
        return self._trace.copy()

    def stream(self):
        return self.torch.cuda.ExternalStream(self.lib.nhf_ensemble_stream(self.h), device=self.device)

    def close(self):
        if getattr(self, 'h', None):
            self.lib.nhf_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
