"""Host description of one solve: the arrays and scalars the step reads.

``StepArrays`` is what the reference uploads to Taichi fields in _evolve
(solver_compact.py:209-268,320-336): per-cell and per-side parameter arrays
in the reference's layout (index 0 is the exterior sentinel), the boundary
cell mapping, rain pixel index, land parameters, theta-scheme open-face
fractions and the hanging-edge reconstruction indices.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .geometry import hanging_geometry, map_land_parameters, open_boundary_face_fractions

STATE_F32 = ('bed', 'depth', 'q', 'rain_time', 'infiltration', 'max_depth', 'max_speed', 'u', 'v')
STATE_U32 = ('peak_hi', 'peak_lo')
G = np.float32(9.81)
MIN_DT = 1e-4


@dataclass
class StepParams:
    afa: float = 0.5
    sita: float = 1.0
    min_h: float = 0.02
    batch_size: int = 32
    g: float = float(G)
    min_dt: float = float(np.float32(MIN_DT))
    # 'auto': the lattice form on uniform grids, else the fused tiled step when
    # the mesh allows it, else multi-pass; 'lattice', 'tiled', 'tile256' /
    # 'tile512' / 'tile1024', 'multipass' ask for one form
    path: str = 'auto'
    # fused step: where the next step's CFL candidate is computed. 'auto': in
    # the step on meshes of less than two waves of tiles, else in a separate
    # pass; 'fused': always in the step; 'pass': always a separate pass
    cfl: str = 'auto'


@dataclass
class StepArrays:
    e_num: int
    s_num: int
    b_num: int
    n_rates: int
    x: np.ndarray
    y: np.ndarray
    bed: np.ndarray
    area: np.ndarray
    width: np.ndarray
    height: np.ndarray
    f0: np.ndarray
    fc: np.ndarray
    k: np.ndarray
    weight: np.ndarray
    boundary_id: np.ndarray
    rain_index: np.ndarray
    face_ptr: np.ndarray
    face_count: np.ndarray
    isl_data: np.ndarray
    topology: np.ndarray
    length: np.ndarray
    side_n: np.ndarray
    sbf: np.ndarray
    kind: np.ndarray
    open_face: np.ndarray | None = None
    edge_index: np.ndarray | None = None
    offsets: np.ndarray | None = None
    slots: np.ndarray | None = None
    hcells: np.ndarray | None = None
    axes: np.ndarray | None = None
    gate: object = None  # nhflood.gate.GateTables when a gate controller is enabled
    extra: dict = field(default_factory=dict)

    @property
    def hang_cells(self) -> int:
        return 0 if self.hcells is None else len(self.hcells)

    @property
    def hang_edges(self) -> int:
        return 0 if self.offsets is None else len(self.offsets)

    @property
    def terms(self) -> int:
        return 4 + 6 * self.b_num

    def nbytes(self) -> int:
        total = 0
        for value in self.__dict__.values():
            if isinstance(value, np.ndarray):
                total += value.nbytes
        return total


def build_step_arrays(mesh, sbf, geometry, forcing, land_parameters, sita: float) -> StepArrays:
    """Assemble the step inputs exactly as _evolve prepares its fields."""
    e_num, s_num = mesh.e_num, mesh.s_num
    side_n, f0, fc, k = map_land_parameters(land_parameters, mesh.land_type, mesh.topology)
    boundary_id = np.full(e_num, -1, dtype=np.int32)
    weight = np.zeros(e_num, dtype=np.float32)
    kind = np.zeros(max(1, len(forcing.boundaries)), dtype=np.int32)
    for i, b in enumerate(forcing.boundaries):
        boundary_id[b.cells] = i
        weight[b.cells] = b.weights
        kind[i] = int(b.kind == 'discharge')
    open_face = None
    if sita != 1.0:
        selected = np.zeros(s_num, dtype=bool)
        for b in forcing.boundaries:
            selected[b.side_ids] = True
        open_face = open_boundary_face_fractions(selected, mesh.side_length, mesh.topology,
                                                 mesh.face_ptr, mesh.counts, mesh.isl_data)
    widths = (geometry.bounds[:, 2] - geometry.bounds[:, 0]).astype(np.float32)
    heights = (geometry.bounds[:, 3] - geometry.bounds[:, 1]).astype(np.float32)
    arrays = StepArrays(
        e_num=e_num, s_num=s_num, b_num=len(forcing.boundaries),
        n_rates=int(forcing.rain.millimetres.shape[1]),
        x=mesh.x.astype(np.float32), y=mesh.y.astype(np.float32), bed=mesh.z.astype(np.float32),
        area=geometry.area.astype(np.float32), width=widths, height=heights,
        f0=f0, fc=fc, k=k, weight=weight, boundary_id=boundary_id,
        rain_index=forcing.rain.pixel_index.astype(np.int32),
        face_ptr=np.ascontiguousarray(mesh.face_ptr, dtype=np.int32),
        face_count=np.ascontiguousarray(mesh.counts, dtype=np.int32),
        isl_data=np.ascontiguousarray(mesh.isl_data, dtype=np.int32),
        topology=np.ascontiguousarray(mesh.topology, dtype=np.int32),
        length=mesh.side_length.astype(np.float32), side_n=side_n.astype(np.float32),
        sbf=np.ascontiguousarray(sbf, dtype=np.uint8), kind=kind, open_face=open_face)
    layout = hanging_geometry(mesh.x, mesh.y, mesh.side_x, mesh.side_y, mesh.topology)
    if layout is not None:
        arrays.edge_index = layout.edge_index
        arrays.offsets = layout.offsets
        arrays.slots = layout.gradient_slots
        arrays.hcells = layout.cells
        arrays.axes = layout.axes
    return arrays


class Engine:
    """Interface the driver uses; implemented by the CUDA engine
    (nhflood.native.CudaEngine). State names: STATE_F32 + STATE_U32."""

    backend = 'abstract'
    device_name = 'unavailable'

    def get(self, name: str) -> np.ndarray: raise NotImplementedError
    def set(self, name: str, values) -> None: raise NotImplementedError
    def initialize(self) -> None: raise NotImplementedError
    def set_clock(self, words) -> None: raise NotImplementedError
    def get_clock(self) -> np.ndarray: raise NotImplementedError
    def set_active(self, active: int) -> None: raise NotImplementedError
    def set_forcing(self, coefficients, rain_rates, raining: bool) -> None: raise NotImplementedError
    def apply_initial_levels(self, targets) -> None: raise NotImplementedError
    def compute_cfl(self) -> None: raise NotImplementedError
    def initial_diagnostics(self) -> None: raise NotImplementedError
    def reset_extrema(self) -> None: raise NotImplementedError
    def run_batch(self, target_words, origin_words) -> np.ndarray: raise NotImplementedError
    def budget_flush(self) -> np.ndarray: raise NotImplementedError
    def cfl(self) -> tuple[float, int, float]: raise NotImplementedError
    def limits(self) -> tuple[np.ndarray, np.ndarray]: raise NotImplementedError
    def reset_limits(self) -> None: raise NotImplementedError
    def sample_stations(self, ids) -> np.ndarray: raise NotImplementedError
    def peak_memory(self): return None
    def close(self) -> None: pass
