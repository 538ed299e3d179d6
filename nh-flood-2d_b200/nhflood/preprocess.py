"""NE/NS mesh preprocessing and the solver's mesh arrays.

Restates the reference's domain preparation (nh-flood-2d
src/nh_flood_2d/preprocess/domain.py):
  * ``filter_ne_ns``      – _filter_ne_ns (domain.py:221-347): drop cells with
                            z == -9999, drop sides left without a relevant
                            neighbour, renumber both;
  * ``build_ne_tables``   – create_ne_fdb_compact (domain.py:83-174): compact
                            CSR side lists ``isl_data`` + ``isl_ptr_{l,r,b,t}``;
  * ``build_ns_tables``   – create_ns_fdb_parallel/_batch_ns_worker
                            (domain.py:349-389,439-470): side records and
                            (orient, lower, higher) topology;
  * ``boundary_flags``    – build_boundary_fdb (domain.py:472-479): every
                            exterior side is closed (``sbf``).
Index 0 of cells and sides is the exterior sentinel (README.md:407).

NE line: ``id,l,r,b,t,<side ids>,x,y,z,type``; NS line:
``id,orient,left,right,bottom,top,length,x,y,z,attr`` (orient 1 horizontal,
2 vertical).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import fdb


@dataclass
class MeshData:
    """Arrays the step reads, in the reference's layout (index 0 sentinel)."""
    x: np.ndarray          # f32 [e]
    y: np.ndarray          # f32 [e]
    z: np.ndarray          # f32 [e] bed
    land_type: np.ndarray  # u8  [e]
    counts: np.ndarray     # i32 [e, 4] side counts l, r, b, t
    face_ptr: np.ndarray   # i32 [e, 4] isl_ptr_{l,r,b,t}
    isl_data: np.ndarray   # i32 [sum counts]
    index: np.ndarray      # u32 [e] NE id column
    side_length: np.ndarray  # f32 [s]
    side_x: np.ndarray     # f32 [s]
    side_y: np.ndarray     # f32 [s]
    side_z: np.ndarray     # f32 [s]
    side_attr: np.ndarray  # u8  [s]
    side_index: np.ndarray  # u32 [s]
    topology: np.ndarray   # i32 [s, 3] orient, lower, higher

    @property
    def e_num(self) -> int:
        return len(self.x)

    @property
    def s_num(self) -> int:
        return len(self.side_length)

    @property
    def sbf(self) -> np.ndarray:
        return boundary_flags(self.topology)


def boundary_flags(topology: np.ndarray) -> np.ndarray:
    """build_boundary_fdb (domain.py:472-479): exterior = exactly one neighbour."""
    return ((topology[:, 1] == 0) ^ (topology[:, 2] == 0)).astype(np.uint8)


def filter_ne_ns(ne_lines: list[str], ns_lines: list[str]) -> tuple[list[str], list[str]]:
    """_filter_ne_ns (domain.py:221-347) on in-memory lines."""
    ne_map: dict[int, int] = {}
    valid_ne = []
    for line in ne_lines:
        parts = line.strip().split(',')
        z_val = float(parts[-2])
        old = int(parts[0])
        if z_val != -9999:
            ne_map[old] = len(valid_ne) + 1
            valid_ne.append(parts)
    ns_map: dict[int, int] = {}
    out_ns = []
    for line in ns_lines:
        parts = line.strip().split(',')
        if len(parts) < 6:
            continue
        old_id, orient = int(parts[0]), int(parts[1])
        left, right, bottom, top = (ne_map.get(int(v), 0) for v in parts[2:6])
        keep = (bottom != 0 or top != 0) if orient == 1 else (left != 0 or right != 0)
        if keep:
            ns_map[old_id] = len(out_ns) + 1
            parts[0] = str(len(out_ns) + 1)
            parts[2], parts[3], parts[4], parts[5] = str(left), str(right), str(bottom), str(top)
            out_ns.append(','.join(parts))
    out_ne = []
    for parts in valid_ne:
        parts = list(parts)
        parts[0] = str(ne_map[int(parts[0])])
        total = sum(int(parts[i]) for i in range(1, 5))
        for i in range(5, 5 + total):
            parts[i] = str(ns_map.get(int(parts[i]), 0))
        out_ne.append(','.join(parts))
    return out_ne, out_ns


def build_ne_tables(ne_lines: list[str]) -> dict[str, np.ndarray]:
    """create_ne_fdb_compact (domain.py:83-174)."""
    e = len(ne_lines) + 1
    index = np.zeros(e, np.uint32)
    xyz = np.zeros((e, 3), np.float32)
    land = np.zeros(e, np.uint8)
    counts = np.zeros((e, 4), np.int64)
    ptr = np.zeros((e, 4), np.int64)
    flat = []
    offset = 0
    for idx, line in enumerate(ne_lines, start=1):
        data = line.split(',')
        c = [int(data[1]), int(data[2]), int(data[3]), int(data[4])]
        total = c[0] + c[1] + c[2] + c[3]
        flat.append(np.array([int(v) for v in data[5:5 + total]], dtype=np.int64))
        index[idx] = int(data[0])
        xyz[idx] = (float(data[-4]), float(data[-3]), float(data[-2]))
        land[idx] = int(data[-1])
        counts[idx] = c
        ptr[idx] = (offset, offset + c[0], offset + c[0] + c[1], offset + c[0] + c[1] + c[2])
        offset += total
    isl = np.concatenate(flat) if flat else np.zeros(0, np.int64)
    return dict(index=index, x=xyz[:, 0].copy(), y=xyz[:, 1].copy(), z=xyz[:, 2].copy(), type=land,
                counts=counts.astype(np.uint32), ptr=ptr.astype(np.uint32), isl=isl.astype(np.uint32))


def build_ns_tables(ns_lines: list[str]) -> dict[str, np.ndarray]:
    """create_ns_fdb_parallel / _batch_ns_worker (domain.py:439-470)."""
    s = len(ns_lines) + 1
    index = np.zeros(s, np.uint32)
    vals = np.zeros((s, 4), np.float32)
    attr = np.zeros(s, np.uint8)
    topo = np.zeros((s, 3), np.uint32)
    for idx, line in enumerate(ns_lines, start=1):
        data = line.split(',')
        orient, left, right, bottom, top = (int(v) for v in data[1:6])
        topo[idx] = (orient, bottom, top) if orient == 1 else (orient, left, right)
        index[idx] = int(data[0])
        vals[idx] = (float(data[6]), float(data[7]), float(data[8]), float(data[9]))
        attr[idx] = int(float(data[10]))
    return dict(index=index, length=vals[:, 0].copy(), x=vals[:, 1].copy(), y=vals[:, 2].copy(),
                z=vals[:, 3].copy(), attr=attr, topo=topo)


def _write_ne(path, t):
    e = len(t['x'])
    fdb.save(path, [
        ('IndexLike', 'isl_data', {'index': t['isl']}),
        ('IndexLike', 'isl_ptr_l', {'index': t['ptr'][:, 0]}),
        ('IndexLike', 'isl_ptr_r', {'index': t['ptr'][:, 1]}),
        ('IndexLike', 'isl_ptr_b', {'index': t['ptr'][:, 2]}),
        ('IndexLike', 'isl_ptr_t', {'index': t['ptr'][:, 3]}),
        ('Ne', None, {'index': t['index'], 'x': t['x'], 'y': t['y'], 'z': t['z'],
                      'l_side_num': t['counts'][:, 0], 'r_side_num': t['counts'][:, 1],
                      'b_side_num': t['counts'][:, 2], 't_side_num': t['counts'][:, 3],
                      'type': t['type'][:e]}),
    ])


def _write_ns(path, t):
    fdb.save(path, [
        ('Ns', None, {'index': t['index'], 'length': t['length'], 'x': t['x'], 'y': t['y'],
                      'z': t['z'], 'attr': t['attr']}),
        ('SideTopoInfo', None, {'info': t['topo'].reshape(-1)}),
    ])


_PREP = None


def native_library():
    """libnhfprep.so (csrc/host/nhf_prep.cpp, include/nhf_prep.h), or None
    when it has not been built."""
    global _PREP
    if _PREP is None:
        import ctypes
        from .build import PREP_LIBRARY
        if not PREP_LIBRARY.exists():
            return None
        lib = ctypes.CDLL(str(PREP_LIBRARY))
        P, V, I64 = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64
        lib.nhp_prepare.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                    ctypes.POINTER(P)]
        lib.nhp_sizes.argtypes = [P, ctypes.POINTER(I64)]
        lib.nhp_copy_cells.argtypes = [P] + [V] * 8
        lib.nhp_copy_sides.argtypes = [P] + [V] * 7
        lib.nhp_free.argtypes = [P]
        lib.nhp_error.restype = ctypes.c_char_p
        _PREP = lib
    return _PREP


def native_tables(ne_text: bytes, ns_text: bytes) -> tuple[dict, dict]:
    """filter_ne_ns + build_ne_tables + build_ns_tables in C++: the same
    tables, for meshes where the per-line Python passes are too slow."""
    import ctypes
    lib = native_library()
    if lib is None:
        raise RuntimeError('libnhfprep.so is not built (python -m nhflood.build)')
    h = ctypes.c_void_p()
    if lib.nhp_prepare(ne_text, len(ne_text), ns_text, len(ns_text), ctypes.byref(h)) != 0:
        raise ValueError(f'NE/NS preprocessing failed: {lib.nhp_error().decode()}')
    try:
        sizes = (ctypes.c_int64 * 3)()
        lib.nhp_sizes(h, sizes)
        e, s, n = int(sizes[0]), int(sizes[1]), int(sizes[2])
        ne = dict(index=np.zeros(e, np.uint32), x=np.zeros(e, np.float32), y=np.zeros(e, np.float32),
                  z=np.zeros(e, np.float32), type=np.zeros(e, np.uint8), counts=np.zeros((e, 4), np.uint32),
                  ptr=np.zeros((e, 4), np.uint32), isl=np.zeros(n, np.uint32))
        ns = dict(index=np.zeros(s, np.uint32), length=np.zeros(s, np.float32), x=np.zeros(s, np.float32),
                  y=np.zeros(s, np.float32), z=np.zeros(s, np.float32), attr=np.zeros(s, np.uint8),
                  topo=np.zeros((s, 3), np.uint32))
        lib.nhp_copy_cells(h, *(ne[k].ctypes.data for k in ('index', 'x', 'y', 'z', 'type', 'counts', 'ptr', 'isl')))
        lib.nhp_copy_sides(h, *(ns[k].ctypes.data for k in ('index', 'length', 'x', 'y', 'z', 'attr', 'topo')))
    finally:
        lib.nhp_free(h)
    return ne, ns


def prepare_domain(cfg) -> None:
    """prepare_domain (domain.py:590-606): filter, build ne/ns/boundary tables.
    Uses the C++ preprocessing when libnhfprep.so is built (the same tables),
    else the Python restatement below."""
    if native_library() is not None:
        ne, ns = native_tables(Path(cfg.ne).read_bytes(), Path(cfg.ns).read_bytes())
        _write_ne(cfg.ne_fdb, ne)
        _write_ns(cfg.ns_fdb, ns)
        fdb.save(cfg.boundary_fdb, [('U8Value', 'sbf', {'value': boundary_flags(ns['topo'].astype(np.int64))})])
        return
    try:
        ne_lines = Path(cfg.ne).read_text(encoding='utf-8').splitlines(keepends=True)
        ns_lines = Path(cfg.ns).read_text(encoding='utf-8').splitlines(keepends=True)
        ne_out, ns_out = filter_ne_ns(ne_lines, ns_lines)
        Path(cfg.tmp_ne).write_text(''.join(line + '\n' for line in ne_out), encoding='utf-8')
        Path(cfg.tmp_ns).write_text(''.join(line + '\n' for line in ns_out), encoding='utf-8')
        ne = build_ne_tables(ne_out)
        ns = build_ns_tables(ns_out)
        _write_ne(cfg.ne_fdb, ne)
        _write_ns(cfg.ns_fdb, ns)
        fdb.save(cfg.boundary_fdb, [('U8Value', 'sbf', {'value': boundary_flags(ns['topo'].astype(np.int64))})])
    finally:
        for tmp in (cfg.tmp_ne, cfg.tmp_ns):
            if Path(tmp).exists():
                os.remove(tmp)


def preprocess(domain_cfg, force_cfg=None) -> None:
    """preprocess/__init__.py:5-6."""
    prepare_domain(domain_cfg)


def load_mesh(cfg) -> tuple[MeshData, np.ndarray]:
    """Read the prepared tables (solver_compact.py:183-200); returns the mesh
    and the ``sbf`` exterior flags."""
    ne_db, ns_db, bd_db = fdb.load(cfg.ne_fdb), fdb.load(cfg.ns_fdb), fdb.load(cfg.boundary_fdb)
    ne = ne_db.table('Ne')
    ns = ns_db.table('Ns')
    isl = ne_db.table('IndexLike', 'isl_data')['index'].astype(np.int32)
    ptr = np.column_stack([ne_db.table('IndexLike', f'isl_ptr_{d}')['index'] for d in 'lrbt']).astype(np.int32)
    counts = np.column_stack([ne[f'{d}_side_num'] for d in 'lrbt']).astype(np.int32)
    topo = ns_db.table('SideTopoInfo')['info'].astype(np.int64).reshape(-1, 3).astype(np.int32)
    sbf = bd_db.table('U8Value', 'sbf')['value']
    mesh = MeshData(x=ne['x'], y=ne['y'], z=ne['z'], land_type=ne['type'], counts=counts, face_ptr=ptr,
                    isl_data=isl, index=ne['index'], side_length=ns['length'], side_x=ns['x'],
                    side_y=ns['y'], side_z=ns['z'], side_attr=ns['attr'], side_index=ns['index'],
                    topology=topo)
    return mesh, sbf


def write_ne_ns(mesh: MeshData, ne_path, ns_path) -> None:
    """Write a mesh back to NE/NS text (the inverse of build_*_tables)."""
    lines = []
    for ei in range(1, mesh.e_num):
        c = mesh.counts[ei]
        p = mesh.face_ptr[ei, 0]
        ids = mesh.isl_data[p:p + int(c.sum())]
        fields = [str(ei), *map(str, c), *map(str, ids),
                  repr(float(mesh.x[ei])), repr(float(mesh.y[ei])), repr(float(mesh.z[ei])),
                  str(int(mesh.land_type[ei]))]
        lines.append(','.join(fields))
    Path(ne_path).write_text('\n'.join(lines) + '\n', encoding='utf-8')
    lines = []
    for si in range(1, mesh.s_num):
        o, lo, hi = (int(v) for v in mesh.topology[si])
        nb = (0, 0, lo, hi) if o == 1 else (lo, hi, 0, 0)
        lines.append(','.join([str(si), str(o), *map(str, nb), repr(float(mesh.side_length[si])),
                               repr(float(mesh.side_x[si])), repr(float(mesh.side_y[si])),
                               repr(float(mesh.side_z[si])), str(int(mesh.side_attr[si]))]))
    Path(ns_path).write_text('\n'.join(lines) + '\n', encoding='utf-8')
