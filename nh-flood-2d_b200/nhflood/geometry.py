"""Mesh geometry and per-cell/per-side parameter arrays (host, once per run).

Same results as the reference's setup helpers, computed in this module's
own way:
  * ``MeshGeometry.from_mesh``        – preprocess/force.py:27-80 (cell bounds
                                        from the first side of each face,
                                        square-cell check, exterior edges)
  * ``map_land_parameters``           – preprocess/hydraulics.py:63-93
  * ``open_boundary_face_fractions``  – preprocess/hydraulics.py:50-60
  * ``connected_still_water``         – preprocess/hydraulics.py:7-47 (the
                                        union-find becomes connected components
                                        of the same edge set)
  * ``hanging_geometry``              – core/pressure.py:19-45
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components

from .input import HortonInfiltration

LEFT, RIGHT, BOTTOM, TOP = 0, 1, 2, 3


@dataclass
class ExteriorEdges:
    side_ids: np.ndarray
    cell_ids: np.ndarray
    face_ids: np.ndarray  # 0 left, 1 right, 2 bottom, 3 top
    lengths: np.ndarray
    segments: np.ndarray  # [edge, endpoint, xy]


@dataclass
class MeshGeometry:
    x: np.ndarray
    y: np.ndarray
    bounds: np.ndarray  # [e, 4] = left, bottom, right, top as F64 of the F32 side coordinates
    area: np.ndarray    # F64, area[0] = 0
    exterior_edges: ExteriorEdges

    @classmethod
    def from_mesh(cls, mesh) -> 'MeshGeometry':
        e = mesh.e_num
        bounds = np.zeros((e, 4), dtype=np.float64)
        if len(mesh.isl_data):
            # A face's first side carries the face coordinate: x for l/r, y for b/t.
            first = mesh.isl_data[np.clip(mesh.face_ptr, 0, len(mesh.isl_data) - 1)]
            bounds[:, 0] = mesh.side_x[first[:, LEFT]]
            bounds[:, 1] = mesh.side_y[first[:, BOTTOM]]
            bounds[:, 2] = mesh.side_x[first[:, RIGHT]]
            bounds[:, 3] = mesh.side_y[first[:, TOP]]
        width = bounds[:, 2] - bounds[:, 0]
        height = bounds[:, 3] - bounds[:, 1]
        if (width[1:] <= 0).any() or (height[1:] <= 0).any():
            raise ValueError('Mesh cells must have positive rectangular areas')
        if (width[1:] != height[1:]).any():
            raise ValueError('Mesh cells must be square for the edge-length CFL scale')
        area = width * height
        area[0] = 0.0
        return cls(mesh.x.astype(np.float64), mesh.y.astype(np.float64), bounds, area,
                   _exterior_edges(mesh, bounds))


def _exterior_edges(mesh, bounds) -> ExteriorEdges:
    topo = mesh.topology
    side_ids = np.flatnonzero((topo[:, 1] == 0) != (topo[:, 2] == 0))
    orient = topo[side_ids, 0]
    if not np.isin(orient, (1, 2)).all():
        raise ValueError('Exterior sides must be horizontal or vertical')
    cells = topo[side_ids, 1] + topo[side_ids, 2]
    sx = mesh.side_x[side_ids].astype(np.float64)
    sy = mesh.side_y[side_ids].astype(np.float64)
    half = mesh.side_length[side_ids].astype(np.float64)
    vertical = orient == 2
    b = bounds[cells]
    hits = np.stack([vertical & (sx == b[:, 0]), vertical & (sx == b[:, 2]),
                     ~vertical & (sy == b[:, 1]), ~vertical & (sy == b[:, 3])], axis=1)
    if (hits.sum(axis=1) != 1).any():
        raise ValueError('Exterior side does not lie on one cell face')
    # Segment endpoints: the side centre moved half a length along the side.
    along = np.where(vertical[:, None], [0.0, 1.0], [1.0, 0.0]) * (half / 2)[:, None]
    centre = np.column_stack([sx, sy])
    segments = np.stack([centre - along, centre + along], axis=1)
    return ExteriorEdges(side_ids, cells, hits.argmax(axis=1), half, segments)


def map_land_parameters(table, land_types: np.ndarray, side_topology: np.ndarray):
    """Side Manning n and cell Horton f0/fc (m/s), k (1/h) from land classes.

    Class lookups go through 256-entry F32 tables; the Horton rates are
    converted in F32 as NumPy 2 does for the reference's ``mm/h * F32(1/3.6e6)``.
    Cell 0 (exterior) has zero parameters; an exterior side takes its one
    interior cell's n (a mirrored ghost cell), an interior side the F32 mean.
    """
    present = set(np.unique(land_types[1:]).tolist())
    missing = sorted(present - set(table.keys()))
    if missing:
        raise ValueError(f'land_parameters missing land types: {missing}')
    lut = np.zeros((4, 256), dtype=np.float32)  # n, f0, fc, k
    to_m_s = np.float32(1.0 / 3_600_000.0)
    for cls_id in present:
        p = table[int(cls_id)]
        lut[0, cls_id] = p.manning_n
        if isinstance(p.infiltration, HortonInfiltration):
            lut[1, cls_id] = np.float32(p.infiltration.f0_mm_h) * to_m_s
            lut[2, cls_id] = np.float32(p.infiltration.fc_mm_h) * to_m_s
            lut[3, cls_id] = p.infiltration.k_per_h
    cell = lut[:, land_types.astype(np.intp)]
    cell[:, 0] = 0.0
    n_cell = cell[0]
    lo, hi = side_topology[:, 1], side_topology[:, 2]
    pair_sum = n_cell[lo] + n_cell[hi]
    interior = (lo != 0) & (hi != 0)
    side_n = np.where(interior, pair_sum * np.float32(0.5), pair_sum).astype(np.float32)
    return side_n, cell[1].copy(), cell[2].copy(), cell[3].copy()


def open_boundary_face_fractions(selected_sides, side_lengths, side_topology,
                                 face_ptrs, face_counts, flat_side_ids):
    """[e, 4] F32: selected exterior length / total length of each face of the
    cells that own a selected side (other cells stay zero)."""
    out = np.zeros((len(face_ptrs), 4), dtype=np.float32)
    owners = np.unique(side_topology[selected_sides][:, 1:].sum(axis=1))
    for cell in owners:
        for face in range(4):
            start = int(face_ptrs[cell, face])
            ids = flat_side_ids[start:start + int(face_counts[cell, face])]
            lens = side_lengths[ids].astype(np.float64)
            out[cell, face] = lens[selected_sides[ids]].sum() / lens.sum()
    return out


def connected_still_water(bed, side_crest, closed_sides, side_topology, boundaries, area):
    """Warm-up fill: each distinct initial level floods the cells connected to
    its level-boundary seeds through open interior sides whose crest lies
    strictly below the level. Two different levels reaching one water body
    are rejected."""
    bed64 = np.asarray(bed, dtype=np.float64)
    crest = np.maximum(np.maximum(bed64[side_topology[:, 1]], bed64[side_topology[:, 2]]),
                       np.asarray(side_crest, dtype=np.float64))
    passable = ((side_topology[:, 1] != 0) & (side_topology[:, 2] != 0)
                & ~np.asarray(closed_sides).astype(bool))
    groups: dict[float, list] = {}
    for b in boundaries:
        if b.kind == 'level':
            groups.setdefault(b.series.at(0.0), []).append(b)
    depth = np.zeros(len(bed64), dtype=np.float32)
    bodies = []
    n = len(bed64)
    for level, members in groups.items():
        seeds = np.unique(np.concatenate([b.cells for b in members]))
        seeds = seeds[bed64[seeds] < level]
        if seeds.size == 0:
            continue
        open_edges = passable & (crest < level)
        lo, hi = side_topology[open_edges, 1], side_topology[open_edges, 2]
        adjacency = coo_matrix((np.ones(lo.size), (lo, hi)), shape=(n, n))
        _, label = connected_components(adjacency, directed=False)
        bodies_hit = np.unique(label[seeds])
        flooded = np.isin(label, bodies_hit)
        for other, others in groups.items():
            if other == level:
                continue
            for b in others:
                if flooded[b.cells].any():
                    names = ', '.join(m.name for m in members)
                    raise ValueError('Conflicting initial levels on connected water body: '
                                     f'{names} ({level}) and {b.name} ({other})')
        depth[flooded] = level - bed64[flooded]
        bodies.append(dict(level_m=float(level), boundaries=[m.name for m in members],
                           connected_components=int(bodies_hit.size),
                           wet_cells=int(flooded.sum())))
    storage = float(np.dot(depth.astype(np.float64), area))
    return depth, dict(wet_cells=int(np.count_nonzero(depth)), storage_m3=storage, levels=bodies)


@dataclass
class HangingGeometry:
    edge_index: np.ndarray      # [s] -> hanging edge slot or -1
    offsets: np.ndarray         # [E, 2] F32 tangential offset of lower/higher centre
    gradient_slots: np.ndarray  # [E, 2] gradient-cell slot or -1
    cells: np.ndarray           # [C] sorted gradient cells
    axes: np.ndarray            # [C, 2] 1 where a gradient along x / y is needed


def hanging_geometry(x, y, side_x, side_y, topology):
    """Interior sides whose neighbour centres are displaced along the side
    (2:1 hanging interfaces) and the cells whose tangential gradient they
    need; None when every centre is aligned."""
    vertical = topology[:, 0] == 2
    nbr = topology[:, 1:]
    # tangential coordinate: y along a vertical side, x along a horizontal one
    side_t = np.where(vertical, side_y, side_x)
    cell_t = np.where(vertical[:, None], y[nbr], x[nbr])
    offset = side_t[:, None] - cell_t
    interior = (nbr[:, 0] != 0) & (nbr[:, 1] != 0)
    edges = np.flatnonzero(interior & (offset != 0.0).any(axis=1))
    if edges.size == 0:
        return None
    offset = offset[edges].astype(np.float32)
    ends = nbr[edges]
    moved = offset != 0.0
    cells = np.unique(ends[moved]).astype(np.int32)
    slots = np.where(moved, np.searchsorted(cells, ends), -1).astype(np.int32)
    axes = np.zeros((cells.size, 2), dtype=np.int32)
    axis_of_edge = np.repeat(vertical[edges].astype(np.intp)[:, None], 2, axis=1)
    axes[slots[moved], axis_of_edge[moved]] = 1
    edge_index = np.full(len(topology), -1, dtype=np.int32)
    edge_index[edges] = np.arange(edges.size, dtype=np.int32)
    return HangingGeometry(edge_index, offset, slots, cells, axes)
