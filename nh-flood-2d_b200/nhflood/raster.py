"""Minimal GeoTIFF reader/writer for rainfall rasters.

The reference reads rain with rasterio (preprocess/force.py:180-193), which
is not installed here. This module handles the subset the solver needs:
baseline (uncompressed) TIFF, 32/64-bit float or integer samples, strips or
tiles, chunky or planar bands, an affine georeference from
ModelPixelScale + ModelTiepoint (or ModelTransformation), the EPSG code from
the GeoKey directory and GDAL's NoData tag. Compressed files are rejected
with a clear error.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

_TYPES = {1: ('B', 1), 2: ('s', 1), 3: ('H', 2), 4: ('I', 4), 5: ('II', 8), 11: ('f', 4), 12: ('d', 8),
          16: ('Q', 8)}


@dataclass
class Raster:
    data: np.ndarray             # [bands, rows, cols]
    transform: tuple             # (a, b, c, d, e, f): x = a*col + b*row + c, y = d*col + e*row + f
    epsg: int | None
    nodata: float | None

    @property
    def height(self) -> int:
        return self.data.shape[1]

    @property
    def width(self) -> int:
        return self.data.shape[2]

    @property
    def count(self) -> int:
        return self.data.shape[0]

    def rowcol(self, xs, ys):
        """Pixel row/col containing each point (floor), as rasterio.transform.rowcol."""
        a, b, c, d, e, f = self.transform
        det = a * e - b * d
        xs = np.asarray(xs, dtype=np.float64)
        ys = np.asarray(ys, dtype=np.float64)
        col = (e * (xs - c) - b * (ys - f)) / det
        row = (-d * (xs - c) + a * (ys - f)) / det
        return np.floor(row).astype(np.int64), np.floor(col).astype(np.int64)


def from_origin(west, north, xsize, ysize) -> tuple:
    return (float(xsize), 0.0, float(west), 0.0, -float(ysize), float(north))


def write_geotiff(path, data, transform, epsg: int, nodata: float | None = None) -> None:
    """Write [bands, rows, cols] float32 data, planar bands, one strip per band row block."""
    data = np.asarray(data, dtype='<f4')
    if data.ndim == 2:
        data = data[None]
    bands, rows, cols = data.shape
    a, b, c, d, e, f = transform
    entries = []  # (tag, type, count, payload bytes)

    def add(tag, typ, values):
        fmt, size = _TYPES[typ]
        if typ == 2:
            payload = values.encode('ascii') + b'\0'
            count = len(payload)
        else:
            values = list(values)
            payload = struct.pack('<' + fmt * len(values), *values)
            count = len(values)
        entries.append((tag, typ, count, payload))

    strip_offsets_placeholder = [0] * bands
    add(256, 4, [cols])
    add(257, 4, [rows])
    add(258, 3, [32] * bands)
    add(259, 3, [1])
    add(262, 3, [1])
    add(273, 4, strip_offsets_placeholder)
    add(277, 3, [bands])
    add(278, 4, [rows])
    add(279, 4, [rows * cols * 4] * bands)
    add(284, 3, [2])
    add(339, 3, [3] * bands)
    if b == 0 and d == 0:
        add(33550, 12, [a, -e, 0.0])
        add(33922, 12, [0.0, 0.0, 0.0, c, f, 0.0])
    else:
        add(34264, 12, [a, b, 0, c, d, e, 0, f, 0, 0, 1, 0, 0, 0, 0, 1])
    add(34735, 3, [1, 1, 0, 3, 1024, 0, 1, 1, 1025, 0, 1, 1, 3072, 0, 1, int(epsg)])
    if nodata is not None:
        add(42113, 2, repr(float(nodata)))
    entries.sort(key=lambda t: t[0])
    n = len(entries)
    ifd_offset = 8
    ifd_size = 2 + 12 * n + 4
    extra = ifd_offset + ifd_size
    # lay out out-of-line payloads, then the image data
    layout = {}
    cursor = extra
    for tag, typ, count, payload in entries:
        if len(payload) > 4:
            layout[tag] = cursor
            cursor += len(payload) + (len(payload) & 1)
    data_start = (cursor + 15) & ~15
    offsets = [data_start + i * rows * cols * 4 for i in range(bands)]
    fixed = []
    for tag, typ, count, payload in entries:
        if tag == 273:
            payload = struct.pack('<' + 'I' * bands, *offsets)
        fixed.append((tag, typ, count, payload))
    with open(path, 'wb') as out:
        out.write(b'II*\0' + struct.pack('<I', ifd_offset))
        out.write(struct.pack('<H', n))
        for tag, typ, count, payload in fixed:
            if len(payload) > 4:
                value = struct.pack('<I', layout[tag])
            else:
                value = payload + b'\0' * (4 - len(payload))
            out.write(struct.pack('<HHI', tag, typ, count) + value)
        out.write(struct.pack('<I', 0))
        for tag, typ, count, payload in fixed:
            if len(payload) > 4:
                out.seek(layout[tag])
                out.write(payload)
        out.seek(data_start)
        for band in range(bands):
            out.write(np.ascontiguousarray(data[band]).tobytes())


def read_geotiff(path) -> Raster:
    with open(path, 'rb') as f:
        blob = f.read()
    order = blob[:2]
    if order == b'II':
        e = '<'
    elif order == b'MM':
        e = '>'
    else:
        raise ValueError(f'{path}: not a TIFF file')
    magic = struct.unpack(e + 'H', blob[2:4])[0]
    if magic != 42:
        raise ValueError(f'{path}: BigTIFF or unknown TIFF variant is not supported')
    ifd = struct.unpack(e + 'I', blob[4:8])[0]
    count = struct.unpack(e + 'H', blob[ifd:ifd + 2])[0]
    tags = {}
    for i in range(count):
        base = ifd + 2 + 12 * i
        tag, typ, n = struct.unpack(e + 'HHI', blob[base:base + 8])
        if typ not in _TYPES:
            continue
        fmt, size = _TYPES[typ]
        total = size * n
        raw = blob[base + 8:base + 12] if total <= 4 else blob[struct.unpack(e + 'I', blob[base + 8:base + 12])[0]:][:total]
        if typ == 2:
            tags[tag] = raw[:n].rstrip(b'\0').decode('ascii', 'replace')
        elif typ == 5:
            vals = struct.unpack(e + 'I' * (2 * n), raw[:8 * n])
            tags[tag] = [vals[2 * k] / vals[2 * k + 1] for k in range(n)]
        else:
            tags[tag] = list(struct.unpack(e + fmt * n, raw[:total]))
    cols, rows = tags[256][0], tags[257][0]
    bps = tags.get(258, [1])
    spp = tags.get(277, [1])[0]
    fmt_code = tags.get(339, [1])[0]
    if tags.get(259, [1])[0] != 1:
        raise ValueError(f'{path}: compressed GeoTIFF is not supported; write it uncompressed')
    bits = bps[0]
    kind = {1: 'u', 2: 'i', 3: 'f'}[fmt_code]
    dtype = np.dtype(f'{e}{kind}{bits // 8}')
    planar = tags.get(284, [1])[0]
    out = np.zeros((spp, rows, cols), dtype=np.float64)
    if 324 in tags:  # tiles
        tw, th = tags[322][0], tags[323][0]
        offs, tiles_x = tags[324], (cols + tw - 1) // tw
        tiles_y = (rows + th - 1) // th
        per_plane = tiles_x * tiles_y
        for t, off in enumerate(offs):
            plane, rest = divmod(t, per_plane) if planar == 2 else (0, t)
            ty, tx = divmod(rest, tiles_x)
            ns = 1 if planar == 2 else spp
            tile = np.frombuffer(blob, dtype=dtype, count=tw * th * ns, offset=off).reshape(th, tw, ns)
            r0, c0 = ty * th, tx * tw
            r1, c1 = min(r0 + th, rows), min(c0 + tw, cols)
            if planar == 2:
                out[plane, r0:r1, c0:c1] = tile[:r1 - r0, :c1 - c0, 0]
            else:
                out[:, r0:r1, c0:c1] = np.moveaxis(tile[:r1 - r0, :c1 - c0, :], 2, 0)
    else:
        offs, rps = tags[273], tags.get(278, [rows])[0]
        strips_per_plane = (rows + rps - 1) // rps
        for s_idx, off in enumerate(offs):
            plane, strip = divmod(s_idx, strips_per_plane) if planar == 2 else (0, s_idx)
            r0 = strip * rps
            r1 = min(r0 + rps, rows)
            ns = 1 if planar == 2 else spp
            chunk = np.frombuffer(blob, dtype=dtype, count=(r1 - r0) * cols * ns, offset=off)
            chunk = chunk.reshape(r1 - r0, cols, ns)
            if planar == 2:
                out[plane, r0:r1] = chunk[:, :, 0]
            else:
                out[:, r0:r1] = np.moveaxis(chunk, 2, 0)
    if 34264 in tags:
        m = tags[34264]
        transform = (m[0], m[1], m[3], m[4], m[5], m[7])
    elif 33550 in tags and 33922 in tags:
        sx, sy = tags[33550][0], tags[33550][1]
        i, j, _, x, y, _ = tags[33922][:6]
        transform = (sx, 0.0, x - i * sx, 0.0, -sy, y + j * sy)
    else:
        raise ValueError(f'{path}: GeoTIFF has no georeference')
    epsg = None
    keys = tags.get(34735)
    if keys:
        for k in range(keys[3]):
            key, loc, _, value = keys[4 + 4 * k: 8 + 4 * k]
            if key in (3072, 2048) and loc == 0:
                epsg = value
    nodata = float(tags[42113]) if 42113 in tags and tags[42113].strip() else None
    return Raster(out, transform, epsg, nodata)
