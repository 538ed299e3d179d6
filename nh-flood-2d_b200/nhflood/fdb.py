"""Named-table column container standing in for fastdb4py ``.fdb`` files.

The reference stores meshes, frames, extrema and checkpoints as fastdb4py
record engines (pinned fastdb4py==0.2.4, a native third-party package that
is not installed here). Its schema is visible in src/nh_flood_2d/schema/
feature.py:1-68 and core/output.py:93-243; its byte layout is not. This
module keeps the same feature names, table names and column names and
dtypes, so readers and writers translate one to one, but the bytes are this
project's own format and are NOT readable by fastdb4py.

File layout: magic ``NHFDB001``, little-endian u64 header length, a UTF-8
JSON header ``{"tables": [{"name", "feature", "count", "columns": [[col,
dtype, offset]]}]}`` and then the column arrays, each 64-byte aligned.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

MAGIC = b'NHFDB001'

# Feature schemas (schema/feature.py:1-68): column -> numpy dtype.
FEATURES: dict[str, dict[str, str]] = {
    'IndexLike': {'index': '<u4'},
    'U8Value': {'value': 'u1'},
    'F32Value': {'value': '<f4'},
    'Ne': {'index': '<u4', 'x': '<f4', 'y': '<f4', 'z': '<f4', 'l_side_num': '<u4',
           'r_side_num': '<u4', 'b_side_num': '<u4', 't_side_num': '<u4', 'type': 'u1'},
    'SideTopoInfo': {'info': '<u4'},
    'Ns': {'index': '<u4', 'length': '<f4', 'x': '<f4', 'y': '<f4', 'z': '<f4', 'attr': 'u1'},
}


def _table_name(feature: str, name: str | None) -> str:
    return name if name else feature


def save(path, tables: list[tuple[str, str | None, dict[str, np.ndarray]]]) -> None:
    """Write ``tables`` = [(feature, name, {column: array})] atomically.

    Mirrors output.py:69-79: a sibling temporary file replaced in one step.
    """
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    header = {'tables': []}
    blobs = []
    offset = 0
    for feature, name, columns in tables:
        schema = FEATURES[feature]
        if set(columns) != set(schema):
            raise ValueError(f'{feature}: columns {sorted(columns)} differ from schema {sorted(schema)}')
        counts = {len(np.asarray(v).reshape(-1)) for v in columns.values()}
        if len(counts) != 1:
            raise ValueError(f'{feature}: column lengths differ')
        count = counts.pop()
        entry = {'name': _table_name(feature, name), 'feature': feature, 'count': count, 'columns': []}
        for column, dtype in schema.items():
            data = np.ascontiguousarray(np.asarray(columns[column]).reshape(-1), dtype=dtype)
            offset = (offset + 63) & ~63
            entry['columns'].append([column, dtype, offset])
            blobs.append((offset, data.tobytes()))
            offset += data.nbytes
        header['tables'].append(entry)
    head = json.dumps(header).encode('utf-8')
    start = len(MAGIC) + 8 + len(head)
    start = (start + 63) & ~63
    temporary = path.with_name(f'.{path.name}.{os.getpid()}.tmp')
    with open(temporary, 'wb') as f:
        f.write(MAGIC)
        f.write(np.uint64(len(head)).tobytes())
        f.write(head)
        f.write(b'\0' * (start - f.tell()))
        for off, blob in blobs:
            pad = start + off - f.tell()
            if pad:
                f.write(b'\0' * pad)
            f.write(blob)
    os.replace(temporary, path)


class Container:
    """Read access to a saved container; ``table(feature, name)`` returns a
    mapping of column name to a numpy array (a private copy)."""

    def __init__(self, path):
        self.path = Path(path)
        with open(self.path, 'rb') as f:
            magic = f.read(len(MAGIC))
            if magic != MAGIC:
                raise ValueError(f'{path}: not an nhflood table container')
            length = int(np.frombuffer(f.read(8), dtype='<u8')[0])
            self.header = json.loads(f.read(length).decode('utf-8'))
            self.start = (len(MAGIC) + 8 + length + 63) & ~63
        self._tables = {t['name']: t for t in self.header['tables']}

    def names(self):
        return list(self._tables)

    def table(self, feature: str, name: str | None = None) -> dict[str, np.ndarray]:
        key = _table_name(feature, name)
        if key not in self._tables:
            raise KeyError(f'{self.path}: no table {key}')
        entry = self._tables[key]
        if entry['feature'] != feature:
            raise ValueError(f'{self.path}: table {key} holds {entry["feature"]}, not {feature}')
        out = {}
        with open(self.path, 'rb') as f:
            for column, dtype, offset in entry['columns']:
                f.seek(self.start + offset)
                out[column] = np.fromfile(f, dtype=dtype, count=entry['count']).copy()
        return out


def load(path) -> Container:
    return Container(path)
