"""Run manifest and F64 water budget (same files and columns as the
reference's core/run_record.py:1-161)."""
from __future__ import annotations

import csv
import hashlib
import json
import os
import subprocess
import time
from datetime import datetime, timedelta, timezone
from pathlib import Path

import numpy as np

SOURCE_RULE = 'nhflood-b200/src-sha256/v1'


def sha256(path) -> str:
    digest = hashlib.sha256()
    with open(path, 'rb') as file:
        for block in iter(lambda: file.read(1 << 20), b''):
            digest.update(block)
    return digest.hexdigest()


def source_tree_sha256(root) -> str:
    """Hash of sorted relative paths, lengths and bytes of the package's
    Python, CUDA and header sources."""
    root = Path(root)
    digest = hashlib.sha256(SOURCE_RULE.encode() + b'\0')
    files = [p for p in root.rglob('*') if p.suffix in ('.py', '.cu', '.cuh', '.h') and p.is_file()]
    for path in sorted(files, key=lambda p: p.relative_to(root).as_posix()):
        content = path.read_bytes()
        digest.update(path.relative_to(root).as_posix().encode() + b'\0')
        digest.update(len(content).to_bytes(8, 'big'))
        digest.update(content)
    return digest.hexdigest()


class RunRecord:
    """manifest.json provenance; refuses to reuse an output directory."""

    def __init__(self, domain, force, pipe=None):
        package = Path(__file__).resolve().parents[1]
        self.path = Path(domain.domain_dir) / 'manifest.json'
        output = Path(domain.domain_dir) / 'output'
        if (self.path.exists() or (self.path.parent / 'mass_balance.csv').exists()
                or (output.exists() and any(output.iterdir()))):
            raise FileExistsError(f'Use a new output directory: {domain.domain_dir}')
        self.clock = time.perf_counter()
        repo = package.parent
        commit = dirty = None
        if (repo / '.git').exists():
            try:
                commit = subprocess.check_output(['git', 'rev-parse', 'HEAD'], cwd=repo, text=True).strip()
                dirty = bool(subprocess.check_output(['git', 'status', '--porcelain'], cwd=repo, text=True).strip())
            except (OSError, subprocess.CalledProcessError):
                pass
        self.data = {
            'source_sha256': source_tree_sha256(package),
            'source_hash_rule': SOURCE_RULE,
            'git_commit': commit,
            'git_dirty': dirty,
            'config': {'domain': domain.model_dump(mode='json'), 'force': force.model_dump(mode='json'),
                       'pipe': pipe.model_dump(mode='json') if pipe else None},
            'input_sha256': {},
            'simulation_start': domain.start.isoformat(),
            'warmup_start': (domain.start - timedelta(seconds=domain.warmup_duration)).isoformat(),
            'simulation_end': (domain.start + timedelta(seconds=domain.duration)).isoformat(),
            'started_at': datetime.now(timezone.utc).isoformat(),
            'steps': 0, 'warmup_steps': 0, 'backend': None, 'device_name': None,
            'peak_device_memory_bytes': 'unavailable', 'status': 'running',
            'budget_accumulator': {
                'device_step_reduction': 'float64 pairwise tree of the F32 terms of each 256-cell block',
                'device_time_reduction': 'float64 TwoSum-compensated per-block partials',
                'host_reduction': 'Neumaier-compensated float64 merge across blocks at each output',
            },
        }
        self.write()

    def __enter__(self):
        return self

    def __exit__(self, error_type, error, traceback):
        if error is not None:
            self.data['error'] = str(error)
        self.finish('failed' if error_type else 'completed')

    def hash_inputs(self, domain, force, pipe=None):
        paths = [domain.ne, domain.ns, *force.input_paths()]
        if domain.restart_state:
            paths.append(domain.restart_state)
        for path in paths:
            self.data['input_sha256'][str(Path(path).resolve())] = sha256(path)
        self.write()

    def device(self, backend: str, name: str, peak_bytes=None):
        self.data['backend'] = backend
        self.data['device_name'] = name
        if peak_bytes is not None:
            self.data['peak_device_memory_bytes'] = int(peak_bytes)

    def write(self):
        self.path.write_text(json.dumps(self.data, indent=2) + '\n')

    def finish(self, status):
        self.data.update(status=status, finished_at=datetime.now(timezone.utc).isoformat(),
                         wall_seconds=time.perf_counter() - self.clock)
        self.write()


def finite_totals(totals):
    """DeviceBudget.flush's check (device_budget.py:71-73): an infinite or NaN
    F32 term in any step poisons the interval's FP64 totals, and the run
    stops with the reference's error."""
    totals = np.asarray(totals)
    if not np.all(np.isfinite(totals)):
        raise FloatingPointError('Nonfinite F32 device budget diagnostic')
    return totals


class WaterBudget:
    """mass_balance.csv rows from device terms and host F64 forcing totals."""

    def __init__(self, path, boundaries, initial_storage):
        self.boundaries = boundaries
        self.initial = float(initial_storage)
        self.rain = np.float64(0)
        self.discharge = np.zeros(len(boundaries), dtype=np.float64)
        self.device_terms = np.zeros(4 + 6 * len(boundaries), dtype=np.float64)
        self.file = open(path, 'w', newline='')
        fields = ['time', 'elapsed_seconds', 'phase', 'rainfall_m3', 'infiltration_m3']
        fields += [f'{b.kind}:{b.name}_m3' for b in boundaries]
        fields += [f'requested_discharge:{b.name}_m3' for b in boundaries if b.kind == 'discharge']
        fields += ['bed_clamp_nonlevel_m3', 'bed_clamp_level_m3', 'gate_bed_m3', 'pipe_exchange_m3',
                   'initial_storage_m3', 'storage_m3', 'residual_m3', 'relative_residual']
        self.writer = csv.DictWriter(self.file, fields)
        self.writer.writeheader()
        self.last_row = None

    def add_forcing(self, dt, rain_rate_volume, boundary_values):
        self.rain += np.float64(dt) * rain_rate_volume
        for i, b in enumerate(self.boundaries):
            if b.kind == 'discharge':
                self.discharge[i] += np.float64(dt) * boundary_values[i]

    def set_device_terms(self, cumulative_terms):
        self.device_terms = cumulative_terms

    def output(self, date, seconds, storage, phase):
        terms = self.device_terms
        nb = len(self.boundaries)
        levels = terms[4:4 + 5 * nb].reshape(nb, 5).sum(axis=1, dtype=np.float64)
        floor, level_floor, pipe = terms[1], terms[2], terms[3]
        actual_discharge = terms[4 + 5 * nb:]
        inputs = self.rain - terms[0] + floor + pipe
        inputs += actual_discharge.sum(dtype=np.float64) + levels.sum(dtype=np.float64)
        residual = float(storage - self.initial - inputs)
        total_in = self.rain + np.maximum(actual_discharge, 0).sum() + np.maximum(levels, 0).sum() + max(pipe, 0.)
        scale = max(self.initial, float(total_in),
                    float(np.abs(actual_discharge).sum() + np.abs(terms[[0, 1, 3]]).sum() + np.abs(levels).sum()))
        row = dict(time=date.isoformat(), elapsed_seconds=seconds, phase=phase,
                   rainfall_m3=float(self.rain), infiltration_m3=float(terms[0]),
                   bed_clamp_nonlevel_m3=float(floor), bed_clamp_level_m3=float(level_floor), gate_bed_m3=0.,
                   pipe_exchange_m3=float(pipe), initial_storage_m3=self.initial,
                   storage_m3=float(storage), residual_m3=residual,
                   relative_residual=residual / scale if scale else None)
        for i, b in enumerate(self.boundaries):
            row[f'{b.kind}:{b.name}_m3'] = float(actual_discharge[i] if b.kind == 'discharge' else levels[i])
            if b.kind == 'discharge':
                row[f'requested_discharge:{b.name}_m3'] = float(self.discharge[i])
        self.writer.writerow(row)
        self.file.flush()
        self.last_row = row
        return row

    def close(self):
        self.file.close()
