"""Run provenance (manifest.json) and the F64 water budget (mass_balance.csv).

The manifest keys and the mass_balance.csv columns and values are
nh-flood-2d's (core/run_record.py), so that tools reading a run's outputs
carry over. The budget's device terms come from this project's FP64
per-block partials instead of the reference's exact integer digits; how
they were reduced is stated under the manifest's ``budget_accumulator``.
"""
from __future__ import annotations

import csv
import hashlib
import json
import subprocess
import time
from dataclasses import dataclass
from datetime import datetime, timedelta, timezone
from pathlib import Path

import numpy as np

SOURCE_RULE = 'nhflood-b200/src-sha256/v1'
_SOURCE_SUFFIXES = ('.py', '.cu', '.cuh', '.h')
_REDUCTION = {
    'device_step_reduction': 'float64 pairwise tree of the F32 terms of each 256-cell block',
    'device_time_reduction': 'float64 TwoSum-compensated per-block partials',
    'host_reduction': 'Neumaier-compensated float64 merge across blocks at each output',
}


def sha256(path) -> str:
    digest = hashlib.sha256()
    with open(path, 'rb') as stream:
        while chunk := stream.read(1 << 20):
            digest.update(chunk)
    return digest.hexdigest()


def source_tree_sha256(root) -> str:
    """Hash of the package's Python, CUDA and header sources: for each file in
    sorted relative-path order its path, its length and its bytes."""
    root = Path(root)
    digest = hashlib.sha256(SOURCE_RULE.encode() + b'\0')
    sources = sorted((p.relative_to(root).as_posix(), p) for p in root.rglob('*')
                     if p.is_file() and p.suffix in _SOURCE_SUFFIXES)
    for relative, path in sources:
        content = path.read_bytes()
        digest.update(relative.encode() + b'\0' + len(content).to_bytes(8, 'big'))
        digest.update(content)
    return digest.hexdigest()


def _git_state(repo: Path):
    """(commit, dirty) of the checkout the package runs from, or (None, None)."""
    if not (repo / '.git').exists():
        return None, None
    try:
        commit = subprocess.check_output(['git', 'rev-parse', 'HEAD'], cwd=repo, text=True).strip()
        status = subprocess.check_output(['git', 'status', '--porcelain'], cwd=repo, text=True)
    except (OSError, subprocess.CalledProcessError):
        return None, None
    return commit, bool(status.strip())


def _refuse_reused(domain_dir: Path) -> None:
    """A run never writes into a directory that holds another run's outputs."""
    output = domain_dir / 'output'
    used = ((domain_dir / 'manifest.json').exists() or (domain_dir / 'mass_balance.csv').exists()
            or (output.exists() and any(output.iterdir())))
    if used:
        raise FileExistsError(f'Use a new output directory: {domain_dir}')


class RunRecord:
    """manifest.json of one run: provenance, configuration, input hashes and,
    at the end, the status. Used as a context manager; an exception leaves
    status "failed" and its message under "error"."""

    def __init__(self, domain, force, pipe=None):
        package = Path(__file__).resolve().parents[1]
        domain_dir = Path(domain.domain_dir)
        _refuse_reused(domain_dir)
        self.path = domain_dir / 'manifest.json'
        self.clock = time.perf_counter()
        commit, dirty = _git_state(package.parent)
        start = domain.start
        self.data = dict(
            source_sha256=source_tree_sha256(package), source_hash_rule=SOURCE_RULE,
            git_commit=commit, git_dirty=dirty,
            config=dict(domain=domain.model_dump(mode='json'), force=force.model_dump(mode='json'),
                        pipe=pipe.model_dump(mode='json') if pipe else None),
            input_sha256={},
            simulation_start=start.isoformat(),
            warmup_start=(start - timedelta(seconds=domain.warmup_duration)).isoformat(),
            simulation_end=(start + timedelta(seconds=domain.duration)).isoformat(),
            started_at=_now(),
            steps=0, warmup_steps=0, backend=None, device_name=None,
            peak_device_memory_bytes='unavailable', status='running',
            budget_accumulator=dict(_REDUCTION))
        self.write()

    def __enter__(self):
        return self

    def __exit__(self, error_type, error, traceback):
        if error is not None:
            self.data['error'] = str(error)
        self.finish('completed' if error_type is None else 'failed')

    def hash_inputs(self, domain, force, pipe=None):
        inputs = [domain.ne, domain.ns, *force.input_paths()] + ([domain.restart_state] if domain.restart_state else [])
        self.data['input_sha256'].update({str(Path(p).resolve()): sha256(p) for p in inputs})
        self.write()

    def device(self, backend: str, name: str, peak_bytes=None):
        self.data.update(backend=backend, device_name=name)
        if peak_bytes is not None:
            self.data['peak_device_memory_bytes'] = int(peak_bytes)

    def write(self):
        self.path.write_text(json.dumps(self.data, indent=2) + '\n')

    def finish(self, status):
        self.data.update(status=status, finished_at=_now(), wall_seconds=time.perf_counter() - self.clock)
        self.write()


def _now() -> str:
    return datetime.now(timezone.utc).isoformat()


def finite_totals(totals):
    """An infinite or NaN F32 term in any step poisons the interval's totals;
    the run stops with the reference's error (device_budget.py:71-73)."""
    totals = np.asarray(totals)
    if not np.isfinite(totals).all():
        raise FloatingPointError('Nonfinite F32 device budget diagnostic')
    return totals


# ------------------------------------------------------------ water budget

@dataclass
class BudgetTerms:
    """Named views of the device's cumulative term vector [4 + 6 B]: 0
    infiltration, 1 bed clamp off level cells, 2 bed clamp on level cells,
    3 pipe exchange, then five components per boundary (level cells), then
    one applied discharge per boundary."""
    values: np.ndarray
    boundaries: int

    @property
    def level_exchange(self) -> np.ndarray:
        """Per boundary, the sum of its five level components."""
        b = self.boundaries
        return self.values[4:4 + 5 * b].reshape(b, 5).sum(axis=1, dtype=np.float64)

    @property
    def discharge(self) -> np.ndarray:
        return self.values[4 + 5 * self.boundaries:]


def balance(rain, initial, storage, terms: BudgetTerms):
    """(residual, scale) of one mass_balance.csv row: storage minus the
    initial storage and every source and sink (rain, infiltration, bed
    clamps, pipe, applied discharge, level exchange); scale is the largest
    of the initial storage, the total inflow and the total exchanged volume."""
    v = terms.values
    levels, discharge = terms.level_exchange, terms.discharge
    inputs = rain - v[0] + v[1] + v[3]
    inputs += discharge.sum(dtype=np.float64) + levels.sum(dtype=np.float64)
    residual = float(storage - initial - inputs)
    inflow = rain + np.maximum(discharge, 0).sum() + np.maximum(levels, 0).sum() + max(v[3], 0.)
    exchanged = np.abs(discharge).sum() + np.abs(v[[0, 1, 3]]).sum() + np.abs(levels).sum()
    return residual, max(initial, float(inflow), float(exchanged))


def budget_columns(boundaries) -> list[str]:
    return (['time', 'elapsed_seconds', 'phase', 'rainfall_m3', 'infiltration_m3']
            + [f'{b.kind}:{b.name}_m3' for b in boundaries]
            + [f'requested_discharge:{b.name}_m3' for b in boundaries if b.kind == 'discharge']
            + ['bed_clamp_nonlevel_m3', 'bed_clamp_level_m3', 'gate_bed_m3', 'pipe_exchange_m3',
               'initial_storage_m3', 'storage_m3', 'residual_m3', 'relative_residual'])


class WaterBudget:
    """mass_balance.csv: the host's F64 forcing totals (rain volume and
    requested discharge, integrated step by step) beside the device's terms,
    one row per output."""

    def __init__(self, path, boundaries, initial_storage):
        self.boundaries = list(boundaries)
        self.initial = float(initial_storage)
        self.rain = np.float64(0)
        self.discharge = np.zeros(len(self.boundaries), dtype=np.float64)
        self.device_terms = np.zeros(4 + 6 * len(self.boundaries), dtype=np.float64)
        self._is_discharge = np.array([b.kind == 'discharge' for b in self.boundaries], dtype=bool)
        self.file = open(path, 'w', newline='')
        self.writer = csv.DictWriter(self.file, budget_columns(self.boundaries))
        self.writer.writeheader()
        self.last_row = None

    def add_forcing(self, dt, rain_rate_volume, boundary_values):
        step = np.float64(dt)
        self.rain += step * rain_rate_volume
        for i in np.flatnonzero(self._is_discharge):
            self.discharge[i] += step * boundary_values[i]

    def set_device_terms(self, cumulative_terms):
        self.device_terms = cumulative_terms

    def output(self, date, seconds, storage, phase):
        terms = BudgetTerms(self.device_terms, len(self.boundaries))
        residual, scale = balance(self.rain, self.initial, storage, terms)
        v = terms.values
        row = dict(time=date.isoformat(), elapsed_seconds=seconds, phase=phase,
                   rainfall_m3=float(self.rain), infiltration_m3=float(v[0]),
                   bed_clamp_nonlevel_m3=float(v[1]), bed_clamp_level_m3=float(v[2]), gate_bed_m3=0.,
                   pipe_exchange_m3=float(v[3]), initial_storage_m3=self.initial,
                   storage_m3=float(storage), residual_m3=residual,
                   relative_residual=residual / scale if scale else None)
        levels, discharge = terms.level_exchange, terms.discharge
        for i, b in enumerate(self.boundaries):
            if self._is_discharge[i]:
                row[f'{b.kind}:{b.name}_m3'] = float(discharge[i])
                row[f'requested_discharge:{b.name}_m3'] = float(self.discharge[i])
            else:
                row[f'{b.kind}:{b.name}_m3'] = float(levels[i])
        self.writer.writerow(row)
        self.file.flush()
        self.last_row = row
        return row

    def close(self):
        self.file.close()
