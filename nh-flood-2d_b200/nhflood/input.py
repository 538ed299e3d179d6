"""Validated domain and forcing configuration (same JSON as the reference).

Field names, defaults and validation rules follow the reference's pydantic
models (nh-flood-2d src/nh_flood_2d/input/domain.py:1-135 and
input/force.py:1-76), so an existing ``domain.json``/``force.json`` loads
unchanged.
"""
from __future__ import annotations

from datetime import datetime
from pathlib import Path
from typing import Annotated, Literal

from pydantic import AwareDatetime, BaseModel, ConfigDict, Field, field_validator, model_validator


def absolute_time(value: str) -> datetime:
    """Parse an ISO 8601 timestamp that must carry a timezone (input/force.py:7-12)."""
    result = datetime.fromisoformat(value.replace('Z', '+00:00'))
    if result.tzinfo is None or result.utcoffset() is None:
        raise ValueError(f'Timestamp must include a timezone: {value}')
    return result


class InputModel(BaseModel):
    model_config = ConfigDict(extra='forbid', allow_inf_nan=False)


class BoundaryConfig(InputModel):
    name: str = Field(min_length=1)
    kind: Literal['level', 'discharge']
    line: str
    series: str


class RainfallConfig(InputModel):
    raster: str
    intervals: str


class GatePointConfig(InputModel):
    name: str = Field(min_length=1)
    inside_point: tuple[float, float]
    control_point: tuple[float, float]


class GateConfig(InputModel):
    """The gate controller block (input/force.py:38-56); resolved by
    nhflood.gate.GateLayout, run on the device when enabled."""
    land_type: int = Field(ge=0, le=255)
    pond_land_type: int = Field(ge=0, le=255)
    enabled: bool
    trigger_level: float
    opening_seconds: float = Field(gt=0)
    open_elevation: float
    gates: list[GatePointConfig] = Field(min_length=1)

    @model_validator(mode='after')
    def unique_gates(self):
        if self.pond_land_type == self.land_type:
            raise ValueError('pond_land_type must differ from gate land_type')
        names = [gate.name for gate in self.gates]
        if len(names) != len(set(names)):
            raise ValueError('Gate names must be unique')
        return self


class ForceConfig(InputModel):
    boundaries: list[BoundaryConfig]
    rainfall: RainfallConfig
    gate: GateConfig | None = None

    @model_validator(mode='after')
    def validate_names(self):
        names = [b.name for b in self.boundaries]
        if len(set(names)) != len(names):
            raise ValueError('Boundary names must be unique')
        return self

    def input_paths(self) -> list[str]:
        return [p for b in self.boundaries for p in (b.line, b.series)] + [
            self.rainfall.raster, self.rainfall.intervals]


class HortonInfiltration(InputModel):
    f0_mm_h: float = Field(ge=0)
    fc_mm_h: float = Field(ge=0)
    k_per_h: float = Field(ge=0)

    @model_validator(mode='after')
    def validate_capacity(self):
        if self.f0_mm_h < self.fc_mm_h:
            raise ValueError('f0_mm_h must be at least fc_mm_h')
        return self


class LandParameters(InputModel):
    manning_n: float = Field(ge=0)
    infiltration: Literal['none'] | HortonInfiltration


class DomainConfig(InputModel):
    ne: str
    ns: str
    epsg_code: int
    domain_dir: str
    afa: float = Field(default=0.5, gt=0, le=1)
    sita: float = Field(default=1.0, ge=0, le=1)
    min_h: float = Field(default=0.02, gt=0)
    start: AwareDatetime = Field(strict=True)
    duration: int = Field(gt=0)
    warmup_duration: int = Field(ge=0)
    land_parameters: dict[Annotated[int, Field(ge=0, le=255)], LandParameters] = Field(min_length=1)
    yield_step: int = Field(default=300, gt=0)
    restart_state: str = ''
    stations: dict[str, tuple[float, float]] = {}
    observation_dir: str = ''

    @property
    def _domain_path(self) -> Path:
        return Path(self.domain_dir)

    @property
    def _preprocessed_path(self) -> Path:
        path = self._domain_path / 'preprocessed'
        path.mkdir(parents=True, exist_ok=True)
        return path

    @property
    def tmp_ne(self) -> str:
        return str(self._domain_path / 'temp_ne.txt')

    @property
    def tmp_ns(self) -> str:
        return str(self._domain_path / 'temp_ns.txt')

    @property
    def ne_fdb(self) -> str:
        return str(self._preprocessed_path / 'ne.fdb')

    @property
    def ns_fdb(self) -> str:
        return str(self._preprocessed_path / 'ns.fdb')

    @property
    def boundary_fdb(self) -> str:
        return str(self._preprocessed_path / 'boundary.fdb')

    @property
    def output_dir(self) -> str:
        path = self._domain_path / 'output'
        path.mkdir(parents=True, exist_ok=True)
        return str(path)

    @property
    def frame_dir(self) -> str:
        path = Path(self.output_dir) / 'frames'
        path.mkdir(exist_ok=True)
        return str(path)

    @model_validator(mode='after')
    def validate_clock_range(self):
        if self.duration + self.warmup_duration >= 2 ** 24:
            raise ValueError('Duration plus warmup must fit the two-U32 clock (less than 2**24 seconds)')
        return self

    @field_validator('ne', 'ns')
    @classmethod
    def validate_paths(cls, v):
        if not Path(v).exists():
            raise ValueError(f'Path does not exist: {v}')
        return v

    @field_validator('domain_dir')
    @classmethod
    def validate_domain_dir(cls, v):
        Path(v).mkdir(parents=True, exist_ok=True)
        return v


def load_domain_config(config_path: str) -> DomainConfig:
    return DomainConfig.model_validate_json(Path(config_path).read_text())


def load_force_config(config_path: str) -> ForceConfig:
    return ForceConfig.model_validate_json(Path(config_path).read_text())
