"""TOML case configuration (the reference's schema, src/config.py:8-128).

Frozen dataclasses, strict key and type checks as in the reference
(``_load_dataclass``/``_validate_config``); every field the reference has is
kept with its meaning.  Optional extensions (default ``None`` reproduces the
reference): ``case.lattice``, ``case.instances``, ``case.seed``,
``numerics.dim``, ``physics.alpha_min``, ``physics.alpha_max``,
``solver.max_steps``, ``execution.precision``; ``execution.backend`` also
accepts ``"b200"``.  Reference TOML files load unchanged.
"""

from __future__ import annotations

import tomllib
from dataclasses import dataclass, fields, is_dataclass
from pathlib import Path
from types import NoneType
from typing import get_args, get_type_hints


@dataclass(frozen=True)
class CaseConfig:
    name: str
    nx: int
    lattice: str | None = None  # "close_packed" (reference), "square" (2-D), "cubic" (3-D)
    instances: int | None = None  # batched form: independent instances
    seed: int | None = None


@dataclass(frozen=True)
class PhysicsConfig:
    gamma: float
    mu0: float
    artificial_viscosity: float
    artificial_thermal_conductivity: float
    artificial_magnetic_dissipation: float
    alpha_min: float | None = None
    alpha_max: float | None = None


@dataclass(frozen=True)
class NumericsConfig:
    kernel: str
    hfact: float
    density: str
    periodic_mode: str | None
    cleaning_speed_factor: float
    cleaning_damping_factor: float
    dim: int | None = None


@dataclass(frozen=True)
class SolverConfig:
    tf: float
    pfreq: int
    adaptive_timestep: bool
    timestep_factor: float
    max_steps: int | None = None


@dataclass(frozen=True)
class ExecutionConfig:
    backend: str
    fused: bool
    directory: str
    precision: str | None = None


@dataclass(frozen=True)
class SimulationConfig:
    case: CaseConfig
    physics: PhysicsConfig
    numerics: NumericsConfig
    solver: SolverConfig
    execution: ExecutionConfig

    def validate(self):
        _validate_config(self)


def load_config(path, config_types):
    with Path(path).open("rb") as stream:
        values = tomllib.load(stream)
    config = _load_dataclass(config_types[values["case"]["name"]], values)
    config.validate()
    return config


def _load_dataclass(config_type, values):
    hints = get_type_hints(config_type)
    config_fields = {f.name: hints[f.name] for f in fields(config_type)}
    optional = {name for name, t in config_fields.items() if NoneType in get_args(t)}
    if not set(values) <= set(config_fields):
        raise ValueError(f"unknown keys {sorted(set(values) - set(config_fields))} for {config_type.__name__}")
    if not set(config_fields) - optional <= set(values):
        raise ValueError(f"missing keys {sorted(set(config_fields) - optional - set(values))} for "
                         f"{config_type.__name__}")
    args = {name: _load_dataclass(t, values[name]) if is_dataclass(t) else values[name]
            for name, t in config_fields.items() if name in values}
    args.update({name: None for name in optional if name not in values})
    return config_type(**args)


def _check(cond, msg):
    if not cond:
        raise ValueError(msg)


def _validate_config(c):
    _check(type(c.case.name) is str and c.case.name, "case.name")
    _check(type(c.case.nx) is int and c.case.nx > 0, "case.nx")
    _check(c.case.lattice in (None, "close_packed", "square", "cubic"), "case.lattice")
    _check(c.case.instances is None or (type(c.case.instances) is int and c.case.instances > 0), "case.instances")
    _check(type(c.physics.gamma) is float and c.physics.gamma > 1.0, "physics.gamma")
    _check(type(c.physics.mu0) is float and c.physics.mu0 > 0.0, "physics.mu0")
    for k in ("artificial_viscosity", "artificial_thermal_conductivity", "artificial_magnetic_dissipation"):
        v = getattr(c.physics, k)
        _check(type(v) is float and v >= 0.0, f"physics.{k}")
    for k in ("alpha_min", "alpha_max"):
        v = getattr(c.physics, k)
        _check(v is None or (type(v) is float and 0.0 <= v <= 1.0), f"physics.{k}")
    _check(c.numerics.kernel in {"cubic", "quintic", "wendland_c2", "wendland_c4", "wendland_c6", "gaussian",
                                 "super_gaussian"}, "numerics.kernel")
    _check(type(c.numerics.hfact) is float and c.numerics.hfact > 0.0, "numerics.hfact")
    _check(c.numerics.density in {"iterate", "single"}, "numerics.density")
    _check(c.numerics.periodic_mode in {None, "ghost", "minimum_image"}, "numerics.periodic_mode")
    _check(c.numerics.dim in (None, 2, 3), "numerics.dim")
    for k in ("cleaning_speed_factor", "cleaning_damping_factor"):
        v = getattr(c.numerics, k)
        _check(type(v) is float and v >= 0.0, f"numerics.{k}")
    _check(type(c.solver.tf) is float and c.solver.tf > 0.0, "solver.tf")
    _check(type(c.solver.pfreq) is int and c.solver.pfreq > 0, "solver.pfreq")
    _check(type(c.solver.adaptive_timestep) is bool, "solver.adaptive_timestep")
    _check(type(c.solver.timestep_factor) is float and c.solver.timestep_factor > 0.0, "solver.timestep_factor")
    _check(c.solver.max_steps is None or (type(c.solver.max_steps) is int and c.solver.max_steps > 0),
           "solver.max_steps")
    _check(c.execution.backend in {"cython", "cuda", "opencl", "b200"}, "execution.backend")
    _check(type(c.execution.fused) is bool, "execution.fused")
    _check(type(c.execution.directory) is str and c.execution.directory, "execution.directory")
    _check(c.execution.precision in (None, "fp64", "fp32"), "execution.precision")


def pysph_arguments(execution):
    """Arguments the reference passed to PySPH; kept for callers that log them."""
    backend = {"cython": (), "cuda": ("--cuda",), "opencl": ("--opencl",), "b200": ("--b200",)}[execution.backend]
    return [*backend, *(("--fused",) if execution.fused else ()), "-d", execution.directory]
