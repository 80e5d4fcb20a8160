"""Simulation parameters, mirroring the reference's pydantic models.

Same sections, field names, defaults and validation as
``src/dnsjax/parameters.py:26-133`` (``dist``, ``phys``, ``geo``, ``res``,
``init``, ``outs``, ``step``, ``stop``, ``debug``, ``solver``), with two
differences: ``solver.backend`` accepts ``"cuda"``, which selects this
package's kernels (and is this package's default), and ``dist.platform``
defaults to ``"cuda"`` (the reference's default is ``"cpu"``).  ``update_parameters``
applies only explicitly-set fields and recomputes the derived values as the
reference does (``parameters.py:173-211``), including the reset of ``ly`` to
4 (periodic) or 2 (walled); a caller that needs another ``ly`` (e.g. a
2*pi box) sets ``derived_params.ly`` after calling it.
"""

from __future__ import annotations

import tomllib
from dataclasses import dataclass
from datetime import timedelta
from math import pi
from pathlib import Path
from typing import Literal

from pydantic import BaseModel, Field

monochromatic_systems: list[str] = ["kolmogorov", "waleffe"]
periodic_systems: list[str] = ["decaying-box", *monochromatic_systems]
cartesian_systems: list[str] = ["plane-couette"]
walled_systems: list[str] = [*cartesian_systems]


class Distribution(BaseModel):
    np: int = Field(ge=1, default=1)
    platform: Literal["cpu", "cuda", "rocm", "tpu"] = "cuda"


class Physics(BaseModel):
    re: float = Field(gt=0, default=1000)
    system: Literal[
        "decaying-box", "kolmogorov", "waleffe", "plane-couette"
    ] = "kolmogorov"
    oversampling_factor: int = Field(ge=2, default=3)
    oversample_y: bool = True


class Geometry(BaseModel):
    lx: float = Field(gt=0, default=4.0)
    lz: float = Field(gt=0, default=4.0)
    tilt_degree: float = Field(gt=-180, le=180, default=0)


class Resolution(BaseModel):
    nx: int = Field(ge=1, default=128)
    ny: int = Field(ge=1, default=128)
    nz: int = Field(ge=1, default=128)
    fd_order: int = Field(ge=2, default=4)
    double_precision: bool = True


class Initiation(BaseModel):
    start_from_laminar: bool = True
    snapshot: Path | None = None
    t0: float = 0
    it0: int = 0


class Outputs(BaseModel):
    it_stats: int | None = None


class TimeStepping(BaseModel):
    dt: float = Field(gt=0, default=0.01)
    implicitness: float = Field(ge=0, le=1, default=0.5)
    corrector_tolerance: float = Field(gt=0, default=1e-5)
    max_corrector_iterations: int = Field(ge=1, default=10)


class Termination(BaseModel):
    max_sim_time: float | None = None
    max_wall_time: timedelta | None = None


class Debugging(BaseModel):
    time_functions: bool = True
    measure_corrections: bool = False
    correct_divergence: bool = True


class Solver(BaseModel):
    # "cuda": this package's sm_100a kernels.  "banded" / "dense" are the
    # reference's JAX backends and are not implemented here.
    backend: Literal["banded", "dense", "cuda"] = "cuda"


class Parameters(BaseModel):
    dist: Distribution | None = Distribution()
    phys: Physics = Physics()
    geo: Geometry = Geometry()
    res: Resolution = Resolution()
    init: Initiation = Initiation()
    outs: Outputs = Outputs()
    step: TimeStepping = TimeStepping()
    stop: Termination | None = Termination()
    debug: Debugging | None = Debugging()
    solver: Solver = Solver()


@dataclass
class DerivedParameters:
    ly: float = 2
    tilt_rad: float = 0
    tilt: bool = False
    tilt_90: bool = False


params: Parameters = Parameters()
derived_params: DerivedParameters = DerivedParameters()


def read_parameters(path: Path) -> Parameters:
    with open(path, "rb") as f:
        return Parameters(**tomllib.load(f))


def derive(p: Parameters, d: DerivedParameters | None = None) -> DerivedParameters:
    """Derived values for ``p`` (reference parameters.py:186-211)."""
    d = DerivedParameters() if d is None else d
    if p.phys.system in periodic_systems:
        d.ly = 4
    elif p.phys.system in cartesian_systems:
        d.ly = 2
    else:
        raise NotImplementedError(p.phys.system)
    t = p.geo.tilt_degree
    d.tilt_rad = pi * t / 180
    if abs(t) == 0 or abs(t - 180) == 0:
        d.tilt, d.tilt_90 = False, False
    elif abs(t + 90) == 0 or abs(t - 90) == 0:
        d.tilt, d.tilt_90 = True, True
    else:
        d.tilt, d.tilt_90 = True, False
    return d


def update_parameters(params_new: Parameters) -> None:
    """Merge explicitly-set fields of ``params_new`` into ``params``."""
    for category, values in params_new.model_dump(exclude_unset=True).items():
        if values is not None:
            for key, value in values.items():
                if value is not None:
                    setattr(getattr(params, category), key, value)
    derive(params, derived_params)


def padded_sizes(p: Parameters) -> tuple[int, int, int]:
    """``(nx_padded, ny_padded, nz_padded)`` (reference parameters.py:214-257).

    For walled flows y is not oversampled and ``ny_padded`` is ``ny``.
    """
    f = p.phys.oversampling_factor
    nxp = f * p.res.nx // 2
    nzp = f * p.res.nz // 2
    if p.phys.system in periodic_systems:
        nyp = f * p.res.ny // 2 if p.phys.oversample_y else p.res.ny
    else:
        nyp = p.res.ny
    return nxp, nyp, nzp


def make_parameters(**sections) -> Parameters:
    """``make_parameters(phys={...}, res={...}, ...)`` convenience builder."""
    return Parameters(**sections)
