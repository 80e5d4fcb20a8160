"""Run configuration for the oracle (test infrastructure only).

Mirrors the fields of the reference's pydantic ``Parameters`` model that
the time-step path reads (``src/dnsjax/parameters.py:26-133``) plus the
derived values (``parameters.py:148-211``: ``ly``, tilt flags) and the 3/2
padded sizes (``parameters.py:214-257``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import pi

PERIODIC = ("kolmogorov", "waleffe", "decaying-box")
MONOCHROMATIC = ("kolmogorov", "waleffe")
WALLED = ("plane-couette",)


@dataclass
class Config:
    system: str = "kolmogorov"
    nx: int = 32
    ny: int = 32
    nz: int = 32
    lx: float = 4.0
    lz: float = 4.0
    # ``derived_params.ly``: 4 for periodic, 2 for walled
    # (parameters.py:186-193); a caller may override it afterwards.
    ly: float | None = None
    re: float = 1000.0
    dt: float = 0.01
    implicitness: float = 0.5
    corrector_tolerance: float = 1e-5
    max_corrector_iterations: int = 10
    fd_order: int = 4
    tilt_degree: float = 0.0
    oversampling_factor: int = 3
    oversample_y: bool = True
    correct_divergence: bool = True
    extra: dict = field(default_factory=dict)

    def __post_init__(self) -> None:
        if self.ly is None:
            self.ly = 4.0 if self.system in PERIODIC else 2.0

    @property
    def periodic(self) -> bool:
        return self.system in PERIODIC

    # parameters.py:203-211 (tilt flags)
    @property
    def tilt_rad(self) -> float:
        return pi * self.tilt_degree / 180

    @property
    def tilt(self) -> bool:
        t = self.tilt_degree
        return not (abs(t) == 0 or abs(t - 180) == 0)

    @property
    def tilt_90(self) -> bool:
        t = self.tilt_degree
        return abs(t + 90) == 0 or abs(t - 90) == 0

    # parameters.py:241-257 (PaddedResolution)
    @property
    def nx_padded(self) -> int:
        return self.oversampling_factor * self.nx // 2

    @property
    def nz_padded(self) -> int:
        return self.oversampling_factor * self.nz // 2

    @property
    def ny_padded(self) -> int:
        if not self.periodic:
            return self.ny
        if self.oversample_y:
            return self.oversampling_factor * self.ny // 2
        return self.ny

    # sharding.py:138-185 (spectral / physical shapes)
    @property
    def spec_shape(self) -> tuple[int, int, int]:
        if self.periodic:
            return (self.ny - 1, self.nz - 1, self.nx // 2)
        return (self.nz - 1, self.nx // 2, self.ny)

    @property
    def phys_shape(self) -> tuple[int, int, int]:
        return (self.ny_padded, self.nz_padded, self.nx_padded)
