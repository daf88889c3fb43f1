"""Grid geometry and the Courant time step.

Mirrors the input type of the reference solver (ac-fdtd ``src/ac_fdtd/grid.py:37-163``) so a
caller can build a grid here or pass the reference's own ``Grid``: the CUDA solver reads only
``dx``, ``nx``, ``ny`` and ``nz`` from it.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = ["Grid", "max_stable_time_step", "cell_index"]

#: A coordinate this close (in cells) below a cell boundary is snapped up to it, so that e.g.
#: 1.2 / 0.01 = 119.99999999999999 lands in cell 120 (ac-fdtd ``src/ac_fdtd/grid.py:31``).
INDEX_TOLERANCE = 1e-6


def max_stable_time_step(dx: float, sound_speed: float) -> float:
    """Largest stable step of the 3D staggered leapfrog, ``c dt sqrt(3) / dx = 1``.

    ac-fdtd ``src/ac_fdtd/grid.py:37-45``.
    """
    return dx / (sound_speed * math.sqrt(3))


def cell_index(dx: float, shape, point) -> tuple[int, int, int]:
    """Cell containing ``point`` (metres), clipped into the grid.

    ac-fdtd ``src/ac_fdtd/grid.py:131-147``: floor(x/dx + 1e-6), then clipped to [0, n-1], so a
    point on the far wall maps to the last cell.
    """
    out = []
    for coordinate, count in zip(point, shape, strict=True):
        index = math.floor(coordinate / dx + INDEX_TOLERANCE)
        out.append(int(min(max(index, 0), count - 1)))
    return tuple(out)


@dataclass(frozen=True)
class Grid:
    """Uniform grid of cubic cells; pressure at centres, velocity on faces.

    Same fields and constructors as the reference ``Grid`` (``src/ac_fdtd/grid.py:48-163``).
    """

    dx: float
    nx: int
    ny: int
    nz: int
    requested_lengths: tuple[float, float, float] | None = None

    def __post_init__(self) -> None:
        if self.dx <= 0.0:
            raise ValueError(f"dx must be positive, got {self.dx}")
        if min(self.nx, self.ny, self.nz) < 1:
            raise ValueError(f"cell counts must be >= 1, got {self.shape}")

    @classmethod
    def from_lengths(cls, lengths, dx: float) -> Grid:
        counts = [max(1, round(length / dx)) for length in lengths]
        return cls(dx=dx, nx=counts[0], ny=counts[1], nz=counts[2],
                   requested_lengths=tuple(lengths))

    @classmethod
    def from_max_frequency(cls, lengths, max_frequency: float, sound_speed: float,
                           points_per_wavelength: float = 10.0) -> Grid:
        if max_frequency <= 0.0:
            raise ValueError(f"max_frequency must be positive, got {max_frequency}")
        if points_per_wavelength <= 0.0:
            raise ValueError(f"points_per_wavelength must be positive, got {points_per_wavelength}")
        return cls.from_lengths(lengths, sound_speed / (points_per_wavelength * max_frequency))

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.nx, self.ny, self.nz)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def lengths(self) -> tuple[float, float, float]:
        return (self.nx * self.dx, self.ny * self.dx, self.nz * self.dx)

    @property
    def length_error(self) -> tuple[float, float, float]:
        if self.requested_lengths is None:
            return (0.0, 0.0, 0.0)
        return tuple(s - r for s, r in zip(self.lengths, self.requested_lengths, strict=True))

    def velocity_shape(self, axis: int) -> tuple[int, int, int]:
        shape = list(self.shape)
        shape[axis] += 1
        return tuple(shape)

    def cell_index(self, point) -> tuple[int, int, int]:
        return cell_index(self.dx, self.shape, point)

    def cell_centres(self, axis: int) -> np.ndarray:
        return (np.arange(self.shape[axis]) + 0.5) * self.dx

    def memory_bytes(self, itemsize: int = 8, extra_fields: int = 0) -> int:
        velocity_cells = sum(math.prod(self.velocity_shape(axis)) for axis in range(3))
        return (self.n_cells * (1 + extra_fields) + velocity_cells) * itemsize
