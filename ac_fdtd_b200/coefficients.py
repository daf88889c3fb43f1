"""The FP64 host coefficient block of one room, rounded the way the reference rounds it.

The reference computes every scheme constant in FP64 and casts it once to the working dtype
with ``dtype.type(...)`` / ``astype(dtype)`` (ac-fdtd ``src/ac_fdtd/scheme.py:127-212``). The
CUDA library takes FP64 values and rounds them to the solver precision once more; for values
already rounded to float32 here that second rounding is exact, so the device sees the same
numbers the NumPy reference multiplies by, in either precision.

Every input object is read by attribute, so the reference's own ``Grid``, ``Medium``,
``WallAdmittances``, ``AbsorbingLayer`` and ``AirAbsorption`` work as well as this package's.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .boundaries import WallAdmittances, layer_profiles, wall_shell
from .grid import max_stable_time_step

__all__ = ["RoomCoefficients", "room_coefficients", "MAX_RELAXATION"]

MAX_RELAXATION = 4


@dataclass
class RoomCoefficients:
    """Everything the two sweeps of one room read, before it crosses the C ABI."""

    shape: tuple[int, int, int]
    dx: float
    dt: float
    dtype: np.dtype
    vel_coef: float
    pres_coef: float
    src_coef: float
    relax_scale: float
    relax_decay: list[float] = field(default_factory=list)
    relax_mean: list[float] = field(default_factory=list)
    relax_gain: list[float] = field(default_factory=list)
    wall_shell: list[np.ndarray] | None = None
    layer_cell: list[np.ndarray] | None = None
    layer_face: list[np.ndarray] | None = None

    @property
    def n_relax(self) -> int:
        return len(self.relax_decay)


def _rounded(dtype: np.dtype, value) -> float:
    """FP64 value of ``dtype.type(value)``: the reference's one rounding to the working dtype."""
    return float(dtype.type(value))


def room_coefficients(grid, medium, courant: float, dtype, walls=None, absorbing_layer=None,
                      air_absorption=None, force_walls: bool = False) -> RoomCoefficients:
    """Host setup of ``AcousticFDTD.__init__`` (``scheme.py:107-212``) as one flat block."""
    if not 0.0 < courant <= 1.0:
        raise ValueError(f"courant must be in (0, 1], got {courant}")
    dtype = np.dtype(dtype)
    if dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError(f"dtype must be float32 or float64, got {dtype}")
    shape = (int(grid.nx), int(grid.ny), int(grid.nz))
    dx = float(grid.dx)
    c = float(medium.sound_speed)
    rho = float(medium.density)
    dt = courant * max_stable_time_step(dx, c)
    walls = walls or WallAdmittances()

    block = RoomCoefficients(
        shape=shape, dx=dx, dt=dt, dtype=dtype,
        vel_coef=_rounded(dtype, dt / (rho * dx)),
        pres_coef=_rounded(dtype, rho * c**2 * dt / dx),
        src_coef=_rounded(dtype, rho * c**2 * dt),
        relax_scale=0.0,
    )

    # Relaxation states (scheme.py:166-191). The gains are summed as working-dtype scalars,
    # exactly as the reference's Python `sum` over its stored gains does.
    if air_absorption is not None:
        processes = air_absorption.processes(c, dt)
        if len(processes) > MAX_RELAXATION:
            raise ValueError(f"the kernel holds at most {MAX_RELAXATION} relaxation processes")
        relaxed_c2 = c**2 / (1.0 + sum(p.strength for p in processes))
        gains = []
        for process in processes:
            decay = math.exp(-dt / process.relaxation_time)
            mean_weight = (process.relaxation_time / dt) * (1.0 - decay)
            gain = dtype.type(rho * relaxed_c2 * process.strength / dx)
            block.relax_decay.append(_rounded(dtype, decay))
            block.relax_mean.append(_rounded(dtype, dt * mean_weight))
            block.relax_gain.append(float(gain))
            gains.append(gain)
        block.relax_scale = _rounded(dtype, dt * sum(gains))

    block.wall_shell = wall_shell(shape, c, dt, dx, walls, force_walls)
    if absorbing_layer is not None:
        block.layer_cell, block.layer_face = layer_profiles(shape, dx, c, dt, absorbing_layer)
    return block
