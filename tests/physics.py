"""Closed-form rigid-box solutions used as exact oracles (test helpers).

Restates ac-fdtd ``src/ac_fdtd/analytic.py:218-300``: the discrete dispersion relation of the
staggered leapfrog and the initial state (p^0, v^{-1/2}) that launches exactly one box mode.
"""

from __future__ import annotations

import math

import numpy as np


def mode_frequency(lengths, mode, sound_speed):
    return 0.5 * sound_speed * math.sqrt(sum((o / L) ** 2 for o, L in zip(mode, lengths, strict=True)))


def discrete_mode_frequency(grid, mode, sound_speed, dt):
    """sin(w dt/2) = (c dt/dx) sqrt(sum sin^2(k dx/2))  (analytic.py:242-263)."""
    dx = grid.dx
    lengths = grid.lengths
    spatial = math.sqrt(sum(math.sin(o * math.pi / L * dx / 2.0) ** 2
                            for o, L in zip(mode, lengths, strict=True)))
    return math.asin(sound_speed * dt / dx * spatial) / (math.pi * dt)


def mode_pressure_field(grid, mode):
    field = np.ones(grid.shape)
    for axis, (order, length) in enumerate(zip(mode, grid.lengths, strict=True)):
        profile = np.cos(order * math.pi * grid.cell_centres(axis) / length)
        field = field * profile.reshape([-1 if a == axis else 1 for a in range(3)])
    return field


def mode_initial_state(grid, mode, medium, dt):
    """p^0 = the mode, v^{-1/2} = dt/(2 rho) grad p^0 on interior faces (analytic.py:275-300)."""
    pressure = mode_pressure_field(grid, mode)
    coefficient = dt / (2.0 * medium.density * grid.dx)
    velocity = []
    for axis in range(3):
        component = np.zeros(grid.velocity_shape(axis))
        inner = tuple(slice(1, -1) if a == axis else slice(None) for a in range(3))
        hi = tuple(slice(1, None) if a == axis else slice(None) for a in range(3))
        lo = tuple(slice(None, -1) if a == axis else slice(None) for a in range(3))
        component[inner] = coefficient * (pressure[hi] - pressure[lo])
        velocity.append(component)
    return pressure, velocity
