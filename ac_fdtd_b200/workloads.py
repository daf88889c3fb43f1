"""Seeded synthetic rooms in the shapes of the benchmark configurations.

No public dataset exists for this path; these generators draw the rooms the benchmarks and the
full-size tests use, from ``numpy.random.default_rng(seed)``:

* ``plain_room_small`` -- 64^3, fp64, absorption 0.15 on all walls, Gaussian-derivative pulse to
  1 kHz at cell (16,16,20), receiver at cell (44,40,24), 2000 steps.
* ``plain_room_large`` -- 384^3, per-wall absorption U(0.05, 0.5), 16-cell sponge on the two x
  faces, ISO air 20 C / 50 % RH (3 relaxation states), Gaussian pulse to 4 kHz, 4 receivers.
* ``differentiable_room`` -- 128^3, six "true" admittances from absorption U(0.05, 0.5), a
  start perturbed by up to +-30 % per wall, Gaussian pulse to 2 kHz, four receivers, 3000 steps.
* ``patch_inversion_rooms`` -- 16 rooms of 96-160 cells per axis, each wall split into 4 x 4
  patches (96 admittances per room, absorption U(0.05, 0.5)), air at 20 C with seeded RH, a
  16-cell sponge on one face, one source and eight receivers per room.
* ``uneven_rooms`` -- 64 rooms, 3-10 m per axis at dx = 5 cm (60-200 cells per axis; the
  reference's 10 points per wavelength at 2 kHz would give 175-583), per-wall absorption
  U(0.05, 0.5), air at U(15, 25) C and U(30, 70) % RH, one source and two receivers at least
  0.5 m from the walls.
"""

from __future__ import annotations

import numpy as np

from .air import AirAbsorption
from .boundaries import AbsorbingLayer, WallAdmittances, admittance_from_absorption
from .grid import Grid

__all__ = ["plain_room_small", "plain_room_large", "uneven_rooms", "differentiable_room",
           "patch_inversion_rooms", "UNEVEN_DX"]

UNEVEN_DX = 0.05


def plain_room_small():
    dx = 343.2 / (10 * 1000.0)
    grid = Grid(dx=dx, nx=64, ny=64, nz=64)
    source = tuple((i + 0.5) * dx for i in (16, 16, 20))
    receiver = tuple((i + 0.5) * dx for i in (44, 40, 24))
    return grid, dict(walls=WallAdmittances.from_absorption(0.15)), source, [receiver]


def plain_room_large(size: int = 384, seed: int = 2, n_receivers: int = 4):
    rng = np.random.default_rng(seed)
    dx = 343.2 / (10 * 4000.0)
    grid = Grid(dx=dx, nx=size, ny=size, nz=size)
    alphas = rng.uniform(0.05, 0.5, 6)
    objects = dict(
        walls=WallAdmittances(*[admittance_from_absorption(a) for a in alphas]),
        absorbing_layer=AbsorbingLayer(thickness=16, faces=((0, 0), (0, 1))),
        air_absorption=AirAbsorption(temperature=20.0, relative_humidity=50.0),
    )
    margin = max(1, min(24, size // 4))
    cells = [tuple(int(v) for v in rng.integers(margin, size - margin, 3))
             for _ in range(1 + n_receivers)]
    points = [tuple((i + 0.5) * dx for i in c) for c in cells]
    return grid, objects, points[0], points[1:]


def uneven_rooms(n_rooms: int = 64, seed: int = 3, dx: float = UNEVEN_DX,
                 lengths=(3.0, 10.0)):
    """List of (spec, source point, [receiver points]) for the uneven-room batch."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_rooms):
        size = rng.uniform(lengths[0], lengths[1], 3)
        grid = Grid.from_lengths(tuple(size), dx)
        alphas = rng.uniform(0.05, 0.5, 6)
        spec = dict(
            grid=grid,
            walls=WallAdmittances(*[admittance_from_absorption(a) for a in alphas]),
            air_absorption=AirAbsorption(temperature=float(rng.uniform(15.0, 25.0)),
                                         relative_humidity=float(rng.uniform(30.0, 70.0))),
        )
        inner = [(0.5, L - 0.5) for L in grid.lengths]
        points = [tuple(float(rng.uniform(lo, hi)) for lo, hi in inner) for _ in range(3)]
        out.append((spec, points[0], points[1:]))
    return out


def differentiable_room(size: int = 128, seed: int = 4, n_receivers: int = 4):
    """(grid, true admittances, start admittances, source point, receiver points)."""
    rng = np.random.default_rng(seed)
    dx = 343.2 / (10 * 2000.0)
    grid = Grid(dx=dx, nx=size, ny=size, nz=size)
    true_xi = np.array([admittance_from_absorption(a) for a in rng.uniform(0.05, 0.5, 6)])
    start_xi = true_xi * (1.0 + rng.uniform(-0.3, 0.3, 6))
    margin = max(1, size // 8)
    cells = [tuple(int(v) for v in rng.integers(margin, size - margin, 3))
             for _ in range(1 + n_receivers)]
    points = [tuple((i + 0.5) * dx for i in c) for c in cells]
    return grid, true_xi, start_xi, points[0], points[1:]


def patch_inversion_rooms(n_rooms: int = 16, seed: int = 5, patches: int = 4,
                          cells=(96, 160), n_receivers: int = 8):
    """List of (spec with true WallPatches, start WallPatches (+-30 %), source, receivers)."""
    from .boundaries import WallPatches

    rng = np.random.default_rng(seed)
    dx = 343.2 / (10 * 2000.0)
    out = []
    for _ in range(n_rooms):
        shape = rng.integers(cells[0], cells[1] + 1, 3)
        grid = Grid(dx=dx, nx=int(shape[0]), ny=int(shape[1]), nz=int(shape[2]))
        alphas = rng.uniform(0.05, 0.5, (6, patches, patches))
        true = WallPatches(np.vectorize(admittance_from_absorption)(alphas))
        start = WallPatches(true.patch_values * (1.0 + rng.uniform(-0.3, 0.3, true.patch_values.shape)))
        face = (int(rng.integers(0, 3)), int(rng.integers(0, 2)))
        spec = dict(grid=grid, walls=true,
                    absorbing_layer=AbsorbingLayer(thickness=16, faces=(face,)),
                    air_absorption=AirAbsorption(temperature=20.0,
                                                 relative_humidity=float(rng.uniform(30.0, 70.0))))
        inner = [(0.2 * L, 0.8 * L) for L in grid.lengths]
        points = [tuple(float(rng.uniform(lo, hi)) for lo, hi in inner) for _ in range(1 + n_receivers)]
        out.append((spec, start, points[0], points[1:]))
    return out
