"""Parity cases shared by the CPU and GPU tests, built from this package's value types.

The five configurations and the 20x17x15 grid are those of the reference's own backend
parity tests (ac-fdtd ``tests/test_c_backend.py:15-42``, ``tests/test_torch_backend.py:23-53``).
"""

from __future__ import annotations

import numpy as np

from ac_fdtd_b200 import (
    AIR,
    AbsorbingLayer,
    AirAbsorption,
    Grid,
    WallAdmittances,
    admittance_from_absorption,
)

GRID = Grid.from_lengths((0.6, 0.5, 0.45), 0.03)
SOURCE = (0.2, 0.2, 0.2)
RECEIVER = (0.4, 0.3, 0.3)

CONFIGURATIONS = {
    "rigid": {},
    "absorbing walls": {"walls": WallAdmittances.uniform(0.3)},
    "absorbing layer": {"absorbing_layer": AbsorbingLayer(thickness=4)},
    "air absorption": {"air_absorption": AirAbsorption()},
    "everything at once": {
        "walls": WallAdmittances(x_min=0.2, z_max=0.7),
        "absorbing_layer": AbsorbingLayer(thickness=3),
        "air_absorption": AirAbsorption(temperature=15.0, relative_humidity=70.0),
    },
}


def prepare(solver, seed: int = 0):
    """Seeded random p0, the Gaussian source and one receiver, as the reference tests do."""
    solver.p[:] = np.random.default_rng(seed).standard_normal(GRID.shape)
    signal = np.exp(-(((np.arange(200) - 30) / 8.0) ** 2))
    solver.add_volume_source(SOURCE, signal)
    solver.add_pressure_receiver(RECEIVER)
    return solver


def full_room(meta: dict):
    """The walls + two-face sponge + ISO air room of the golden ``rooms.npz``."""
    grid = Grid(dx=meta["dx"], nx=meta["shape"][0], ny=meta["shape"][1], nz=meta["shape"][2])
    walls = WallAdmittances(*[admittance_from_absorption(a) for a in meta["alphas"]])
    layer = AbsorbingLayer(thickness=meta["layer"]["thickness"],
                           faces=tuple(tuple(f) for f in meta["layer"]["faces"]))
    air = AirAbsorption(**meta["air"])
    return grid, dict(walls=walls, absorbing_layer=layer, air_absorption=air)


def plain_room(meta: dict):
    grid = Grid(dx=meta["dx"], nx=meta["shape"][0], ny=meta["shape"][1], nz=meta["shape"][2])
    return grid, dict(walls=WallAdmittances.from_absorption(meta["absorption"]))


__all__ = ["AIR", "GRID", "SOURCE", "RECEIVER", "CONFIGURATIONS", "prepare", "full_room",
           "plain_room"]
