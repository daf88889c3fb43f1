"""Ragged batches of rooms: each room equals its own oracle run bit for bit.

Rooms of different shapes (including a 1-cell duct and sizes that are not multiples of the
vector width) and different physics (rigid, walls, sponge, air at different conditions) are
packed into one persistent launch per sweep; every room's final fields and recordings must be
exactly what the oracle -- and hence the reference -- computes for that room alone.
"""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200 import (
    AIR,
    AbsorbingLayer,
    AirAbsorption,
    CudaAcousticFDTD,
    Grid,
    RoomBatch,
    WallAdmittances,
)
from oracle.leapfrog import OracleFDTD

pytestmark = pytest.mark.gpu


def mixed_rooms(with_air: bool = True):
    shapes = [(20, 17, 15), (9, 13, 31), (33, 8, 6), (40, 1, 1), (16, 16, 16), (7, 5, 3)]
    physics = [
        dict(walls=WallAdmittances.uniform(0.3)),
        dict(absorbing_layer=AbsorbingLayer(thickness=3)),
        dict(walls=WallAdmittances(x_min=0.2, z_max=0.7), absorbing_layer=AbsorbingLayer(thickness=2)),
        dict(walls=WallAdmittances(x_min=1.0, x_max=0.25)),
        dict(),
        dict(walls=WallAdmittances(0.1, 0.2, 0.3, 0.4, 0.5, 0.6)),
    ]
    rooms = []
    for n, (shape, phys) in enumerate(zip(shapes, physics, strict=True)):
        spec = dict(grid=Grid(dx=0.03, nx=shape[0], ny=shape[1], nz=shape[2]), **phys)
        if with_air:
            spec["air_absorption"] = AirAbsorption(temperature=15.0 + 2 * n, relative_humidity=30.0 + 7 * n)
        rooms.append(spec)
    return rooms


def populate(solver_like, room_index, spec, seed):
    """Seeded p0, one source and two receivers; works for a batch room or a single solver."""
    grid = spec["grid"]
    rng = np.random.default_rng(seed)
    p0 = rng.standard_normal(grid.shape)
    lengths = grid.lengths
    source = tuple(0.3 * L for L in lengths)
    receivers = [tuple(0.7 * L for L in lengths), tuple(0.5 * L for L in lengths)]
    signal = np.hanning(25)
    if isinstance(solver_like, RoomBatch):
        solver_like.set_field(room_index, 0, p0.astype(solver_like.dtype))
        solver_like.add_volume_source(room_index, source, signal)
        for point in receivers:
            solver_like.add_pressure_receiver(room_index, point)
    else:
        solver_like.p[:] = p0
        solver_like.add_volume_source(source, signal)
        for point in receivers:
            solver_like.add_pressure_receiver(point)


@pytest.mark.parametrize("scheme", ["two_sweeps", "fused"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("with_air", [True, False])
def test_every_room_matches_its_oracle(dtype, with_air, scheme):
    rooms = mixed_rooms(with_air)
    batch = RoomBatch(rooms, dtype=dtype, steps_per_graph=16, scheme=scheme)
    oracles = []
    for r, spec in enumerate(rooms):
        populate(batch, r, spec, seed=r)
        oracle = OracleFDTD(spec["grid"], AIR, dtype=dtype,
                            **{k: v for k, v in spec.items() if k != "grid"})
        populate(oracle, r, spec, seed=r)
        oracles.append(oracle)
    batch.run(37)
    batch.run(53)
    for oracle in oracles:
        oracle.run(90)
    for r, oracle in enumerate(oracles):
        np.testing.assert_array_equal(batch.p(r), oracle.p, err_msg=f"room {r}")
        for axis, v in enumerate(batch.velocity(r)):
            np.testing.assert_array_equal(v, oracle.velocity[axis], err_msg=f"room {r} v{axis}")
        np.testing.assert_array_equal(batch.recorded_pressure(r), oracle.recorded_pressure)


def test_launch_geometry_does_not_change_results():
    rooms = mixed_rooms(True)
    results = []
    # (scheme, block threads, planes, CTAs per SM, L2 prefetch of the next plane)
    for scheme, *geometry, prefetch in (
            ("two_sweeps", 256, 4, 4, None), ("two_sweeps", 64, 1, 2, None),
            ("two_sweeps", 128, 8, 0, True), ("fused", 128, 16, 8, None),
            ("fused", 32, 3, 1, True), ("fused", 128, 8, 0, None), ("fused", 64, 5, 0, True)):
        batch = RoomBatch(rooms, dtype=np.float32, steps_per_graph=8, scheme=scheme)
        batch.set_launch(*geometry)
        batch.set_prefetch(prefetch)
        for r, spec in enumerate(rooms):
            populate(batch, r, spec, seed=10 + r)
        batch.run(30)
        results.append([batch.p(r) for r in range(len(rooms))] +
                       [batch.recorded_pressure(r) for r in range(len(rooms))])
        batch.close()
    for other in results[1:]:
        for a, b in zip(results[0], other, strict=True):
            np.testing.assert_array_equal(a, b)


def test_batch_room_equals_single_room_solver_and_energy():
    rooms = mixed_rooms(True)
    batch = RoomBatch(rooms, dtype=np.float64)
    singles = []
    for r, spec in enumerate(rooms):
        populate(batch, r, spec, seed=20 + r)
        single = CudaAcousticFDTD(spec["grid"], dtype=np.float64,
                                  **{k: v for k, v in spec.items() if k != "grid"})
        populate(single, r, spec, seed=20 + r)
        singles.append(single)
    batch.run(70)
    for r, single in enumerate(singles):
        single.run(70)
        np.testing.assert_array_equal(batch.p(r), single.p)
        assert batch.energy(r) == pytest.approx(single.energy(), rel=1e-12)


def test_profiled_and_graphed_batch_runs_agree():
    rooms = mixed_rooms(True)
    a = RoomBatch(rooms, dtype=np.float32, steps_per_graph=16)
    b = RoomBatch(rooms, dtype=np.float32, steps_per_graph=0)
    for batch in (a, b):
        for r, spec in enumerate(rooms):
            populate(batch, r, spec, seed=40 + r)
    a.run(64)
    b.profile(True)
    b.run(64)
    velocity_ms, pressure_ms, steps = b.profile_read()
    assert steps == 64 and velocity_ms > 0 and pressure_ms > 0
    for r in range(len(rooms)):
        np.testing.assert_array_equal(a.p(r), b.p(r))
        np.testing.assert_array_equal(a.recorded_pressure(r), b.recorded_pressure(r))


def test_fused_batch_switches_schemes_and_resets():
    """The fused batch alternates every room between two copies of p and v: odd step counts,
    state written between runs, a switch back to the two sweeps, a reset and a fresh run must
    all see the current copy."""
    rooms = mixed_rooms(True)
    batch = RoomBatch(rooms, dtype=np.float64, steps_per_graph=8, scheme="fused")
    oracles = []
    for r, spec in enumerate(rooms):
        populate(batch, r, spec, seed=60 + r)
        oracle = OracleFDTD(spec["grid"], AIR, **{k: v for k, v in spec.items() if k != "grid"})
        populate(oracle, r, spec, seed=60 + r)
        oracles.append(oracle)
    for scheme, n in (("fused", 9), ("fused", 16), ("two_sweeps", 5), ("fused", 3)):
        batch.set_scheme(scheme)
        batch.run(n)
        for oracle in oracles:
            oracle.run(n)
    p1 = np.random.default_rng(1).standard_normal(rooms[1]["grid"].shape)
    batch.set_field(1, 0, p1)
    oracles[1].p[:] = p1
    batch.run(7)
    for oracle in oracles:
        oracle.run(7)
    for r, oracle in enumerate(oracles):
        np.testing.assert_array_equal(batch.p(r), oracle.p, err_msg=f"room {r}")
        np.testing.assert_array_equal(batch.recorded_pressure(r), oracle.recorded_pressure)
    batch.reset_state()
    for r in range(len(rooms)):
        assert not np.any(batch.p(r)) and not any(np.any(v) for v in batch.velocity(r))
