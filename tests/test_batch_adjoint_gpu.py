"""Batched adjoint: every room's gradients equal the single-room adjoint's, bit for bit, and a
patch gradient matches central finite differences (float64)."""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid, WallAdmittances, gaussian_pulse
from ac_fdtd_b200.adjoint import DifferentiableBatch, DifferentiableRoom
from ac_fdtd_b200.boundaries import WallPatches

pytestmark = pytest.mark.gpu

STEPS = 70


def rooms():
    rng = np.random.default_rng(11)
    return [
        dict(grid=Grid(dx=0.05, nx=13, ny=11, nz=9),
             walls=WallPatches(rng.uniform(0.05, 0.6, (6, 2, 2))),
             air_absorption=AirAbsorption(temperature=20.0, relative_humidity=40.0)),
        dict(grid=Grid(dx=0.05, nx=9, ny=14, nz=12), walls=WallAdmittances(0.2, 0.1, 0.3, 0.05, 0.4, 0.15),
             absorbing_layer=AbsorbingLayer(thickness=3, faces=((1, 1),)),
             air_absorption=AirAbsorption(temperature=20.0, relative_humidity=60.0)),
        dict(grid=Grid(dx=0.05, nx=16, ny=7, nz=10),
             walls=WallPatches(rng.uniform(0.05, 0.6, (6, 3, 3))),
             air_absorption=AirAbsorption(temperature=20.0, relative_humidity=50.0)),
    ]


def points(spec, seed):
    rng = np.random.default_rng(seed)
    L = spec["grid"].lengths
    return [tuple(float(rng.uniform(0.2, 0.8)) * x for x in L) for _ in range(4)]


def setup_batch(specs):
    batch = DifferentiableBatch(specs, dtype=np.float64, max_steps=STEPS)
    for r, spec in enumerate(specs):
        pts = points(spec, r)
        batch.batch.add_volume_source(r, pts[0], gaussian_pulse(STEPS, batch.batch.dt(r), 2000.0))
        for p in pts[1:]:
            batch.batch.add_pressure_receiver(r, p)
    return batch


def test_batched_gradients_equal_single_room_gradients():
    specs = rooms()
    batch = setup_batch(specs)
    batch.batch.set_prefetch(True)     # forced on for the batch; the single rooms run without
    recs = batch.forward(STEPS)
    weights = [np.random.default_rng(20 + r).standard_normal(rec.shape) for r, rec in enumerate(recs)]
    grads = batch.backward([w * rec for w, rec in zip(weights, recs, strict=True)])
    for r, spec in enumerate(specs):
        room = DifferentiableRoom(spec["grid"], dtype=np.float64, walls=spec["walls"],
                                  absorbing_layer=spec.get("absorbing_layer"),
                                  air_absorption=spec["air_absorption"], max_steps=STEPS)
        pts = points(spec, r)
        room.solver.add_volume_source(pts[0], gaussian_pulse(STEPS, room.dt, 2000.0))
        for p in pts[1:]:
            room.solver.add_pressure_receiver(p)
        rec = room.forward(STEPS)
        np.testing.assert_array_equal(rec, recs[r])
        single = room.backward(weights[r] * rec)
        np.testing.assert_array_equal(grads[r].walls, single.walls)
        np.testing.assert_array_equal(grads[r].signal, single.signal)
        room.solver.close()


def test_batched_patch_gradient_matches_central_differences():
    specs = rooms()
    batch = setup_batch(specs)
    recs = batch.forward(STEPS)
    weights = [np.random.default_rng(30 + r).standard_normal(rec.shape) for r, rec in enumerate(recs)]
    grads = batch.backward([w * rec for w, rec in zip(weights, recs, strict=True)])

    def loss():
        out = batch.forward(STEPS)
        return sum(0.5 * float(np.sum(w * o**2)) for w, o in zip(weights, out, strict=True))

    values = specs[2]["walls"].patch_values
    checked = ((1, 2, 0), (4, 0, 1), (5, 1, 1))
    fds = []
    for f, a, b in checked:
        h = 1e-6 * values[f, a, b]
        plus, minus = values.copy(), values.copy()
        plus[f, a, b] += h
        minus[f, a, b] -= h
        batch.set_walls(2, WallPatches(plus))
        lp = loss()
        batch.set_walls(2, WallPatches(minus))
        lm = loss()
        fds.append((lp - lm) / (2 * h))
    got = np.array([grads[2].walls[c] for c in checked])
    assert np.max(np.abs(got - np.array(fds))) <= 1e-6 * np.max(np.abs(grads[2].walls)), (got, fds)


@pytest.mark.parametrize("air", [None, AirAbsorption(temperature=21.0, relative_humidity=45.0)])
def test_single_precision_lean_recorded_rooms_equal_the_batch(air):
    """Without air gradients, a single-precision room with nz a multiple of 4 records its forward
    run with the lean one-sweep step (writing the boundary history as it goes) and reverses it
    with the packed adjoint step, while a batch records with two sweeps and reverses with the
    generic adjoint sweeps: recordings and wall and source gradients agree bit for bit, with and
    without relaxation states and a sponge, over an odd number of steps (the state ends in the
    second copy and is moved back), and the final pressure equals a plain run's."""
    from ac_fdtd_b200 import CudaAcousticFDTD

    steps = 71
    specs = [
        dict(grid=Grid(dx=0.05, nx=13, ny=11, nz=12), walls=WallAdmittances(0.3, 0.1, 0.45, 0.2, 0.08, 0.27)),
        dict(grid=Grid(dx=0.05, nx=9, ny=14, nz=16), walls=WallAdmittances(0.2, 0.1, 0.3, 0.05, 0.4, 0.15),
             absorbing_layer=AbsorbingLayer(thickness=3, faces=((1, 1),))),
    ]
    if air is not None:
        specs = [dict(spec, air_absorption=air) for spec in specs]
    batch = DifferentiableBatch(specs, dtype=np.float32, max_steps=steps)
    for r, spec in enumerate(specs):
        pts = points(spec, r)
        batch.batch.add_volume_source(r, pts[0], gaussian_pulse(steps, batch.batch.dt(r), 2000.0))
        for p in pts[1:]:
            batch.batch.add_pressure_receiver(r, p)
    recs = batch.forward(steps)
    weights = [np.random.default_rng(40 + r).standard_normal(rec.shape) for r, rec in enumerate(recs)]
    grads = batch.backward([w * rec.astype(np.float64) for w, rec in zip(weights, recs, strict=True)])
    for r, spec in enumerate(specs):
        pts = points(spec, r)
        room = DifferentiableRoom(spec["grid"], dtype=np.float32, walls=spec["walls"],
                                  absorbing_layer=spec.get("absorbing_layer"), air_absorption=air,
                                  max_steps=steps)
        plain = CudaAcousticFDTD(spec["grid"], dtype=np.float32, walls=spec["walls"],
                                 absorbing_layer=spec.get("absorbing_layer"), air_absorption=air)
        for s in (room.solver, plain):
            s.add_volume_source(pts[0], gaussian_pulse(steps, s.dt, 2000.0))
            for p in pts[1:]:
                s.add_pressure_receiver(p)
        rec = room.forward(steps)
        plain.run(steps)
        np.testing.assert_array_equal(rec, recs[r])
        np.testing.assert_array_equal(room.solver.p, plain.p)
        single = room.backward(weights[r] * rec.astype(np.float64))
        np.testing.assert_array_equal(grads[r].walls, single.walls)
        np.testing.assert_array_equal(grads[r].signal, single.signal)
        room.solver.close()
        plain.close()


@pytest.mark.parametrize("shape", [(2, 3, 4), (5, 1, 8), (1, 6, 12), (7, 6, 16)])
def test_packed_adjoint_on_small_and_degenerate_rooms(shape):
    """The packed single-precision adjoint step on rooms where one chunk is both the bottom and
    the top of its row (nz = 4), with a single row or a single plane, a sponge on every face,
    walls and relaxation states, sources and receivers on the room's corners: recordings and wall
    and source gradients equal the batch's generic adjoint bit for bit."""
    steps = 45
    grid = Grid(dx=0.05, nx=shape[0], ny=shape[1], nz=shape[2])
    spec = dict(grid=grid, walls=WallAdmittances(0.3, 0.1, 0.45, 0.2, 0.08, 0.27),
                absorbing_layer=AbsorbingLayer(thickness=1),
                air_absorption=AirAbsorption(temperature=22.0, relative_humidity=40.0))
    other = dict(spec, grid=Grid(dx=0.05, nx=4, ny=5, nz=8))
    L = grid.lengths
    corner = tuple(0.999 * x for x in L)
    pts = [(0.0, 0.0, 0.0), corner, (0.0, corner[1], 0.0)]
    batch = DifferentiableBatch([spec, other], dtype=np.float32, max_steps=steps)
    for r in range(2):
        batch.batch.add_volume_source(r, pts[0], gaussian_pulse(steps, batch.batch.dt(r), 2000.0))
        for p in pts[1:]:
            batch.batch.add_pressure_receiver(r, p)
    recs = batch.forward(steps)
    w = np.random.default_rng(sum(shape)).standard_normal(recs[0].shape)
    grads = batch.backward([w * recs[0].astype(np.float64), np.zeros_like(recs[1], dtype=np.float64)])
    room = DifferentiableRoom(grid, dtype=np.float32, walls=spec["walls"],
                              absorbing_layer=spec["absorbing_layer"],
                              air_absorption=spec["air_absorption"], max_steps=steps)
    room.solver.add_volume_source(pts[0], gaussian_pulse(steps, room.dt, 2000.0))
    for p in pts[1:]:
        room.solver.add_pressure_receiver(p)
    rec = room.forward(steps)
    np.testing.assert_array_equal(rec, recs[0])
    single = room.backward(w * rec.astype(np.float64))
    np.testing.assert_array_equal(grads[0].walls, single.walls)
    np.testing.assert_array_equal(grads[0].signal, single.signal)
    room.solver.close()
