"""The product's FP64 host setup equals the reference's, bit for bit, in both precisions.

Coefficients are compared with the golden values the reference produced
(``tests/golden/setup.npz``); the wall shells are checked against the reference's sparse wall
list cell by cell. Also mirrors the reference's value-type tests (``tests/test_grid.py``,
``tests/test_boundaries.py:156-170,181-193,222-239``, ``tests/test_air.py:288-340``).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from ac_fdtd_b200 import (
    AIR,
    AbsorbingLayer,
    AirAbsorption,
    Grid,
    WallAdmittances,
    admittance_from_absorption,
    max_stable_time_step,
    reflection_coefficient,
)
from ac_fdtd_b200.boundaries import layer_profiles, wall_cell_coefficients
from ac_fdtd_b200.coefficients import room_coefficients
from tests.test_oracle_golden import realise


def shell_to_sparse(shape, sums):
    """Expand six per-face ``a`` maps into (flat index -> a) for the cells they cover."""
    out = {}
    for f, (axis, side) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1))):
        b, c = [x for x in range(3) if x != axis]
        for ib in range(shape[b]):
            for ic in range(shape[c]):
                idx = [0, 0, 0]
                idx[axis] = 0 if side == 0 else shape[axis] - 1
                idx[b], idx[c] = ib, ic
                flat = (idx[0] * shape[1] + idx[1]) * shape[2] + idx[2]
                value = sums[f][ib, ic]
                if flat in out:
                    assert out[flat] == value  # every face of a corner holds the same sum
                out[flat] = value
    return out


def test_product_setup_is_the_reference_setup(golden_meta, golden_setup):
    for name, case in golden_meta["setup"].items():
        grid = Grid(dx=case["dx"], nx=case["shape"][0], ny=case["shape"][1], nz=case["shape"][2])
        objects = realise(case["spec"])
        block = room_coefficients(grid, AIR, 1.0, np.dtype(case["dtype"]), **objects)
        got = [block.dt, block.vel_coef, block.pres_coef, block.src_coef, block.relax_scale]
        assert np.array_equal(np.array(got), golden_setup[name + "/scalars"]), name
        relax = np.array([block.relax_decay, block.relax_mean, block.relax_gain]).T.reshape(-1, 3)
        assert np.array_equal(relax, golden_setup[name + "/relax"]), name

        walls = objects.get("walls", WallAdmittances())
        sums = wall_cell_coefficients(case["shape"], AIR.sound_speed, block.dt, case["dx"], walls)
        index = golden_setup[name + "/wall_index"]
        a = golden_setup[name + "/wall_a"]
        if sums is None:
            assert index.size == 0
        else:
            sparse = shell_to_sparse(case["shape"], sums)
            nonzero = {k: v for k, v in sparse.items() if v != 0.0}
            assert sorted(nonzero) == index.tolist(), name
            assert np.array_equal(np.array([nonzero[k] for k in index.tolist()]), a), name
            # the pair the kernel reads is 1/(1+a), a/(1+a) in FP64 (scheme.py:156-157)
            for f, shell in enumerate(block.wall_shell):
                pair = shell.reshape(-1, 2)
                flat_a = sums[f].reshape(-1)
                assert np.array_equal(pair[:, 0], 1.0 / (1.0 + flat_a))
                assert np.array_equal(pair[:, 1], flat_a / (1.0 + flat_a))

        if "air_absorption" in objects:
            processes = objects["air_absorption"].processes(AIR.sound_speed, block.dt)
            got = np.array([[p.strength, p.relaxation_time] for p in processes]).reshape(-1, 2)
            assert np.array_equal(got, golden_setup[name + "/processes"]), name
        if "absorbing_layer" in objects:
            for axis in range(3):
                assert np.array_equal(block.layer_cell[axis], golden_setup[name + f"/cell{axis}"])
                assert np.array_equal(block.layer_face[axis], golden_setup[name + f"/face{axis}"])


def test_courant_out_of_range_is_refused():
    for bad in (0.0, -0.5, 1.5):
        with pytest.raises(ValueError, match="courant"):
            room_coefficients(Grid(dx=0.1, nx=2, ny=2, nz=2), AIR, bad, np.float64)


def test_more_than_four_relaxation_processes_is_refused():
    class FiveProcesses:
        def processes(self, c, dt):
            from ac_fdtd_b200 import RelaxationProcess

            return tuple(RelaxationProcess(1e-3, 1e-4) for _ in range(5))

    with pytest.raises(ValueError, match="at most 4"):
        room_coefficients(Grid(dx=0.1, nx=2, ny=2, nz=2), AIR, 1.0, np.float64,
                          air_absorption=FiveProcesses())


# -- value types, after the reference's own tests ------------------------------------------

def test_lengths_report_the_room_actually_simulated():
    grid = Grid.from_lengths((1.75, 1.0, 1.0), dx=0.1)
    assert grid.shape == (18, 10, 10)
    assert grid.lengths[0] == pytest.approx(1.8)
    assert grid.length_error[0] == pytest.approx(0.05)


def test_time_step_is_at_the_courant_limit():
    dt = max_stable_time_step(0.05, AIR.sound_speed)
    assert AIR.sound_speed * dt * math.sqrt(3) / 0.05 == pytest.approx(1.0)


def test_cell_index_clips_and_snaps():
    grid = Grid.from_lengths((1.0, 1.0, 1.0), dx=0.1)
    assert grid.cell_index((0.0, 0.0, 0.0)) == (0, 0, 0)
    assert grid.cell_index((0.55, 0.05, 0.05)) == (5, 0, 0)
    assert grid.cell_index((1.0, 1.0, 1.0)) == (9, 9, 9)
    assert Grid(dx=0.01, nx=200, ny=1, nz=1).cell_index((1.2, 0.0, 0.0))[0] == 120


def test_air_is_the_reference_air():
    assert AIR.sound_speed == pytest.approx(343.2, abs=0.05)
    assert AIR.density == pytest.approx(1.204, abs=0.001)


def test_absorption_and_admittance_are_inverse():
    for absorption in (0.0, 0.1, 0.5, 0.9, 1.0):
        xi = admittance_from_absorption(absorption)
        assert 1.0 - reflection_coefficient(xi) ** 2 == pytest.approx(absorption)


def test_negative_admittance_is_refused():
    with pytest.raises(ValueError, match="generates sound"):
        WallAdmittances(x_min=-0.1)


def test_corner_cells_sum_every_face_they_touch():
    sums = wall_cell_coefficients((3, 3, 3), AIR.sound_speed, 1e-5, 0.1, WallAdmittances.uniform(1.0))
    sparse = shell_to_sparse((3, 3, 3), sums)
    assert len(sparse) == 26
    unit = min(sparse.values())
    counts = np.round(np.array(list(sparse.values())) / unit).astype(int)
    assert list(np.bincount(counts)[1:]) == [6, 12, 8]


def test_the_layer_leaves_the_interior_alone():
    cell, face = layer_profiles((20, 20, 20), 0.05, AIR.sound_speed, 1e-5, AbsorbingLayer(thickness=4))
    for axis in range(3):
        assert np.all(cell[axis][4:-4] == 1.0)
        assert np.any(cell[axis][:4] < 1.0)
        assert np.all(face[axis][5:-5] == 1.0)


def test_iso_landmarks():
    air = AirAbsorption(temperature=20.0, relative_humidity=50.0)
    assert 100.0 < air.nitrogen_relaxation_frequency < 1000.0
    assert 10e3 < air.oxygen_relaxation_frequency < 100e3
    per_km = 1000.0 * air.attenuation(np.array([1000.0, 8000.0]))
    assert 4.0 < per_km[0] < 6.0 and 80.0 < per_km[1] < 130.0
    f = np.geomspace(50.0, 16000.0, 60)
    assert np.max(np.abs(air.model_attenuation(f, AIR.sound_speed, 3.4e-6) / air.attenuation(f) - 1)) < 0.01
    assert len(air.processes(AIR.sound_speed, 3.4e-6)) == 3
    assert len(AirAbsorption(classical=False).processes(AIR.sound_speed, 3.4e-6)) == 2


def test_reference_objects_are_accepted_by_duck_typing():
    """Objects that only carry the reference's attributes configure the solver the same way."""

    class G:
        dx, nx, ny, nz = 0.03, 20, 17, 15

    class W:
        values = (0.2, 0.0, 0.0, 0.0, 0.0, 0.7)

    class L:
        thickness, target_reflection, order = 3, 1e-5, 3.0
        faces = ((0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1))

    ours = room_coefficients(Grid(dx=0.03, nx=20, ny=17, nz=15), AIR, 1.0, np.float32,
                             walls=WallAdmittances(x_min=0.2, z_max=0.7),
                             absorbing_layer=AbsorbingLayer(thickness=3))
    theirs = room_coefficients(G(), AIR, 1.0, np.float32, walls=W(), absorbing_layer=L())
    for f in range(6):
        assert np.array_equal(ours.wall_shell[f], theirs.wall_shell[f])
    for a in range(3):
        assert np.array_equal(ours.layer_cell[a], theirs.layer_cell[a])
