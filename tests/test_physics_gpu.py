"""The reference's physics oracles, run on the CUDA backend.

Each test restates one of ac-fdtd's own solver tests with ``CudaAcousticFDTD`` in place of
``AcousticFDTD``: exact energy conservation (``tests/test_scheme.py:28-42``), pure box modes
(``:75-98``), passive walls and layer (``tests/test_boundaries.py:196-219``), the
(1 - xi)/(1 + xi) reflection in a duct (``:242-273``) and ISO attenuation in a long duct
(``tests/test_air.py:364-397``). Then the two benchmark rooms at their full sizes.
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
    WallAdmittances,
    admittance_from_absorption,
    gaussian_derivative_pulse,
    gaussian_pulse,
)
from tests.physics import discrete_mode_frequency, mode_initial_state, mode_pressure_field

pytestmark = pytest.mark.gpu


def _box(dx=0.05, lengths=(0.8, 0.65, 0.55), courant=1.0, **kw):
    return CudaAcousticFDTD(Grid.from_lengths(lengths, dx), courant=courant, **kw)


@pytest.mark.parametrize("courant", [1.0, 0.9, 0.5])
def test_energy_is_conserved_to_round_off(courant):
    solver = _box(courant=courant)
    solver.p[:] = np.random.default_rng(1).standard_normal(solver.grid.shape)
    initial = solver.energy()
    drift = []
    for _ in range(40):
        solver.run(50)
        drift.append(abs(solver.energy() - initial) / initial)
    assert max(drift) < 1e-11


@pytest.mark.parametrize("mode", [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 1, 1), (3, 2, 1)])
def test_a_single_mode_stays_exactly_sinusoidal(mode):
    solver = _box(dx=0.04)
    frequency = discrete_mode_frequency(solver.grid, mode, AIR.sound_speed, solver.dt)
    shape = mode_pressure_field(solver.grid, mode)
    pressure, velocity = mode_initial_state(solver.grid, mode, AIR, solver.dt)
    solver.p[:] = pressure
    for axis in range(3):
        solver.velocity[axis][:] = velocity[axis]
    # Record the whole field through receivers would be heavy; probe every 10th step exactly.
    errors = []
    for _ in range(60):
        solver.run(10)
        expected = np.cos(2 * np.pi * frequency * solver.time) * shape
        errors.append(np.max(np.abs(solver.p - expected)))
    assert max(errors) < 1e-11


@pytest.mark.parametrize("xi", [0.1, 0.5, 1.0, 3.0])
def test_absorbing_walls_are_passive(xi):
    solver = _box(walls=WallAdmittances.uniform(xi))
    solver.p[:] = np.random.default_rng(3).standard_normal(solver.grid.shape)
    energies = [solver.energy()]
    for _ in range(60):
        solver.run(10)
        energies.append(solver.energy())
    energies = np.array(energies)
    assert np.all(np.diff(energies) <= 0.0)
    assert energies[-1] < 0.5 * energies[0]


def test_the_absorbing_layer_is_passive_and_empties_the_domain():
    solver = _box(absorbing_layer=AbsorbingLayer(thickness=6, target_reflection=1e-4))
    solver.p[:] = np.random.default_rng(3).standard_normal(solver.grid.shape)
    energies = [solver.energy()]
    for _ in range(60):
        solver.run(10)
        energies.append(solver.energy())
    energies = np.array(energies)
    assert np.all(np.diff(energies) <= 0.0)
    assert energies[-1] < 1e-6 * energies[0]


def test_zero_admittance_reproduces_the_rigid_solver_exactly():
    rigid = _box()
    explicit = _box(walls=WallAdmittances.uniform(0.0))
    initial = np.random.default_rng(3).standard_normal(rigid.grid.shape)
    for solver in (rigid, explicit):
        solver.p[:] = initial
        solver.run(50)
    assert np.array_equal(rigid.p, explicit.p)


def test_no_absorption_leaves_the_scheme_untouched():
    grid = Grid.from_lengths((0.4, 0.35, 0.3), 0.05)
    plain = CudaAcousticFDTD(grid)
    disabled = CudaAcousticFDTD(grid, air_absorption=AirAbsorption(classical=False, relaxation=False))
    for solver in (plain, disabled):
        solver.p[:] = np.random.default_rng(5).standard_normal(grid.shape)
        solver.run(40)
    assert np.array_equal(plain.p, disabled.p)


def test_absorbing_air_removes_energy():
    grid = Grid.from_lengths((0.4, 0.35, 0.3), 0.02)
    solver = CudaAcousticFDTD(grid, air_absorption=AirAbsorption())
    solver.p[:] = np.random.default_rng(6).standard_normal(grid.shape)
    initial = solver.energy()
    solver.run(400)
    assert 0.0 < solver.energy() < initial


@pytest.mark.parametrize(("xi", "expected"), [(0.0, 1.0), (0.25, 0.6), (0.5, 1.0 / 3.0), (1.0, 0.0)])
def test_normal_incidence_reflection_matches_theory(xi, expected):
    dx = 0.01
    solver = CudaAcousticFDTD(Grid(dx=dx, nx=600, ny=1, nz=1),
                              walls=WallAdmittances(x_min=1.0, x_max=xi))
    n_steps, width = 2600, 60.0
    index = np.arange(n_steps)
    solver.add_volume_source((1.0, 0.005, 0.005), np.exp(-(((index - 4 * width) / width) ** 2)))
    solver.add_pressure_receiver((2.0, 0.005, 0.005))
    solver.run(n_steps)
    recorded = solver.recorded_pressure[0]
    window = 1200
    incident = np.fft.rfft(recorded[:window])
    reflected = np.fft.rfft(recorded[1300: 1300 + window])
    frequencies = np.fft.rfftfreq(window, solver.dt)
    band = (frequencies > 80.0) & (frequencies < 800.0)
    measured = np.mean(np.abs(reflected[band] / incident[band]))
    assert measured == pytest.approx(expected, abs=0.03)


@pytest.mark.parametrize("frequency", [2000.0, 4000.0])
def test_measured_attenuation_matches_iso(frequency):
    dx = 0.003
    air = AirAbsorption(temperature=20.0, relative_humidity=50.0)
    solver = CudaAcousticFDTD(Grid(dx=dx, nx=3000, ny=1, nz=1),
                              walls=WallAdmittances(x_min=1.0, x_max=1.0), air_absorption=air)
    n_steps, width = 5200, 4.0
    index = np.arange(n_steps)
    solver.add_volume_source((0.5, dx / 2, dx / 2), np.exp(-(((index - 4 * width) / width) ** 2)))
    near, far = 1.5, 8.0
    solver.add_pressure_receiver((near, dx / 2, dx / 2))
    solver.add_pressure_receiver((far, dx / 2, dx / 2))
    solver.run(n_steps)
    recorded = solver.recorded_pressure
    spectra = np.abs(np.fft.rfft(recorded, axis=1))
    frequencies = np.fft.rfftfreq(n_steps, solver.dt)
    b = int(np.argmin(np.abs(frequencies - frequency)))
    measured = -20.0 * np.log10(spectra[1, b] / spectra[0, b]) / (far - near)
    assert measured == pytest.approx(float(air.attenuation(frequencies[b])), rel=0.05)


def test_plain_room_64_cubed_matches_the_oracle():
    """The plain-method room at its full size: 64^3 fp64, alpha 0.15, 2000 steps."""
    from oracle.leapfrog import OracleFDTD

    dx = 343.2 / (10 * 1000.0)
    grid = Grid(dx=dx, nx=64, ny=64, nz=64)
    walls = WallAdmittances.from_absorption(0.15)
    n_steps = 2000
    cuda = CudaAcousticFDTD(grid, walls=walls)
    oracle = OracleFDTD(grid, AIR, walls=walls)
    signal = gaussian_derivative_pulse(n_steps, cuda.dt, 1000.0)
    for solver in (cuda, oracle):
        solver.add_volume_source(tuple((i + 0.5) * dx for i in (16, 16, 20)), signal)
        solver.add_pressure_receiver(tuple((i + 0.5) * dx for i in (44, 40, 24)))
    cuda.run(n_steps)
    oracle.run(n_steps)
    np.testing.assert_array_equal(cuda.recorded_pressure, oracle.recorded_pressure)
    np.testing.assert_array_equal(cuda.p, oracle.p)


def test_large_room_single_precision_error_against_double():
    """384^3, walls + two-face 16-cell sponge + ISO air, fp32 vs fp64 on the receivers.

    The full-size check of the fp32 production path: relative L2 receiver error <= 1e-5
    against the fp64 run (which matches the reference bitwise at every size tested).
    """
    rng = np.random.default_rng(384)
    n = 384
    dx = 343.2 / (10 * 4000.0)
    grid = Grid(dx=dx, nx=n, ny=n, nz=n)
    walls = WallAdmittances(*[admittance_from_absorption(a) for a in rng.uniform(0.05, 0.5, 6)])
    layer = AbsorbingLayer(thickness=16, faces=((0, 0), (0, 1)))
    air = AirAbsorption(temperature=20.0, relative_humidity=50.0)
    cells = [tuple(int(v) for v in rng.integers(32, n - 32, 3)) for _ in range(5)]
    points = [tuple((i + 0.5) * dx for i in c) for c in cells]
    n_steps = 1500
    recordings = {}
    for dtype in (np.float64, np.float32):
        solver = CudaAcousticFDTD(grid, dtype=dtype, walls=walls, absorbing_layer=layer,
                                  air_absorption=air)
        solver.add_volume_source(points[0], gaussian_pulse(n_steps, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)
        solver.run(n_steps)
        recordings[dtype] = solver.recorded_pressure.astype(np.float64)
        solver.close()
    ref, single = recordings[np.float64], recordings[np.float32]
    for r in range(4):
        rel_l2 = np.linalg.norm(single[r] - ref[r]) / np.linalg.norm(ref[r])
        assert rel_l2 <= 1e-5, (r, rel_l2)
