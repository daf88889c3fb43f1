"""The pressure-only scheme (second-order wave equation on p alone) on a GPU.

The reference plans this scheme (PLAN.md:52-56, milestone M8) and has no implementation, so its
pins are the oracles the p-v scheme already satisfies: with the velocities eliminated, the
recurrence p^{n+1} = fu (2 p^n + lam2 L p^n) - (fu - fp) p^{n-1} - S^{n-1} + S^n is the p-v
leapfrog exactly in real arithmetic, so pressures and recordings must equal the NumPy oracle's
to rounding (1e-12 of the peak in float64 over hundreds of steps; 1e-4 in float32, the
reference's own float32 bound); its conserved energy stays constant in a rigid box and does not
grow with impedance walls; and rooms with a sponge or air absorption are refused.
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
)
from ac_fdtd_b200._native import NativeError
from oracle.leapfrog import OracleFDTD
from tests.cases import GRID, RECEIVER, SOURCE

pytestmark = pytest.mark.gpu

WALLS = {
    "rigid": None,
    "uniform": WallAdmittances.uniform(0.3),
    "faces": WallAdmittances(x_min=0.2, z_max=0.7),
    "all different": WallAdmittances(0.4, 0.1, 0.0, 0.7, 0.2, 0.05),
}


def close_to_peak(got, want, tol, scale=None):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    peak = np.max(np.abs(want)) if scale is None else scale
    assert peak > 0
    err = np.max(np.abs(got - want))
    assert err <= tol * peak, f"{err / peak:.2e} of the peak"


def pair(grid, walls, dtype=np.float64, seed=0, velocity=False, steps=150):
    rng = np.random.default_rng(seed)
    p0 = rng.standard_normal(grid.shape)
    v0 = [rng.standard_normal(grid.velocity_shape(a)) * 1e-3 for a in range(3)] if velocity else None
    signal = np.exp(-(((np.arange(steps) - 30) / 8.0) ** 2))
    oracle = OracleFDTD(grid, AIR, dtype=np.float64, walls=walls)
    cuda = CudaAcousticFDTD(grid, dtype=dtype, walls=walls, scheme="pressure_only")
    for s in (oracle, cuda):
        s.p[:] = p0
        if v0 is not None:
            for a in range(3):
                s.velocity[a][:] = v0[a]
        s.add_volume_source(SOURCE if grid is GRID else tuple(0.4 * n * grid.dx for n in grid.shape), signal)
        s.add_volume_source(tuple(0.7 * n * grid.dx for n in grid.shape), signal[::-1].copy())
        s.add_pressure_receiver(RECEIVER if grid is GRID else tuple(0.6 * n * grid.dx for n in grid.shape))
    return oracle, cuda


@pytest.mark.parametrize("velocity", [False, True])
@pytest.mark.parametrize("walls", list(WALLS))
def test_pressure_only_equals_the_pv_oracle(walls, velocity):
    oracle, cuda = pair(GRID, WALLS[walls], velocity=velocity)
    oracle.run(300)
    for n in (1, 63, 64, 172):          # the first step, graphs of either parity, a tail
        cuda.run(n)
    close_to_peak(cuda.recorded_pressure, oracle.recorded_pressure, 1e-12)
    close_to_peak(cuda.p, oracle.p, 1e-12)
    cuda.close()


def test_single_precision_is_within_the_references_float32_bound():
    oracle, cuda = pair(GRID, WALLS["faces"], dtype=np.float32)
    oracle.run(300)
    cuda.run(300)
    close_to_peak(cuda.recorded_pressure, oracle.recorded_pressure, 1e-4)
    close_to_peak(cuda.p, oracle.p, 1e-4)


@pytest.mark.parametrize("shape", [(1, 1, 9), (5, 1, 1), (3, 2, 7), (2, 3, 1), (7, 5, 13),
                                   (4, 4, 4), (9, 6, 16)])
def test_odd_and_degenerate_grids(shape):
    grid = Grid(dx=0.02, nx=shape[0], ny=shape[1], nz=shape[2])
    oracle, cuda = pair(grid, WALLS["all different"], seed=sum(shape))
    scale = np.max(np.abs(oracle.p))       # the initial field: tiny rooms lose most of it
    oracle.run(60)
    cuda.run(60)
    close_to_peak(cuda.recorded_pressure, oracle.recorded_pressure, 1e-12, scale)
    close_to_peak(cuda.p, oracle.p, 1e-12, scale)


def test_entering_the_scheme_mid_run():
    """Selected after 37 fused p-v steps, the first pressure-only step starts from (p, v)."""
    walls = WALLS["uniform"]
    oracle, _ = pair(GRID, walls, velocity=True)
    cuda = CudaAcousticFDTD(GRID, walls=walls, scheme="fused")
    cuda.p[:] = np.random.default_rng(0).standard_normal(GRID.shape)
    rng = np.random.default_rng(0)
    rng.standard_normal(GRID.shape)
    for a in range(3):
        cuda.velocity[a][:] = rng.standard_normal(GRID.velocity_shape(a)) * 1e-3
    signal = np.exp(-(((np.arange(150) - 30) / 8.0) ** 2))
    cuda.add_volume_source(SOURCE, signal)
    cuda.add_volume_source(tuple(0.7 * n * GRID.dx for n in GRID.shape), signal[::-1].copy())
    cuda.add_pressure_receiver(RECEIVER)
    oracle.run(37)
    cuda.run(37)
    cuda.set_scheme("pressure_only")
    oracle.run(100)
    cuda.run(100)
    close_to_peak(cuda.recorded_pressure, oracle.recorded_pressure, 1e-12)
    close_to_peak(cuda.p, oracle.p, 1e-12)


def test_energy_is_conserved_in_a_rigid_box_and_decays_with_walls():
    grid = Grid(dx=0.05, nx=24, ny=20, nz=16)
    p0 = np.random.default_rng(3).standard_normal(grid.shape)
    rigid = CudaAcousticFDTD(grid, scheme="pressure_only")
    lossy = CudaAcousticFDTD(grid, walls=WallAdmittances.uniform(0.3), scheme="pressure_only")
    energies = {"rigid": [], "lossy": []}
    for name, s in (("rigid", rigid), ("lossy", lossy)):
        s.p[:] = p0
        for _ in range(40):
            s.run(13)
            energies[name].append(s.energy())
    e = np.array(energies["rigid"])
    assert np.max(np.abs(e - e[0])) <= 1e-12 * e[0]
    e = np.array(energies["lossy"])
    assert np.all(np.diff(e) <= 1e-12 * e[0])
    assert e[-1] < 0.9 * e[0]


def test_refusals_and_what_the_scheme_does_not_keep():
    with pytest.raises(ValueError):
        CudaAcousticFDTD(GRID, absorbing_layer=AbsorbingLayer(thickness=3), scheme="pressure_only")
    with pytest.raises(ValueError):
        CudaAcousticFDTD(GRID, air_absorption=AirAbsorption(), scheme="pressure_only")
    cuda = CudaAcousticFDTD(GRID, walls=WALLS["uniform"], scheme="pressure_only")
    cuda.p[:] = np.random.default_rng(1).standard_normal(GRID.shape)
    cuda.run(5)
    with pytest.raises(NativeError):
        cuda.velocity  # noqa: B018 -- the velocities are not kept
    with pytest.raises(NativeError):
        cuda.energy_terms()
    with pytest.raises(NativeError):
        cuda.set_scheme("fused")
    assert np.isfinite(cuda.energy())
    cuda.reset_state()
    cuda.set_scheme("fused")             # allowed again from rest
    cuda.run(3)
    assert np.all(cuda.p == 0.0)
    cuda.close()


def test_large_room_single_precision_against_double():
    """256^3 fp32 with walls (the L2 plane prefetch on at this size), 400 steps from a source:
    the pressure-only scheme and the fused p-v scheme in fp32, each against the p-v scheme in
    fp64. The second-order form carries p^{n-1} rather than a velocity, so its float32 rounding
    accumulates faster than the p-v form's: it is held to 3e-4 of the peak, the p-v form to 3e-5."""
    grid = Grid(dx=343.2 / 40000.0, nx=256, ny=256, nz=256)
    walls = WallAdmittances(0.11, 0.05, 0.2, 0.31, 0.07, 0.4)
    out = {}
    for scheme, dtype in (("fused", np.float64), ("fused", np.float32), ("pressure_only", np.float32)):
        s = CudaAcousticFDTD(grid, dtype=dtype, walls=walls, scheme=scheme)
        s.add_volume_source((0.4, 0.5, 0.6), np.hanning(40))
        for point in ((1.1, 1.2, 0.9), (0.3, 1.9, 1.7)):
            s.add_pressure_receiver(point)
        s.run(400)
        out[(scheme, np.dtype(dtype).name)] = (s.recorded_pressure.astype(np.float64),
                                               s.p.astype(np.float64))
        s.close()
    double = out[("fused", "float64")]
    for key, tol in ((("fused", "float32"), 3e-5), (("pressure_only", "float32"), 3e-4)):
        close_to_peak(out[key][0], double[0], tol)
        close_to_peak(out[key][1], double[1], tol)
