"""Two steps per launch (temporal blocking of the fused single-precision sweep) on a GPU.

The reference names this as the step after its fused sweep (ac-fdtd ``src/ac_fdtd/c/acfdtd.c``
lines 12-14) and does not build it, so its pin is the one-step scheme it must equal bit for bit:
the lean single-precision column, itself equal to the oracle's float32 bits. Covered: rooms with
one CTA per x-plane group and with CTAs that wait on neighbours in y and in z, several x groups
(each recomputing the first step one plane past its ends), step counts that leave a tail of
single steps, sources and receivers on a group boundary and on the room's edges, the relaxation
states' second copy, and the bounded waits running out through the test hook.
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
from ac_fdtd_b200._native import ERR_STATE, NativeError
from oracle.leapfrog import OracleFDTD

pytestmark = pytest.mark.gpu

EVERYTHING = dict(walls=WallAdmittances(0.4, 0.1, 0.0, 0.7, 0.2, 0.05),
                  absorbing_layer=AbsorbingLayer(thickness=3),
                  air_absorption=AirAbsorption())


def _solver(grid, blocking, configuration, initial, points, scheme="fused"):
    cuda = CudaAcousticFDTD(grid, dtype=np.float32, scheme=scheme, **configuration)
    if blocking:
        cuda.set_time_blocking(2)
        assert cuda.time_blocking == 2
    cuda.p[:] = initial
    for where, signal in points["sources"]:
        cuda.add_volume_source(where, signal)
    for where in points["receivers"]:
        cuda.add_pressure_receiver(where)
    return cuda


def _points(grid):
    dx = grid.dx
    last = tuple((n - 0.5) * dx for n in grid.shape)
    middle = tuple(0.5 * n * dx for n in grid.shape)
    eighth = (8.5 * dx if grid.nx > 9 else 0.0, middle[1], middle[2])   # an x-group boundary
    return {
        "sources": [((0.0, 0.0, 0.0), np.hanning(12)), (last, np.hanning(7)),
                    (eighth, np.hanning(20))],
        "receivers": [last, (0.0, last[1], 0.0), eighth, middle],
    }


def _same(a, b):
    np.testing.assert_array_equal(a.p, b.p)
    for axis in range(3):
        np.testing.assert_array_equal(a.velocity[axis], b.velocity[axis])
    np.testing.assert_array_equal(a.recorded_pressure, b.recorded_pressure)
    for x, y in zip(a.relaxation_states, b.relaxation_states, strict=True):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("shape", [(13, 11, 24), (1, 1, 4), (2, 9, 4), (6, 1, 8), (40, 12, 16),
                                   (24, 40, 136), (17, 70, 8), (9, 5, 260)])
def test_two_steps_per_launch_equal_the_one_step_sweep_and_the_oracle(shape):
    """One CTA per group, CTAs waiting across y (70 rows) and z (136 and 260 cells: 34 and 65
    chunks of 4, two and three CTAs along z), 5 x groups (40 planes), one-plane rooms; runs of
    1, 3, 4, 7 and 33 steps (tails of single steps, units of four): the float32 bits of the one-
    step sweep and of the oracle, state, recordings and relaxation states."""
    grid = Grid(dx=0.02, nx=shape[0], ny=shape[1], nz=shape[2])
    initial = np.random.default_rng(sum(shape)).standard_normal(shape).astype(np.float32)
    points = _points(grid)
    one = _solver(grid, False, EVERYTHING, initial, points)
    two = _solver(grid, True, EVERYTHING, initial, points)
    oracle = OracleFDTD(grid, AIR, dtype=np.float32, **EVERYTHING)
    oracle.p[:] = initial
    for where, signal in points["sources"]:
        oracle.add_volume_source(where, signal)
    for where in points["receivers"]:
        oracle.add_pressure_receiver(where)
    for n in (1, 3, 4, 7, 33):
        for s in (one, two, oracle):
            s.run(n)
    _same(two, one)
    np.testing.assert_array_equal(two.p, oracle.p)
    np.testing.assert_array_equal(two.recorded_pressure, oracle.recorded_pressure)
    for got, (want, *_rest) in zip(two.relaxation_states, oracle.relax, strict=True):
        np.testing.assert_array_equal(got, want)
    one.close()
    two.close()


@pytest.mark.parametrize("configuration", [
    {},
    {"walls": WallAdmittances.uniform(0.3)},
    {"absorbing_layer": AbsorbingLayer(thickness=4, faces=((0, 0), (0, 1)))},
    {"air_absorption": AirAbsorption(temperature=15.0, relative_humidity=70.0)},
])
def test_each_feature_alone(configuration):
    """Rigid, walls only, the bench's two-face sponge only, air only: the one-step sweep's bits
    over 64 + 6 steps."""
    grid = Grid(dx=0.02, nx=33, ny=21, nz=40)
    initial = np.random.default_rng(4).standard_normal(grid.shape).astype(np.float32)
    points = _points(grid)
    one = _solver(grid, False, configuration, initial, points)
    two = _solver(grid, True, configuration, initial, points)
    for s in (one, two):
        s.run(64)
        s.run(6)
    _same(two, one)


def test_the_setting_survives_schemes_and_resets():
    """Two steps per launch apply while the scheme is "fused"; switching to the two-sweep scheme
    and back, resetting the state, or turning the setting off keeps the bits."""
    grid = Grid(dx=0.02, nx=20, ny=18, nz=28)
    initial = np.random.default_rng(9).standard_normal(grid.shape).astype(np.float32)
    points = _points(grid)
    one = _solver(grid, False, EVERYTHING, initial, points)
    two = _solver(grid, True, EVERYTHING, initial, points)
    for s in (one, two):
        s.run(10)
        s.set_scheme("two_sweeps")
        s.run(5)
        s.set_scheme("fused")
        s.run(9)
    _same(two, one)
    two.set_time_blocking(1)
    assert two.time_blocking == 1
    for s in (one, two):
        s.run(8)
    _same(two, one)
    two.set_time_blocking(2)
    for s in (one, two):
        s.reset_state()
        s.step_index = 0
        s.p[:] = initial
        s.run(12)
    _same(two, one)


def test_refusals():
    grid = Grid(dx=0.02, nx=10, ny=10, nz=15)
    with pytest.raises(NativeError):
        CudaAcousticFDTD(grid, dtype=np.float32).set_time_blocking(2)     # nz not a multiple of 4
    grid = Grid(dx=0.02, nx=10, ny=10, nz=16)
    with pytest.raises(NativeError):
        CudaAcousticFDTD(grid, dtype=np.float64).set_time_blocking(2)     # double precision
    with pytest.raises(NativeError):
        CudaAcousticFDTD(grid, dtype=np.float32).set_time_blocking(3)


def test_a_wait_that_runs_out_is_reported_and_the_handle_recovers():
    """The first CTA stops publishing from plane 2 on (test hook), so its neighbours' waits run
    out after 5 ms each, raise the wait bit and stop waiting; the kernel returns and the run
    reports ERR_STATE. With the hook off and the state reset, the same handle gives the one-step
    sweep's bits again."""
    grid = Grid(dx=0.02, nx=12, ny=40, nz=160)      # 2 x 10 CTAs per x group
    initial = np.random.default_rng(6).standard_normal(grid.shape).astype(np.float32)
    points = _points(grid)
    two = _solver(grid, True, EVERYTHING, initial, points)
    lib = two._lib
    assert lib.acf_set_wait_test(two._handle, 5_000_000, 2) == 0
    two.run(4)
    with pytest.raises(NativeError) as error:
        two.synchronize()
    assert error.value.status == ERR_STATE
    assert lib.acf_set_wait_test(two._handle, 0, -1) == 0
    one = _solver(grid, False, EVERYTHING, initial, points)
    two.reset_state()
    two.step_index = 0
    two.p[:] = initial
    for s in (one, two):
        s.run(9)
    _same(two, one)


def test_a_non_finite_pressure_is_reported():
    grid = Grid(dx=0.02, nx=16, ny=12, nz=20)
    two = _solver(grid, True, {}, np.zeros(grid.shape, np.float32), {"sources": [], "receivers": []})
    p = np.zeros(grid.shape, np.float32)
    p[5, 6, 7] = np.nan
    two.p[:] = p
    two.run(4)
    with pytest.raises(NativeError):
        two.synchronize()


def test_bench_room_thirty_two_steps():
    """The 384^3 bench room (walls, 16-cell sponge on both x faces, three relaxation
    processes, a source and four receivers): 32 steps in 16 two-step launches equal 32 lean
    steps bit for bit (two x groups of 192 planes, 3 x 96 CTAs each)."""
    from ac_fdtd_b200.workloads import plain_room_large

    grid, configuration, source, receivers = plain_room_large()
    out = []
    for blocking in (False, True):
        cuda = CudaAcousticFDTD(grid, dtype=np.float32, scheme="fused", **configuration)
        if blocking:
            cuda.set_time_blocking(2)
        cuda.p[:] = np.random.default_rng(1).standard_normal(grid.shape).astype(np.float32)
        cuda.add_volume_source(source, np.hanning(64))
        for r in receivers:
            cuda.add_pressure_receiver(r)
        cuda.run(32)
        out.append((cuda.p.copy(), cuda.recorded_pressure, [v.copy() for v in cuda.velocity]))
        cuda.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    for a, b in zip(out[0][2], out[1][2], strict=True):
        np.testing.assert_array_equal(a, b)
