"""Failure detection, on a GPU, in forms that fault nothing.

* A non-finite state: NaN or infinity written into p on the host. Every sweep that writes p
  checks what it writes (one fused multiply-add per value) and raises a bit of the handle's
  status word; ``synchronize`` turns it into ``NativeError`` with status ``ACF_ERR_NUMERIC``,
  and the next ``run`` reports it from the status copied after the previous run, without
  waiting for the device.
* A staged sweep whose copies never arrive: a test hook makes the producer of the first CTA
  leave out one plane's copies and shortens every wait to 10 ms; the consumers' bounded waits
  run out, the kernel returns, and the status reports it. The context stays usable: the same
  solver, hook removed and state reset, then matches the oracle bit for bit.
* An allocation failure injected on the host (``ACF_INJECT_ALLOC_FAILURE``): constructors raise
  ``NativeError`` with status ``ACF_ERR_MEMORY`` and nothing is left allocated.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from ac_fdtd_b200 import AIR, AirAbsorption, CudaAcousticFDTD, Grid, RoomBatch, WallAdmittances
from ac_fdtd_b200._native import NativeError
from oracle.leapfrog import OracleFDTD

pytestmark = pytest.mark.gpu

ERR_MEMORY, ERR_STATE, ERR_NUMERIC = 3, 4, 5
GRID = Grid(dx=0.02, nx=13, ny=11, nz=24)
CONFIG = dict(walls=WallAdmittances.uniform(0.2), air_absorption=AirAbsorption())


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("dtype,scheme", [(np.float32, "fused"), (np.float64, "two_sweeps"),
                                          (np.float32, "staged"), (np.float32, "two_sweeps")])
def test_a_non_finite_pressure_is_reported(dtype, scheme, bad):
    solver = CudaAcousticFDTD(GRID, dtype=dtype, scheme=scheme, **CONFIG)
    solver.run(5)
    solver.synchronize()                      # a finite state reports nothing
    p = solver.p
    p[6, 5, 11] = bad
    solver.run(10)
    with pytest.raises(NativeError) as error:
        solver.synchronize()
    assert error.value.status == ERR_NUMERIC
    solver.close()


def test_the_next_run_reports_it_without_waiting():
    solver = CudaAcousticFDTD(GRID, dtype=np.float32, scheme="fused", **CONFIG)
    solver.velocity[2][3, 3, 3] = np.nan       # a velocity reaches p within a step
    solver.run(4)
    assert solver._lib.acf_synchronize(solver._stream) == 0   # wait, without reading the word
    with pytest.raises(NativeError) as error:
        solver.run(1)
    assert error.value.status == ERR_NUMERIC
    solver.close()


def test_a_batch_reports_a_non_finite_room():
    batch = RoomBatch([dict(grid=GRID, **CONFIG),
                       dict(grid=Grid(dx=0.02, nx=9, ny=8, nz=16), **CONFIG)], dtype=np.float32)
    batch.run(3)
    batch.synchronize()
    p = batch.p(1)
    p[4, 4, 4] = np.nan
    batch.set_field(1, 0, p)
    batch.run(6)
    with pytest.raises(NativeError) as error:
        batch.synchronize()
    assert error.value.status == ERR_NUMERIC
    batch.close()


def test_a_staged_wait_that_runs_out_is_reported_and_the_context_survives():
    oracle = OracleFDTD(GRID, AIR, dtype=np.float32, **CONFIG)
    solver = CudaAcousticFDTD(GRID, dtype=np.float32, **CONFIG)
    solver.set_staging(1, 3, 6, 4)
    solver.set_scheme("staged")
    lib = solver._lib
    assert lib.acf_set_wait_test(solver._handle, 10_000_000, 1) == 0       # 10 ms, plane 1
    solver.run(1)                                  # one direct launch (shorter than a graph)
    with pytest.raises(NativeError) as error:
        solver.synchronize()
    assert error.value.status == ERR_STATE
    # hook off, state reset: the same handle on the same context gives the oracle's bits
    assert lib.acf_set_wait_test(solver._handle, 0, -1) == 0
    solver.reset_state()
    solver.step_index = 0
    initial = np.random.default_rng(2).standard_normal(GRID.shape).astype(np.float32)
    for s in (oracle, solver):
        s.p[:] = initial
        s.add_volume_source((0.05, 0.05, 0.05), np.hanning(9))
        s.add_pressure_receiver((0.2, 0.15, 0.4))
        s.run(30)
    solver.synchronize()
    np.testing.assert_array_equal(solver.p, oracle.p)
    np.testing.assert_array_equal(solver.recorded_pressure, oracle.recorded_pressure)
    # the hook's arguments are checked
    assert lib.acf_set_wait_test(solver._handle, 10, -1) == 1
    assert lib.acf_set_wait_test(solver._handle, 0, -2) == 1
    solver.close()


def test_an_injected_allocation_failure_raises_cleanly(monkeypatch):
    monkeypatch.setenv("ACF_INJECT_ALLOC_FAILURE", "1")
    with pytest.raises(NativeError) as error:
        CudaAcousticFDTD(GRID, dtype=np.float32, **CONFIG)
    assert error.value.status == ERR_MEMORY
    assert "injected" in str(error.value)
    with pytest.raises(NativeError) as error:
        RoomBatch([dict(grid=GRID), dict(grid=GRID)], dtype=np.float64)
    assert error.value.status == ERR_MEMORY
    monkeypatch.setenv("ACF_INJECT_ALLOC_FAILURE", "0")
    solver = CudaAcousticFDTD(GRID, dtype=np.float32, **CONFIG)
    solver.run(3)
    solver.synchronize()
    solver.close()
    monkeypatch.delenv("ACF_INJECT_ALLOC_FAILURE")
    assert "ACF_INJECT_ALLOC_FAILURE" not in os.environ
