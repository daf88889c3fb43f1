"""Parity at the benchmark configurations' own sizes, on a GPU.

The other parity tests run rooms of 20-64 cells per axis. These run the rooms ``bench.py``
times, at their full size, for a bounded number of steps:

* the 384^3 plain-method room (walls drawn per face, a 16-cell sponge on both x faces, ISO air
  with three relaxation states, four seeded receivers), started from seeded random pressure so
  every cell carries signal from the first step, against the reference's own compiled C
  backend (``oracle/_ref``, ac-fdtd ``src/ac_fdtd/c/acfdtd.c:355-376``) on the host cores, in
  float64 (max |difference| <= 1e-13 of the peak, on every receiver and over the whole final
  pressure field) and float32 (<= 1e-5 of the peak). The C loop multiplies the sponge factors
  in another order than the NumPy reference (``scheme.py:285-296``), which the CUDA path
  follows bit for bit, so the two differ by rounding only;
* eight of the 64 uneven rooms of the batched configuration, including the smallest and the
  largest, run as one ``RoomBatch`` and each on its own ``CudaAcousticFDTD`` in float64: equal
  bit for bit; and the smallest room against the reference C backend at 1e-13.
"""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200 import AIR, CudaAcousticFDTD, RoomBatch, gaussian_pulse
from ac_fdtd_b200.workloads import plain_room_large, uneven_rooms
from oracle import ref_c

pytestmark = pytest.mark.gpu

needs_reference_c = pytest.mark.skipif(not ref_c.available(),
                                       reason="oracle/_ref (the reference C backend) not built")

LARGE_STEPS = 120


def _large_room_pair(dtype, scheme):
    grid, objects, source, receivers = plain_room_large(384, 2, 4)
    initial = (np.random.default_rng(11).standard_normal(grid.shape) * 0.01).astype(dtype)
    reference = ref_c.RefCSolver(grid, AIR, dtype=dtype, threads=0, **objects)
    cuda = CudaAcousticFDTD(grid, dtype=dtype, scheme=scheme, **objects)
    signal = gaussian_pulse(LARGE_STEPS, cuda.dt, 4000.0)
    for solver in (reference, cuda):
        solver.p[:] = initial
        solver.add_volume_source(source, signal)
        for point in receivers:
            solver.add_pressure_receiver(point)
    return reference, cuda


def _assert_close_to_peak(got, want, tol):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    peak = np.max(np.abs(want))
    assert peak > 0
    err = np.max(np.abs(got - want))
    assert err <= tol * peak, f"max |difference| {err:.3e} = {err / peak:.2e} of peak {peak:.3e}"


@needs_reference_c
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 1e-5)])
def test_benchmark_room_384_against_the_reference_c_backend(dtype, tol):
    reference, cuda = _large_room_pair(dtype, "fused")
    reference.run(LARGE_STEPS)
    cuda.run(LARGE_STEPS)
    rec_ref = reference.recorded_pressure
    rec_gpu = cuda.recorded_pressure
    assert rec_gpu.shape == rec_ref.shape == (4, LARGE_STEPS)
    for r in range(4):
        _assert_close_to_peak(rec_gpu[r], rec_ref[r], tol)
    _assert_close_to_peak(cuda.p, reference.p, tol)
    # plane sums as well: a shifted or missing plane would show here even where it is small
    _assert_close_to_peak(cuda.p.sum(axis=(1, 2), dtype=np.float64),
                          reference.p.sum(axis=(1, 2), dtype=np.float64), 100 * tol)
    cuda.close()


def test_benchmark_room_384_two_sweeps_equal_fused_bitwise():
    """The bench picks a scheme per shape; both give the same float64 bits at full size."""
    grid, objects, source, receivers = plain_room_large(384, 2, 4)
    initial = np.random.default_rng(12).standard_normal(grid.shape) * 0.01
    out = {}
    for scheme in ("two_sweeps", "fused"):
        cuda = CudaAcousticFDTD(grid, dtype=np.float64, scheme=scheme, **objects)
        cuda.p[:] = initial
        cuda.add_volume_source(source, gaussian_pulse(60, cuda.dt, 4000.0))
        for point in receivers:
            cuda.add_pressure_receiver(point)
        cuda.run(60)
        out[scheme] = (cuda.recorded_pressure, cuda.p.copy())
        cuda.close()
    np.testing.assert_array_equal(out["two_sweeps"][0], out["fused"][0])
    np.testing.assert_array_equal(out["two_sweeps"][1], out["fused"][1])


def _picked_uneven_rooms():
    rooms = uneven_rooms()
    cells = [spec["grid"].n_cells for spec, _, _ in rooms]
    order = np.argsort(cells)
    picked = [int(order[0]), int(order[-1])]
    picked += [int(r) for r in np.random.default_rng(21).choice(
        [int(x) for x in order[1:-1]], 6, replace=False)]
    return [rooms[r] for r in sorted(picked)]


@pytest.mark.parametrize("scheme", ["two_sweeps", "fused"])
def test_uneven_rooms_batch_equals_rooms_alone_bitwise(scheme):
    steps = 100
    rooms = _picked_uneven_rooms()
    sizes = [spec["grid"].n_cells for spec, _, _ in rooms]
    all_sizes = [spec["grid"].n_cells for spec, _, _ in uneven_rooms()]
    assert min(sizes) == min(all_sizes) and max(sizes) == max(all_sizes)
    batch = RoomBatch([spec for spec, _, _ in rooms], dtype=np.float64)
    batch.set_scheme(scheme)
    for r, (spec, source, receivers) in enumerate(rooms):
        batch.add_volume_source(r, source, gaussian_pulse(steps, batch.dt(r), 2000.0))
        for point in receivers:
            batch.add_pressure_receiver(r, point)
    batch.run(steps)
    for r, (spec, source, receivers) in enumerate(rooms):
        alone = CudaAcousticFDTD(spec["grid"], dtype=np.float64, walls=spec["walls"],
                                 air_absorption=spec["air_absorption"], scheme=scheme)
        alone.add_volume_source(source, gaussian_pulse(steps, alone.dt, 2000.0))
        for point in receivers:
            alone.add_pressure_receiver(point)
        alone.run(steps)
        np.testing.assert_array_equal(batch.recorded_pressure(r), alone.recorded_pressure)
        np.testing.assert_array_equal(batch.p(r), alone.p)
        alone.close()
    batch.close()


@needs_reference_c
def test_smallest_uneven_room_against_the_reference_c_backend():
    steps = 300
    rooms = uneven_rooms()
    spec, source, receivers = min(rooms, key=lambda r: r[0]["grid"].n_cells)
    objects = dict(walls=spec["walls"], air_absorption=spec["air_absorption"])
    reference = ref_c.RefCSolver(spec["grid"], AIR, dtype=np.float64, threads=0, **objects)
    batch = RoomBatch([spec], dtype=np.float64)
    signal = gaussian_pulse(steps, batch.dt(0), 2000.0)
    reference.add_volume_source(source, signal)
    batch.add_volume_source(0, source, signal)
    for point in receivers:
        reference.add_pressure_receiver(point)
        batch.add_pressure_receiver(0, point)
    reference.run(steps)
    batch.run(steps)
    got = batch.recorded_pressure(0)
    for r in range(len(receivers)):
        _assert_close_to_peak(got[r], reference.recorded_pressure[r], 1e-13)
    _assert_close_to_peak(batch.p(0), reference.p, 1e-13)
    batch.close()
