"""A room cut into x slabs against the same room on one solver, on a GPU.

Every part runs the whole room's arithmetic on its planes, so owned cells, faces and
recordings equal the single-solver run bit for bit -- in both precisions and both step
schemes, for slabs of one plane each, with walls, a layer and sources and receivers on either
side of the cuts -- and therefore the oracle.
"""

from __future__ import annotations

import socket

import numpy as np
import pytest

from ac_fdtd_b200 import (
    AIR,
    AbsorbingLayer,
    AirAbsorption,
    CudaAcousticFDTD,
    Grid,
    WallAdmittances,
    gaussian_pulse,
)
from ac_fdtd_b200.slabs import DistributedSlabRoom, SlabGroup
from oracle.leapfrog import OracleFDTD

pytestmark = pytest.mark.gpu

GRID = Grid(dx=0.05, nx=13, ny=9, nz=11)
CONFIG = dict(walls=WallAdmittances(0.3, 0.1, 0.7, 0.05, 0.2, 0.5),
              absorbing_layer=AbsorbingLayer(thickness=3, faces=((0, 0), (0, 1), (1, 1))),
              air_absorption=AirAbsorption())
SOURCES = [((0.12, 0.2, 0.3), 2000.0), ((0.58, 0.33, 0.21), 1500.0)]
RECEIVERS = [(0.03, 0.4, 0.5), (0.31, 0.11, 0.07), (0.33, 0.2, 0.3), (0.64, 0.44, 0.52)]


def populate(solver_like, steps):
    for point, f_max in SOURCES:
        solver_like.add_volume_source(point, gaussian_pulse(steps, solver_like.dt, f_max))
    for point in RECEIVERS:
        solver_like.add_pressure_receiver(point)


def start_from(group, initial):
    for s in group.slabs:
        s.owned(s.solver.p)[:] = initial[s.x0:s.x1]


def assert_same(group, whole):
    np.testing.assert_array_equal(group.p, whole.p)
    for got, want in zip(group.velocity, whole.velocity, strict=True):
        np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(group.recorded_pressure, whole.recorded_pressure)


@pytest.mark.parametrize("scheme", ["two_sweeps", "fused"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("parts", [2, 3, 13])
def test_slabs_equal_the_whole_room_bitwise(parts, dtype, scheme):
    steps = 60
    whole = CudaAcousticFDTD(GRID, dtype=dtype, scheme=scheme, **CONFIG)
    group = SlabGroup(GRID, dtype=dtype, parts=parts, scheme=scheme, **CONFIG)
    initial = np.random.default_rng(parts).standard_normal(GRID.shape).astype(dtype)
    whole.p[:] = initial
    start_from(group, initial)
    populate(whole, steps)
    populate(group, steps)
    whole.run(steps)
    group.run(23)          # in pieces: the exchange at the start of a run sees the same state
    group.run(steps - 23)
    assert group.step_index == steps
    assert_same(group, whole)
    # energy: every part's sums over its owned cells and faces add up to the whole room's
    assert group.energy() == pytest.approx(whole.energy(), rel=1e-11, abs=0)
    group.close()
    whole.close()


def test_slabs_match_the_oracle():
    steps = 40
    oracle = OracleFDTD(GRID, AIR, dtype=np.float64, **CONFIG)
    group = SlabGroup(GRID, dtype=np.float64, parts=4, **CONFIG)
    populate(oracle, steps)
    populate(group, steps)
    oracle.run(steps)
    group.run(steps)
    np.testing.assert_array_equal(group.p, oracle.p)
    np.testing.assert_array_equal(group.recorded_pressure, oracle.recorded_pressure)
    group.close()


def test_energy_over_plane_ranges_adds_up_to_the_room():
    whole = CudaAcousticFDTD(GRID, dtype=np.float64, **CONFIG)
    populate(whole, 25)
    whole.run(25)
    terms = whole.energy_terms()
    np.testing.assert_array_equal(whole.energy_terms(planes=(0, GRID.nx)), terms)
    for cut in (1, 6, 12):
        parts = whole.energy_terms(planes=(0, cut)) + whole.energy_terms(planes=(cut, GRID.nx))
        for got, want in zip(parts, terms, strict=True):   # another summation order only
            assert got == pytest.approx(want, rel=1e-9)
    without_far = whole.energy_terms(planes=(0, GRID.nx), far_face=False)
    np.testing.assert_array_equal(without_far[[0, 2, 3, 4, 5, 6]], terms[[0, 2, 3, 4, 5, 6]])
    assert without_far[1] <= terms[1]
    with pytest.raises(RuntimeError):
        whole.energy_terms(planes=(3, GRID.nx + 1))
    whole.close()


def test_plane_views_address_the_solvers_planes():
    group = SlabGroup(GRID, dtype=np.float32, parts=3, **CONFIG)
    populate(group, 10)
    group.run(10)
    for s in group.slabs:
        _, strides = s.solver.field_pointer(0)
        for plane in (s.first_owned, s.last_owned):
            view = s.plane_view(plane).cpu().numpy().reshape(GRID.ny + 1, strides[1])
            np.testing.assert_array_equal(view[:GRID.ny, :GRID.nz], s.solver.p[plane])
    group.close()


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def test_a_one_rank_distributed_room_is_the_whole_room():
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        steps = 30
        room = DistributedSlabRoom(GRID, dtype=np.float32, **CONFIG)
        whole = CudaAcousticFDTD(GRID, dtype=np.float32, **CONFIG)
        populate(room, steps)
        populate(whole, steps)
        room.run(steps)
        whole.run(steps)
        np.testing.assert_array_equal(room.p, whole.p)
        np.testing.assert_array_equal(room.gather_recordings(), whole.recorded_pressure)
        assert room.energy() == whole.energy()
        room.close()
    finally:
        dist.destroy_process_group()


def test_the_slab_runner_refuses_parts_that_do_not_fit():
    import ctypes

    from ac_fdtd_b200 import _native

    group = SlabGroup(GRID, dtype=np.float32, parts=2, **CONFIG)
    lib = _native.library()
    handles = (ctypes.c_void_p * 2)(*[s.solver._handle.value for s in group.slabs])
    good_lo = [s.first_owned for s in group.slabs]
    good_hi = [s.last_owned + 1 for s in group.slabs]
    for lo, hi in (([1, 1], good_hi), (good_lo, [good_hi[0] + 1, good_hi[1]]),
                   (good_lo, [good_hi[0], good_hi[1] - 1])):
        status = lib.acf_run_slabs(handles, 2, (ctypes.c_int32 * 2)(*lo),
                                   (ctypes.c_int32 * 2)(*hi), 1, 0, None)
        assert status == 1          # ACF_ERR_ARGUMENT, before any launch
    group.slabs[1].solver.set_scheme("fused")
    status = lib.acf_run_slabs(handles, 2, (ctypes.c_int32 * 2)(*good_lo),
                               (ctypes.c_int32 * 2)(*good_hi), 1, 0, None)
    assert status == 4              # ACF_ERR_STATE: the runner steps two-sweep parts
    group.close()


def _gpu_count() -> int:
    import torch

    return torch.cuda.device_count() if torch.cuda.is_available() else 0


@pytest.mark.skipif(_gpu_count() < 2, reason="needs two GPUs: peer stores between devices")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_slabs_on_two_gpus_equal_the_whole_room_bitwise(dtype):
    """Parts alternate between GPUs 0 and 1: each pressure sweep stores its boundary planes into
    the neighbour's ghost plane on the other GPU (plain peer stores, no multicast), and the
    steps are ordered by events between the devices."""
    steps = 50
    whole = CudaAcousticFDTD(GRID, dtype=dtype, **CONFIG)
    group = SlabGroup(GRID, dtype=dtype, parts=4, devices=[0, 1], **CONFIG)
    assert {s.solver.device for s in group.slabs} == {0, 1}
    initial = np.random.default_rng(7).standard_normal(GRID.shape).astype(dtype)
    whole.p[:] = initial
    start_from(group, initial)
    populate(whole, steps)
    populate(group, steps)
    whole.run(steps)
    group.run(17)
    group.run(steps - 17)
    assert_same(group, whole)
    # right after a run: the parts' sums must see the neighbours' last peer stores
    assert group.energy() == pytest.approx(whole.energy(), rel=1e-11, abs=0)
    group.close()
    whole.close()


def test_the_slab_runner_refuses_a_stream_for_parts_on_several_gpus():
    import ctypes

    from ac_fdtd_b200 import _native

    if _gpu_count() < 2:
        pytest.skip("needs two GPUs")
    group = SlabGroup(GRID, dtype=np.float32, parts=2, devices=[0, 1], **CONFIG)
    lib = _native.library()
    handles = (ctypes.c_void_p * 2)(*[s.solver._handle.value for s in group.slabs])
    lo = (ctypes.c_int32 * 2)(*[s.first_owned for s in group.slabs])
    hi = (ctypes.c_int32 * 2)(*[s.last_owned + 1 for s in group.slabs])
    assert lib.acf_run_slabs(handles, 2, lo, hi, 1, 0, ctypes.c_void_p(1)) == 1
    group.close()
