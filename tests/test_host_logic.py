"""Host-side logic of the Python layer, on the CPU, against a stub of the C ABI.

The stub records every call and answers with success; no device work happens. These tests pin
what the Python layer sends across the boundary: the coefficient block, when sources and
receivers are pushed, how snapshots are flushed before a run, the absolute step offsets, and
the refusal of bad input before any native call.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from ac_fdtd_b200 import (
    AbsorbingLayer,
    AirAbsorption,
    CudaAcousticFDTD,
    Grid,
    RoomBatch,
    WallAdmittances,
    _native,
)


class StubLibrary:
    """Answers every acf_* call with ACF_OK and remembers (name, args)."""

    def __init__(self):
        self.calls = []
        self.handles = 0

    def __getattr__(self, name):
        if not name.startswith("acf_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append((name, args))
            if name in ("acf_create", "acf_batch_create"):
                out = args[-1]
                self.handles += 1
                ctypes.cast(out, ctypes.POINTER(ctypes.c_void_p))[0] = 0x1000 + self.handles
            if name == "acf_device_count":
                ctypes.cast(args[0], ctypes.POINTER(ctypes.c_int))[0] = 1
            if name == "acf_host_alloc":
                nbytes = args[0]
                buffer = ctypes.create_string_buffer(max(int(nbytes), 1))
                self._keep = getattr(self, "_keep", []) + [buffer]
                ctypes.cast(args[1], ctypes.POINTER(ctypes.c_void_p))[0] = ctypes.addressof(buffer)
            if name == "acf_launch_count":
                return 0
            if name == "acf_last_error":
                return b""
            return 0

        return call

    def names(self):
        return [name for name, _ in self.calls]


@pytest.fixture
def stub(monkeypatch):
    lib = StubLibrary()
    monkeypatch.setattr(_native, "_lib", lib)
    monkeypatch.setattr(_native, "library", lambda: lib)
    return lib


GRID = Grid(dx=0.03, nx=20, ny=17, nz=15)


def test_constructor_sends_the_coefficient_block(stub):
    solver = CudaAcousticFDTD(GRID, dtype=np.float32, walls=WallAdmittances.uniform(0.3),
                              absorbing_layer=AbsorbingLayer(thickness=3),
                              air_absorption=AirAbsorption(), scheme="fused")
    create = [args for name, args in stub.calls if name == "acf_create"][0]
    config = ctypes.cast(create[0], ctypes.POINTER(_native.AcfConfig)).contents
    assert (config.nx, config.ny, config.nz, config.precision, config.n_relax) == (20, 17, 15, 4, 3)
    assert config.vel_coef == solver.coefficients.vel_coef
    assert all(bool(config.wall_shell[f]) for f in range(6))
    assert all(bool(config.cell[a]) and bool(config.face[a]) for a in range(3))
    assert stub.names().index("acf_set_scheme") > stub.names().index("acf_create")
    scheme = [args for name, args in stub.calls if name == "acf_set_scheme"][-1]
    assert scheme[1] == _native.SCHEME_FUSED


def test_points_are_pushed_once_and_runs_carry_absolute_offsets(stub):
    solver = CudaAcousticFDTD(GRID)
    solver.add_volume_source((0.2, 0.2, 0.2), np.hanning(10))
    solver.add_pressure_receiver((0.4, 0.3, 0.3))
    solver.run(7)
    solver.run(5)
    names = stub.names()
    assert names.count("acf_set_sources") == 1 and names.count("acf_set_receivers") == 1
    runs = [args for name, args in stub.calls if name == "acf_run"]
    assert [(a[1], a[2]) for a in runs] == [(7, 0), (5, 7)]
    assert solver.step_index == 12
    # a receiver added later starts at the current step
    solver.add_pressure_receiver((0.1, 0.1, 0.1))
    solver.run(1)
    receivers = [args for name, args in stub.calls if name == "acf_set_receivers"][-1]
    starts = ctypes.cast(receivers[3], ctypes.POINTER(ctypes.c_int64))
    assert (starts[0], starts[1]) == (0, 12)


def test_snapshots_written_by_the_caller_are_uploaded_before_the_next_run(stub):
    solver = CudaAcousticFDTD(GRID)
    solver.p[:] = 1.0
    before = stub.names().count("acf_upload")
    solver.run(1)
    uploads = [args for name, args in stub.calls if name == "acf_upload"][before:]
    assert [a[1] for a in uploads] == [_native.FIELD_P]
    assert stub.names().index("acf_run") > stub.names().index("acf_upload")
    solver.run(1)
    assert stub.names().count("acf_upload") == before + 1  # nothing new to flush


def test_bad_input_is_refused_before_the_native_layer(stub):
    with pytest.raises(ValueError, match="courant"):
        CudaAcousticFDTD(GRID, courant=1.2)
    with pytest.raises(ValueError, match="scheme"):
        CudaAcousticFDTD(GRID, scheme="leapfrog")
    with pytest.raises(ValueError, match="dtype"):
        CudaAcousticFDTD(GRID, dtype=np.float16)


def test_a_status_becomes_a_python_exception(monkeypatch):
    class Failing(StubLibrary):
        def __getattr__(self, name):
            if name == "acf_create":
                return lambda *args: 3
            if name == "acf_last_error":
                return lambda: b"cudaMalloc of 8 bytes of state failed"
            return super().__getattr__(name)

    lib = Failing()
    monkeypatch.setattr(_native, "_lib", lib)
    monkeypatch.setattr(_native, "library", lambda: lib)
    with pytest.raises(_native.NativeError, match="out of memory: cudaMalloc"):
        CudaAcousticFDTD(GRID)


def test_batch_sends_one_config_per_room(stub):
    rooms = [dict(grid=Grid(dx=0.05, nx=n, ny=n + 1, nz=n + 2), walls=WallAdmittances.uniform(0.1 * n))
             for n in (4, 5, 6)]
    batch = RoomBatch(rooms, dtype=np.float32)
    create = [args for name, args in stub.calls if name == "acf_batch_create"][0]
    assert create[0] == 3
    configs = ctypes.cast(create[1], ctypes.POINTER(_native.AcfConfig))
    assert [(configs[r].nx, configs[r].ny, configs[r].nz) for r in range(3)] == [(4, 5, 6), (5, 6, 7), (6, 7, 8)]
    batch.add_volume_source(1, (0.1, 0.1, 0.1), np.ones(3))
    batch.run(4)
    assert ("acf_batch_set_sources" in stub.names()) and ("acf_batch_run" in stub.names())


def test_a_device_is_selected_before_the_handle_is_created(stub):
    """With device=, the library's runtime is switched to that GPU before the handle that will
    live there is created; without it, no device call is made."""
    grid = Grid(dx=0.05, nx=6, ny=5, nz=4)
    CudaAcousticFDTD(grid, device=3)
    names = stub.names()
    assert names.index("acf_set_device") < names.index("acf_create")
    assert [args for name, args in stub.calls if name == "acf_set_device"] == [(3,)]
    stub.calls.clear()
    RoomBatch([dict(grid=grid), dict(grid=grid)], device=1)
    names = stub.names()
    assert names.index("acf_set_device") < names.index("acf_batch_create")
    stub.calls.clear()
    CudaAcousticFDTD(grid)
    assert "acf_set_device" not in stub.names()


def test_prefetch_modes_cross_the_boundary_as_minus_one_zero_one(stub):
    solver = CudaAcousticFDTD(GRID, dtype=np.float32)
    batch = RoomBatch([dict(grid=GRID), dict(grid=Grid(dx=0.03, nx=9, ny=8, nz=7))],
                      dtype=np.float32)
    for enabled in (True, False, None):
        solver.set_prefetch(enabled)
        batch.set_prefetch(enabled)
    sent = [args[1] for name, args in stub.calls if name == "acf_set_prefetch"]
    sent_batch = [args[1] for name, args in stub.calls if name == "acf_batch_set_prefetch"]
    assert sent == sent_batch == [1, 0, -1]
