"""The allocation-free energy entry point agrees with the ordinary one.

``acf_energy_terms_noalloc`` exists for callers that cannot have this library allocate device
memory: an application that owns the whole device-memory budget and hands out buffers from its
own pool (an audio plug-in host, a game or simulation engine), or a real-time thread where
cudaMalloc/cudaFree could block or synchronize the device. Such a caller keeps the fields in
its own device memory; the entry point works on them with a static scratch array.

This file is collected last on purpose, so that a run stopping at the first failure has run
every other test before it. It passes alone in a fresh process and after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense_device_copy(torch, solver):
    """The solver's fields copied into caller-owned device memory, reference layout."""
    from ac_fdtd_b200 import _native

    lib = _native.library()
    dtype = torch.float64 if solver.dtype == np.float64 else torch.float32
    shapes = [solver.grid.shape] + [solver.grid.velocity_shape(a) for a in range(3)]
    tensors = [torch.empty(shape, dtype=dtype, device="cuda") for shape in shapes]
    torch.cuda.synchronize()
    for field, tensor in enumerate(tensors):
        _native.check(lib.acf_download(solver._handle, field, tensor.data_ptr(), None), "acf_download")
    _native.check(lib.acf_synchronize(None), "acf_synchronize")
    return tensors


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_energy_matches_the_allocating_entry_point(dtype):
    torch = pytest.importorskip("torch")
    from ac_fdtd_b200 import (
        AbsorbingLayer,
        AirAbsorption,
        CudaAcousticFDTD,
        Grid,
        WallAdmittances,
        _native,
    )

    lib = _native.library()
    grid = Grid(dx=0.03, nx=37, ny=29, nz=23)
    solver = CudaAcousticFDTD(grid, dtype=dtype, walls=WallAdmittances(0.2, 0.0, 0.4, 0.1, 0.0, 0.7),
                              absorbing_layer=AbsorbingLayer(thickness=4),
                              air_absorption=AirAbsorption())
    solver.p[:] = np.random.default_rng(11).standard_normal(grid.shape)
    solver.add_volume_source((0.3, 0.3, 0.3), np.hanning(40))
    terms_out = torch.zeros(7, dtype=torch.float64, device="cuda")

    for _ in range(2):  # two calls in a row, each after more steps
        solver.run(45)
        expected = solver.energy_terms()
        p, vx, vy, vz = _dense_device_copy(torch, solver)
        for _call in range(2):
            terms_out.fill_(-1.0)
            torch.cuda.synchronize()
            status = lib.acf_energy_terms_noalloc(
                p.data_ptr(), vx.data_ptr(), vy.data_ptr(), vz.data_ptr(), grid.nx, grid.ny,
                grid.nz, solver.dtype.itemsize, ctypes.c_double(grid.dx), terms_out.data_ptr(),
                None)
            _native.check(status, "acf_energy_terms_noalloc")
            _native.check(lib.acf_synchronize(None), "acf_synchronize")
            got = terms_out.cpu().numpy()
            scale = np.max(np.abs(expected))
            np.testing.assert_allclose(got, expected, rtol=1e-12, atol=1e-12 * scale)
    solver.close()


def test_noalloc_energy_refuses_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from ac_fdtd_b200 import _native

    lib = _native.library()
    buffer = torch.zeros(8, dtype=torch.float64, device="cuda")
    terms = torch.zeros(7, dtype=torch.float64, device="cuda")
    status = lib.acf_energy_terms_noalloc(buffer.data_ptr(), buffer.data_ptr(), buffer.data_ptr(),
                                          buffer.data_ptr(), 4096, 1, 1, 8, ctypes.c_double(0.1),
                                          terms.data_ptr(), None)
    assert status == 1
    assert "exceeds the static scratch" in lib.acf_last_error().decode()
