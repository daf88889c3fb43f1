"""The autograd fixtures (tests/golden/make_golden.py, part ``autograd``): gradients of a linear
receiver loss taken by PyTorch autograd through the reference's Torch backend in float64.

On the CPU: the fixture's forward recording equals the oracle's run of the same room, so the
gradients below belong to the scheme this package reproduces. On the GPU: the hand-written
adjoint kernels give the same gradients -- source signal, initial pressure, six wall
admittances, ISO relaxation strengths and times -- to within the rounding of two different
summation orders."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from ac_fdtd_b200 import AIR, AbsorbingLayer, AirAbsorption, Grid, WallAdmittances
from oracle.leapfrog import OracleFDTD

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def case():
    data = np.load(GOLDEN / "autograd.npz")
    meta = json.loads((GOLDEN / "golden.json").read_text())["autograd"]
    grid = Grid(dx=meta["dx"], nx=meta["shape"][0], ny=meta["shape"][1], nz=meta["shape"][2])
    objects = dict(walls=WallAdmittances(*meta["xi"]),
                   absorbing_layer=AbsorbingLayer(thickness=meta["layer_thickness"]),
                   air_absorption=AirAbsorption(**meta["air"]))
    return data, meta, grid, objects


def test_the_fixture_forward_is_the_oracle_run(case):
    data, meta, grid, objects = case
    oracle = OracleFDTD(grid, AIR, dtype=np.float64, **objects)
    oracle.p[:] = data["p0"]
    oracle.add_volume_source(tuple(meta["source"]), data["signal"])
    for point in meta["receivers"]:
        oracle.add_pressure_receiver(tuple(point))
    oracle.run(meta["steps"])
    np.testing.assert_allclose(oracle.recorded_pressure, data["recording"], rtol=0,
                               atol=1e-12 * np.max(np.abs(data["recording"])))


@pytest.mark.gpu
def test_adjoint_gradients_equal_autograd_through_the_reference(case):
    from ac_fdtd_b200.adjoint import DifferentiableRoom

    data, meta, grid, objects = case
    room = DifferentiableRoom(grid, dtype=np.float64, max_steps=meta["steps"],
                              wrt=("signal", "walls", "air"), **objects)
    room.solver.add_volume_source(tuple(meta["source"]), data["signal"])
    for point in meta["receivers"]:
        room.solver.add_pressure_receiver(tuple(point))
    rec = room.forward(meta["steps"], p0=data["p0"])
    np.testing.assert_allclose(rec, data["recording"], rtol=0,
                               atol=1e-12 * np.max(np.abs(data["recording"])))
    g = room.backward(data["w"])

    def close(got, want, what):
        got, want = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= 1e-9, f"{what}: relative error {err:.3e}"

    close(g.signal[0], data["grad_signal"], "dL/dsignal")
    close(g.initial_p, data["grad_p0"], "dL/dp0")
    close(g.walls, data["grad_xi"], "dL/dxi")
    close(g.strength, data["grad_strength"], "dL/dstrength")
    close(g.relaxation_time, data["grad_relaxation_time"], "dL/dtau")
