"""The room workflow around the solver: statistical formulae, decay metrics, and
``simulate_impulse_response`` end to end, against what the reference computed for the same room
(``tests/golden/impulse.npz``). On the CPU the solver slot is filled by the oracle; on the GPU by
the CUDA backend, bit for bit in float64."""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200.room import (
    Room,
    clarity,
    early_decay_time,
    reverberation_time,
    simulate_impulse_response,
)
from oracle.leapfrog import OracleFDTD


@pytest.fixture(scope="module")
def impulse(golden_meta):
    return golden_meta["impulse"]


def make_room(meta):
    return Room(tuple(meta["dimensions"]), absorption=meta["absorption"])


def test_statistical_formulae_match_the_reference(impulse):
    room = make_room(impulse)
    f = impulse["formulae"]
    assert room.sabine_reverberation_time() == f["sabine"]
    assert room.eyring_reverberation_time() == f["eyring"]
    assert room.diffuse_absorption == f["diffuse_absorption"]
    assert room.air_coefficient(1000.0) == f["air_coefficient"]


def test_decay_metrics_match_the_reference(impulse):
    data = _golden_impulse()
    f = impulse["formulae"]
    sr = impulse["sample_rate"]
    assert reverberation_time(data["signals"][0], sr, 20.0) == pytest.approx(f["t20"], rel=1e-12)
    assert early_decay_time(data["signals"][0], sr) == pytest.approx(f["edt"], rel=1e-12)
    assert clarity(data["signals"][0], sr, split=0.002) == pytest.approx(f["c2ms"], rel=1e-12)


def _golden_impulse():
    from tests.conftest import GOLDEN

    return dict(np.load(GOLDEN / "impulse.npz"))


def test_workflow_with_the_oracle_solver_reproduces_the_reference(impulse):
    from ac_fdtd_b200 import AIR

    data = _golden_impulse()

    class Oracle(OracleFDTD):
        def __init__(self, grid, medium=AIR, **kw):
            super().__init__(grid, medium, **kw)

    ir = simulate_impulse_response(make_room(impulse), tuple(impulse["source"]),
                                   [tuple(r) for r in impulse["receivers"]],
                                   impulse["max_frequency"], solver_class=Oracle)
    assert list(ir.grid.shape) == impulse["shape"]
    np.testing.assert_array_equal(ir.excitation, data["excitation"])
    np.testing.assert_array_equal(ir.recorded, data["recorded"])
    np.testing.assert_array_equal(ir.signals, data["signals"])


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["two_sweeps", "fused", "staged"])
def test_workflow_on_the_gpu_reproduces_the_reference_bitwise(impulse, scheme):
    data = _golden_impulse()
    ir = simulate_impulse_response(make_room(impulse), tuple(impulse["source"]),
                                   [tuple(r) for r in impulse["receivers"]],
                                   impulse["max_frequency"], scheme=scheme, postprocess="host")
    np.testing.assert_array_equal(ir.recorded, data["recorded"])
    np.testing.assert_array_equal(ir.signals, data["signals"])
    assert ir.sample_rate == impulse["sample_rate"]


@pytest.mark.gpu
def test_workflow_with_device_postprocessing_matches_the_reference(impulse):
    """The default with the CUDA solver: recordings stay on the GPU and are deconvolved there in
    FP64 (cuFFT, this library's spectral division); the reference's signals to 1e-12 of their
    peak, and its decay metrics to 1e-12 relative."""
    data = _golden_impulse()
    ir = simulate_impulse_response(make_room(impulse), tuple(impulse["source"]),
                                   [tuple(r) for r in impulse["receivers"]],
                                   impulse["max_frequency"], scheme="fused")
    np.testing.assert_array_equal(ir.recorded, data["recorded"])
    peak = np.max(np.abs(data["signals"]))
    assert np.max(np.abs(ir.signals - data["signals"])) <= 1e-12 * peak
    f = impulse["formulae"]
    metrics = ir.decay_metrics()
    assert metrics["t20"][0] == pytest.approx(f["t20"], rel=1e-12)
    assert metrics["edt"][0] == pytest.approx(f["edt"], rel=1e-12)
    host = ir.decay_metrics(device=False)
    for name in ("t20", "t30", "edt", "c50", "c80"):
        np.testing.assert_allclose(metrics[name], host[name], rtol=1e-12)   # NaN where both are
