"""The room workflow's post-processing in FP64 on the GPU against the reference's arithmetic.

The fixtures of ``tests/golden/impulse.npz`` were computed by the reference itself (its
``simulate_impulse_response``: recordings, excitation, deconvolved signals, and the decay
metrics in ``golden.json``). The host functions of ``ac_fdtd_b200.room`` reproduce the
reference's NumPy arithmetic bit for bit (``tests/test_room_workflow.py``), so they stand in
for it on long synthetic responses. The device sums are tree-shaped where NumPy's are
sequential: signals agree to 1e-12 of their peak, decay curves to 1e-9 dB, fitted times and
clarities to 1e-12 relative.
"""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200 import postprocess as device
from ac_fdtd_b200 import room as host
from ac_fdtd_b200.sources import deconvolve as host_deconvolve
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN / "impulse.npz"))


def decaying_noise(channels=4, n=200_000, sample_rate=48_000.0, seed=1):
    rng = np.random.default_rng(seed)
    t = np.arange(n) / sample_rate
    rates = rng.uniform(20.0, 60.0, channels)[:, None]    # T60 between 0.35 and 1 s
    return rng.standard_normal((channels, n)) * np.exp(-rates * t), sample_rate


def test_deconvolution_matches_the_reference(golden, golden_meta):
    meta = golden_meta["impulse"]
    dt = 1.0 / meta["sample_rate"]
    got = device.deconvolve(golden["recorded"], golden["excitation"], dt, meta["max_frequency"])
    want = golden["signals"]
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    one = device.deconvolve(golden["recorded"][1], golden["excitation"], dt, meta["max_frequency"])
    assert np.max(np.abs(one - want[1])) <= 1e-12 * np.max(np.abs(want))


def test_deconvolution_of_long_signals_matches_the_host(golden):
    x, sr = decaying_noise(channels=3, n=65_537)
    excitation = np.zeros(x.shape[1])
    excitation[:40] = np.hanning(40)
    got = device.deconvolve(x, excitation, 1.0 / sr, 9000.0)
    want = host_deconvolve(x, excitation, 1.0 / sr, 9000.0)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_decay_metrics_match_the_reference(golden, golden_meta):
    meta = golden_meta["impulse"]
    f = meta["formulae"]
    sr = meta["sample_rate"]
    s = golden["signals"][0]
    assert device.reverberation_time(s, sr, 20.0) == pytest.approx(f["t20"], rel=1e-12)
    assert device.early_decay_time(s, sr) == pytest.approx(f["edt"], rel=1e-12)
    assert device.clarity(s, sr, split=0.002) == pytest.approx(f["c2ms"], rel=1e-12)


def test_schroeder_curves_match_the_host_on_long_responses():
    x, sr = decaying_noise()
    got = device.schroeder_decay(x)
    want = host.schroeder_decay(x)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-9
    assert np.all(got[:, 0] == 0.0)
    for c in range(x.shape[0]):
        np.testing.assert_allclose(device.schroeder_decay(x[c]), got[c], rtol=0, atol=1e-12)


def test_fitted_times_and_clarity_match_the_host_on_long_responses():
    x, sr = decaying_noise()
    t20 = device.reverberation_time(x, sr, 20.0)
    t30 = device.reverberation_time(x, sr, 30.0)
    edt = device.early_decay_time(x, sr)
    c50 = device.clarity(x, sr, 0.05)
    for c in range(x.shape[0]):
        assert t20[c] == pytest.approx(host.reverberation_time(x[c], sr, 20.0), rel=1e-12)
        assert t30[c] == pytest.approx(host.reverberation_time(x[c], sr, 30.0), rel=1e-12)
        assert edt[c] == pytest.approx(host.early_decay_time(x[c], sr), rel=1e-12)
        assert c50[c] == pytest.approx(host.clarity(x[c], sr, 0.05), rel=1e-12)


def test_a_decay_too_short_to_fit_is_refused_as_the_reference_does():
    x = np.exp(-np.arange(100) / 5000.0)      # the curve reaches -5 dB, never -25 dB
    with pytest.raises(ValueError):
        host.reverberation_time(x, 1000.0, 20.0)
    with pytest.raises(ValueError):
        device.reverberation_time(x, 1000.0, 20.0)
